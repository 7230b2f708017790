// LM kernels of the B200 bundle adjuster: linearisation, point elimination (Schur complement),
// back-substitution, parameter update and cost.  See lm.cuh for the data layout.
//
// The arithmetic restates V3D/src/Math/v3d_optimization.cpp:784-1187 (weighting, J^T e, the
// U/V/W/X/Y/Z blocks, damping, update, cost with the old weights) on a point-eliminated system.
// Residuals, weights, gradient and cost are FP64.  The normal-equation blocks are stored in
// `Real` (float in mixed mode, double in FP64 mode); their sums are taken in FP64, except the
// camera-pair Schur sums of the mixed mode, which accumulate in FP32.  All reductions run in a
// fixed order (no floating-point atomics), so results are bit-reproducible run to run.
//
// Per-observation storage differs by precision.  FP32 blocks store the products W_k = A_k^T B_k
// and T_k = W_k Vinv_j (two 4-byte 6x3 blocks), which the Schur, rhs and back-substitution
// kernels gather.  FP64 blocks store B_k instead (2x3) and apply W_k and T_k factor by factor
// (W_k x = A_k^T (B_k x), T_k^T y = Vinv_j B_k^T (A_k y)): the linearisation writes 96 bytes less
// per observation and the point elimination writes no per-observation block at all, against
// 126 instead of 108 FMAs and one more point-block gather per Schur pair.
#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "lm.cuh"
#include "model.cuh"

namespace v3dba {

// ---- layout ---------------------------------------------------------------------------------

__host__ __device__ constexpr int round4(int x) { return (x + 3) & ~3; }
__host__ __device__ constexpr int nsym(int n) { return n * (n + 1) / 2; }

// x elements of T rounded up to whole 16-byte vectors (4 floats, 2 doubles).
template <typename T>
__host__ __device__ constexpr int vround(int x) {
  return sizeof(T) == 4 ? (x + 3) & ~3 : (x + 1) & ~1;
}

// Strides of the blocks stored in `Real`, in whole 16-byte vectors.
template <int DA, int DC, typename Real = float>
struct Lay {
  static constexpr int DCc = DC > 0 ? DC : 1;
  static constexpr int SA = vround<Real>(2 * DA);    // A_k, Real
  static constexpr int SW = round4(3 * DA);          // W_k / T_k, float (FP32 blocks only)
  static constexpr int SC = vround<Real>(2 * DCc);   // C_k, Real
  static constexpr int SG = (DA + 1) & ~1;           // A_k^T r_k, double
  static constexpr int SV = vround<Real>(6);         // V_j / Vinv_j upper triangle, Real
  static constexpr int SY = vround<Real>(3 * DCc);   // Y_j / Vinv_j Y_j, Real
  static constexpr int SU = vround<Real>(DA * DA);   // U_i, Real
  static constexpr int SX = vround<Real>(DA * DCc);  // X_i, Real
  static constexpr int NZ = nsym(DC);
};

// symmetric 3x3 index of the packed upper triangle (00,01,02,11,12,22)
__device__ __forceinline__ int s3(int r, int c) {
  const int a = r < c ? r : c, b = r < c ? c : r;
  return a == 0 ? b : (a == 1 ? 2 + b : 5);
}

template <int N>
__device__ __forceinline__ void vload(const float* __restrict__ p, float (&v)[N]) {
  static_assert(N % 4 == 0, "float vectors are loaded 4 at a time");
  const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
  for (int t = 0; t < N / 4; ++t) {
    const float4 u = __ldg(q + t);
    v[4 * t] = u.x; v[4 * t + 1] = u.y; v[4 * t + 2] = u.z; v[4 * t + 3] = u.w;
  }
}
template <int N>
__device__ __forceinline__ void vload(const double* __restrict__ p, double (&v)[N]) {
  static_assert(N % 2 == 0, "double vectors are loaded 2 at a time");
  const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int t = 0; t < N / 2; ++t) {
    const double2 u = __ldg(q + t);
    v[2 * t] = u.x; v[2 * t + 1] = u.y;
  }
}
template <int N>
__device__ __forceinline__ void vstore(float* p, const float (&v)[N]) {
  float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
  for (int t = 0; t < N / 4; ++t) q[t] = make_float4(v[4 * t], v[4 * t + 1], v[4 * t + 2], v[4 * t + 3]);
}
template <int N>
__device__ __forceinline__ void vstore(double* p, const double (&v)[N]) {
  double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
  for (int t = 0; t < N / 2; ++t) q[t] = make_double2(v[2 * t], v[2 * t + 1]);
}

// Deterministically folds the NV per-block partials of `nblk` blocks (first NS summed, the rest
// maxed), stored value-major: part[t * nblk + b] (see store_partials).  Warp w folds values w,
// w + nwarps, ...: lane l reads blocks l, l + 32, ... in order (coalesced), then a fixed shuffle
// tree.  Every thread receives the results in out[0..NV); smem needs NV doubles.
template <int NV, int NS>
__device__ void fold_partials(const double* __restrict__ part, int nblk, double (&out)[NV], double* smem) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int t = wid; t < NV; t += nw) {
    const bool sum = t < NS;
    double acc = sum ? 0.0 : -1e30;
    for (int b = lane; b < nblk; b += 32) {
      const double u = part[(size_t)t * nblk + b];
      acc = sum ? acc + u : fmax(acc, u);
    }
    acc = sum ? warp_sum(acc) : warp_max(acc);
    if (lane == 0) smem[t] = acc;
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < NV; ++t) out[t] = smem[t];
  __syncthreads();   // smem may be reused right away
}

// The block's NV partials (valid in thread 0) to part[t * nblk + bid] (by default the launch's
// block index and count; a stage run as a block range of a merged launch passes its own).
template <int NV>
__device__ __forceinline__ void store_partials(double* __restrict__ part, const double (&v)[NV], int bid, int nblk) {
  if (threadIdx.x == 0) {
#pragma unroll
    for (int t = 0; t < NV; ++t) part[(size_t)t * nblk + bid] = v[t];
  }
}
template <int NV>
__device__ __forceinline__ void store_partials(double* __restrict__ part, const double (&v)[NV]) {
  store_partials(part, v, (int)blockIdx.x, (int)gridDim.x);
}

// Warp-wide sum of V values (V a multiple of 32) by recursive halving: each of the five
// butterfly stages exchanges half of the remaining values, V - V/32 shuffles in total instead
// of 5V.  Afterwards lane L holds the totals of values [L*V/32, (L+1)*V/32) in v[0 .. V/32).
template <int H, typename T, int V>
__device__ __forceinline__ void rt_stage(T (&v)[V], int lane, int m) {
#pragma unroll
  for (int t = 0; t < H; ++t) {
    const bool up = (lane & m) != 0;
    const T send = up ? v[t] : v[t + H];
    const T keep = up ? v[t + H] : v[t];
    v[t] = keep + __shfl_xor_sync(0xffffffffu, send, m);
  }
}
template <int V, typename T>
__device__ __forceinline__ void warp_reduce_transpose(T (&v)[V]) {
  static_assert(V % 32 == 0, "pad the value count to a multiple of 32");
  const int lane = threadIdx.x & 31;
  rt_stage<V / 2>(v, lane, 16);
  rt_stage<V / 4>(v, lane, 8);
  rt_stage<V / 8>(v, lane, 4);
  rt_stage<V / 16>(v, lane, 2);
  rt_stage<V / 32>(v, lane, 1);
}

__host__ __device__ constexpr int round32(int x) { return (x + 31) & ~31; }

// value layout of the per-camera sums: U (packed upper triangle), ga, X
template <int DA, int DC>
struct CamV {
  static constexpr int NU = nsym(DA);
  static constexpr int NX = DC > 0 ? DA * DC : 0;
  static constexpr int NV = NU + DA + NX;
  static constexpr int VP = round32(NV);
};
// value layout of the per-camera reduced rhs / border sums: W q, T Y
template <int DA, int DC>
struct RhsV {
  static constexpr int NX = DC > 0 ? DA * DC : 0;
  static constexpr int NV = DA + NX;
  static constexpr int VP = round32(NV);
};
template <int DA>
struct SchurV {
  static constexpr int NV = DA * DA;
  static constexpr int VP = round32(NV);
};

// row / column of the packed upper-triangle index u of a DA x DA matrix
template <int DA>
__device__ __forceinline__ void unpack_sym(int u, int& r, int& c) {
  r = 0;
  int start = 0;
  while (u >= start + (DA - r)) { start += DA - r; ++r; }
  c = r + (u - start);
}

// ---- relinearisation --------------------------------------------------------------------

constexpr int kPtThreads = 128;
constexpr int kCamWarps = 4;
// Lanes per point of the track kernels that store or load one block per observation: the lanes of
// a group take the observations of one track in turn, so a warp's 16-byte stores / loads of one
// trip hit runs of consecutive blocks instead of 32 scattered ones (the observations of a track
// are contiguous in the point-major order), at the price of idle lanes on short tracks and of
// the group sums.  Measured on the 200-camera scene (375k observations, tracks of 3-12), in µs
// per launch for 1 / 2 / 4 / 8 lanes: k_linearize FP32 53.8 / 51.3 / 61.1 / 86.8, FP64 105.6 /
// 87.9 / 92.1 / 113.3; k_point_backsub FP32 13.5 / 16.6 / 14.8 / 14.6, FP64 30.2 / 17.7 / 20.8 /
// 21.0; k_point_eliminate was fastest with one lane (23.1 / 49.7) and keeps one.
constexpr int kLinLanes = 2;
template <typename Real>
__host__ __device__ constexpr int backsub_lanes() { return sizeof(Real) == 8 ? 2 : 1; }
constexpr int kMaxPtLanes = 2;

// Sum over the G consecutive lanes of a group (all lanes of the warp take part).
template <int G, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// FP32 blocks store W_k and T_k per observation; FP64 blocks store B_k (see the file header).
template <typename Real>
__host__ __device__ constexpr bool stores_products() { return sizeof(Real) == 4; }
constexpr int kSB = 6;   // stride of B_k (2 x 3 row-major) in doubles

template <int DC>
struct RelinNV {
  static constexpr int NZ = nsym(DC);
  static constexpr int NS = 1 + NZ + DC;   // cost, Z (packed), gc
  static constexpr int NV = NS + 2;        // + max |gb|, max diag V
};

// kLinLanes lanes per point: each linearises every kLinLanes-th observation of the track (FP64),
// stores the weighted blocks, and accumulates its share of V_j, gb_j, Y_j, summed over the group
// at the end in a fixed order; Z, gc and the cost go to per-block partials.
template <int MODEL, int DA, int DC, typename Real>
__global__ void __launch_bounds__(kPtThreads) k_linearize(DevState s, double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  using L = Lay<DA, DC, Real>;
  constexpr int DCc = L::DCc;
  constexpr int NS = RelinNV<DC>::NS, NV = RelinNV<DC>::NV, NZ = L::NZ;
  __shared__ double red[(kPtThreads / 32) * NV];
  const Dims& D = s.d;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int tp = gt / kLinLanes, lig = gt % kLinLanes;
  const int j = tp < D.M ? (s.p_order ? s.p_order[tp] : tp) : D.M;   // longest tracks first (p_order)
  double v[NV];
#pragma unroll
  for (int t = 0; t < NV; ++t) v[t] = (t < NS) ? 0.0 : -1e30;
  double V[6] = {0, 0, 0, 0, 0, 0}, gb[3] = {0, 0, 0}, Y[3][DCc];
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int c = 0; c < DCc; ++c) Y[b][c] = 0.0;
  const bool fixB = j < D.nnB;
  int k0 = 0, k1 = 0;

  if (j < D.M) {
    const double X[3] = {s.cur.X[3 * j], s.cur.X[3 * j + 1], s.cur.X[3 * j + 2]};
    Real* oA = reinterpret_cast<Real*>(s.o_A);
    Real* oC = reinterpret_cast<Real*>(s.o_C);
    k0 = s.p_ptr[j];
    k1 = s.p_ptr[j + 1];
    for (int k = k0 + lig; k < k1; k += kLinLanes) {
      const int i = s.o_cam[k];
      const bool fixA = i < D.nnA;
      Cam cam;
      load_cam<MODEL>(cam, s.cur.R, s.cur.T, s.cur.K, s.cur.dist, i);
      if (MODEL == kModelStereo) load_rig(cam, s.rig, s.o_sub[k]);
      double e[2], A[2][DA], B[2][3], C[2][DCc];
      linearize_obs<MODEL, DA, DC>(cam, X, s.o_meas[2 * k], s.o_meas[2 * k + 1], D.mode, D.cached_ar, e, A, B, C);
      const double w = huber_weight(D.thr, e);
      s.o_w[k] = w;
      v[0] += w * w * (e[0] * e[0] + e[1] * e[1]);
      const double r0 = -w * e[0], r1 = -w * e[1];
      const double wa = fixA ? 0.0 : w, wb = fixB ? 0.0 : w;
#pragma unroll
      for (int r = 0; r < 2; ++r) {
#pragma unroll
        for (int q = 0; q < DA; ++q) A[r][q] *= wa;
#pragma unroll
        for (int q = 0; q < 3; ++q) B[r][q] *= wb;
#pragma unroll
        for (int q = 0; q < DCc; ++q) C[r][q] = (DC > 0 && q >= D.nnC) ? C[r][q] * w : 0.0;
      }
      // per-observation blocks
      {
        Real a[L::SA];
#pragma unroll
        for (int t = 0; t < L::SA; ++t) a[t] = Real(0);
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int q = 0; q < DA; ++q) a[r * DA + q] = Real(A[r][q]);
        vstore(oA + (size_t)k * L::SA, a);
        if constexpr (stores_products<Real>()) {
          float wv[L::SW];
#pragma unroll
          for (int t = 0; t < L::SW; ++t) wv[t] = 0.f;
#pragma unroll
          for (int q = 0; q < DA; ++q)
#pragma unroll
            for (int b = 0; b < 3; ++b) wv[q * 3 + b] = float(A[0][q] * B[0][b] + A[1][q] * B[1][b]);
          vstore(s.o_W + (size_t)k * L::SW, wv);
        } else {
          double bv[kSB];
#pragma unroll
          for (int t = 0; t < kSB; ++t) bv[t] = 0.0;
#pragma unroll
          for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int b = 0; b < 3; ++b) bv[r * 3 + b] = B[r][b];
          vstore(s.o_B + (size_t)k * kSB, bv);
        }
        if (DC > 0) {
          Real cv[L::SC];
#pragma unroll
          for (int t = 0; t < L::SC; ++t) cv[t] = Real(0);
#pragma unroll
          for (int r = 0; r < 2; ++r)
#pragma unroll
            for (int q = 0; q < DCc; ++q) cv[r * DCc + q] = Real(C[r][q]);
          vstore(oC + (size_t)k * L::SC, cv);
        }
        double g[L::SG];
#pragma unroll
        for (int t = 0; t < L::SG; ++t) g[t] = 0.0;
#pragma unroll
        for (int q = 0; q < DA; ++q) g[q] = A[0][q] * r0 + A[1][q] * r1;
        vstore(s.o_ga + (size_t)k * L::SG, g);
      }
      // point sums
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = r; c < 3; ++c) V[s3(r, c)] += B[0][r] * B[0][c] + B[1][r] * B[1][c];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        gb[b] += B[0][b] * r0 + B[1][b] * r1;
#pragma unroll
        for (int c = 0; c < DCc; ++c) Y[b][c] += B[0][b] * C[0][c] + B[1][b] * C[1][c];
      }
      if (DC > 0) {
        int z = 0;
#pragma unroll
        for (int r = 0; r < DCc; ++r)
#pragma unroll
          for (int c = r; c < DCc; ++c) v[1 + z++] += C[0][r] * C[0][c] + C[1][r] * C[1][c];
#pragma unroll
        for (int c = 0; c < DCc; ++c) v[1 + NZ + c] += C[0][c] * r0 + C[1][c] * r1;
      }
    }
  }
  // the group's sums (every lane takes part in the shuffles)
#pragma unroll
  for (int t = 0; t < 6; ++t) V[t] = group_sum<kLinLanes>(V[t]);
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    gb[b] = group_sum<kLinLanes>(gb[b]);
#pragma unroll
    for (int c = 0; c < DCc; ++c) Y[b][c] = DC > 0 ? group_sum<kLinLanes>(Y[b][c]) : 0.0;
  }
  if (j < D.M && lig == 0) {
    Real vv[L::SV];
#pragma unroll
    for (int t = 0; t < L::SV; ++t) vv[t] = t < 6 ? Real(V[t]) : Real(0);
    vstore(reinterpret_cast<Real*>(s.p_V) + (size_t)j * L::SV, vv);
    double g4[4] = {gb[0], gb[1], gb[2], 0.0};
    vstore(s.p_gb + (size_t)j * 4, g4);
    if (DC > 0) {
      Real yv[L::SY];
#pragma unroll
      for (int t = 0; t < L::SY; ++t) yv[t] = Real(0);
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < DCc; ++c) yv[b * DCc + c] = Real(Y[b][c]);
      vstore(reinterpret_cast<Real*>(s.p_Y) + (size_t)j * L::SY, yv);
    }
    if (!fixB && k1 > k0) {
      v[NS] = fmax(fabs(gb[0]), fmax(fabs(gb[1]), fabs(gb[2])));
      v[NS + 1] = fmax(V[0], fmax(V[3], V[5]));
    } else if (!fixB) {
      v[NS] = 0.0;
      v[NS + 1] = 0.0;
    }
  }
  block_reduce<NV, NS>(v, red);
  store_partials(part, v);
}

// One warp per chunk of a camera's observation list: partial U = sum A^T A, ga = sum A^T r,
// X = sum A^T C (FP64 sums); the partials of a camera are folded in chunk order afterwards.
template <int DA, int DC, typename Real>
__global__ void __launch_bounds__(kCamWarps * 32) k_camera_chunks(DevState s, double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  using L = Lay<DA, DC, Real>;
  using CV = CamV<DA, DC>;
  constexpr int DCc = L::DCc;
  const int lane = threadIdx.x & 31;
  const int ch = blockIdx.x * kCamWarps + (threadIdx.x >> 5);
  if (ch >= s.nch_cam) return;
  double acc[CV::VP];
#pragma unroll
  for (int t = 0; t < CV::VP; ++t) acc[t] = 0.0;
  const Real* oA = reinterpret_cast<const Real*>(s.o_A);
  const Real* oC = reinterpret_cast<const Real*>(s.o_C);
  for (int idx = s.cc_beg[ch] + lane; idx < s.cc_end[ch]; idx += 32) {
    const int k = s.c_obs[idx];
    Real a[L::SA];
    vload(oA + (size_t)k * L::SA, a);
    double g[L::SG];
    vload(s.o_ga + (size_t)k * L::SG, g);
    int u = 0;
#pragma unroll
    for (int r = 0; r < DA; ++r) {
      acc[CV::NU + r] += g[r];
#pragma unroll
      for (int c = r; c < DA; ++c)
        acc[u++] += double(a[r]) * double(a[c]) + double(a[DA + r]) * double(a[DA + c]);
    }
    if (DC > 0) {
      Real cv[L::SC];
      vload(oC + (size_t)k * L::SC, cv);
#pragma unroll
      for (int r = 0; r < DA; ++r)
#pragma unroll
        for (int c = 0; c < DCc; ++c)
          acc[CV::NU + DA + r * DCc + c] += double(a[r]) * double(cv[c]) + double(a[DA + r]) * double(cv[DCc + c]);
    }
  }
  warp_reduce_transpose(acc);
#pragma unroll
  for (int t = 0; t < CV::VP / 32; ++t) part[(size_t)ch * CV::VP + lane * (CV::VP / 32) + t] = acc[t];
}

// One warp per camera: folds its chunk partials in order and stores U_i, ga_i, X_i; gradient
// max and max diagonal of the varying cameras go to per-block partials.
template <int DA, int DC, typename Real>
__global__ void __launch_bounds__(kCamWarps * 32) k_camera_finish(DevState s, const double* __restrict__ cpart,
                                                                   double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  using L = Lay<DA, DC, Real>;
  using CV = CamV<DA, DC>;
  constexpr int DCc = L::DCc;
  constexpr int PER = CV::VP / 32;
  __shared__ double red[kCamWarps * 2];
  const Dims& D = s.d;
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * kCamWarps + (threadIdx.x >> 5);
  double v[2] = {-1e30, -1e30};
  if (i < D.N) {
    double sum[PER];
#pragma unroll
    for (int t = 0; t < PER; ++t) sum[t] = 0.0;
    for (int ch = s.cam_cc_ptr[i]; ch < s.cam_cc_ptr[i + 1]; ++ch)
#pragma unroll
      for (int t = 0; t < PER; ++t) sum[t] += cpart[(size_t)ch * CV::VP + lane + 32 * t];
    Real* cU = reinterpret_cast<Real*>(s.c_U) + (size_t)i * L::SU;
    Real* cX = reinterpret_cast<Real*>(s.c_X) + (size_t)i * L::SX;
    double gm = 0.0, dm = -1e30;
#pragma unroll
    for (int t = 0; t < PER; ++t) {
      const int vi = lane + 32 * t;
      if (vi < CV::NU) {
        int r, c;
        unpack_sym<DA>(vi, r, c);
        cU[r * DA + c] = Real(sum[t]);
        cU[c * DA + r] = Real(sum[t]);
        if (r == c) dm = fmax(dm, sum[t]);
      } else if (vi < CV::NU + DA) {
        s.c_ga[(size_t)i * L::SG + (vi - CV::NU)] = sum[t];
        gm = fmax(gm, fabs(sum[t]));
      } else if (vi < CV::NV) {
        const int x = vi - CV::NU - DA;
        cX[(x / DCc) * DCc + x % DCc] = Real(sum[t]);
      }
    }
    gm = warp_max(gm);
    dm = warp_max(dm);
    if (i >= D.nnA) {
      v[0] = gm;
      v[1] = dm;
    }
  }
  block_reduce<2, 0>(v, red);
  store_partials(part, v);
}

// Sums the relinearisation partials: cost, Z, gc, gradient max, max diagonal, initial lambda.
template <int DC>
__global__ void __launch_bounds__(256) k_relin_finalize(DevState s, const double* __restrict__ part_pt, int nbp,
                                                        const double* __restrict__ part_cam, int nbc,
                                                        int init_lambda, double tau) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  constexpr int NS = RelinNV<DC>::NS, NV = RelinNV<DC>::NV, NZ = nsym(DC);
  constexpr int DCc = DC > 0 ? DC : 1;
  __shared__ double red[8 * (NV > 2 ? NV : 2)];
  double a[NV];
  fold_partials<NV, NS>(part_pt, nbp, a, red);
  double b[2];
  fold_partials<2, 0>(part_cam, nbc, b, red);
  if (threadIdx.x == 0) {
    const Dims& D = s.d;
    double gmax = fmax(fmax(a[NS], b[0]), 0.0);
    double dmax = fmax(a[NS + 1], b[1]);
    if (DC > 0) {
      int z = 0;
      for (int r = 0; r < DCc; ++r)
        for (int c = r; c < DCc; ++c, ++z) {
          s.g_Z[r * DCc + c] = a[1 + z];
          s.g_Z[c * DCc + r] = a[1 + z];
          if (r == c && r >= D.nnC) dmax = fmax(dmax, a[1 + z]);
        }
      for (int c = 0; c < DCc; ++c) {
        s.g_gc[c] = a[1 + NZ + c];
        if (c >= D.nnC) gmax = fmax(gmax, fabs(a[1 + NZ + c]));
      }
    }
    s.d_relin[0] = a[0];
    s.d_relin[1] = gmax;
    s.d_relin[2] = dmax;
    if (init_lambda) *s.d_lambda = tau * dmax;
  }
}

// ---- reduced system ---------------------------------------------------------------------

template <int DC>
struct ElimNV {
  static constexpr int NZ = nsym(DC);
  static constexpr int NV = (DC > 0) ? NZ + DC : 1;
};

__device__ __forceinline__ bool inv3(const double a[6], double o[6]) {
  // inverse of the symmetric matrix [[a0,a1,a2],[a1,a3,a4],[a2,a4,a5]] by cofactors
  const double c00 = a[3] * a[5] - a[4] * a[4];
  const double c01 = a[2] * a[4] - a[1] * a[5];
  const double c02 = a[1] * a[4] - a[2] * a[3];
  const double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  if (!(det != 0.0) || !isfinite(det)) return false;
  const double id = 1.0 / det;
  o[0] = c00 * id;
  o[1] = c01 * id;
  o[2] = c02 * id;
  o[3] = (a[0] * a[5] - a[2] * a[2]) * id;
  o[4] = (a[1] * a[2] - a[0] * a[4]) * id;
  o[5] = (a[0] * a[3] - a[1] * a[1]) * id;
  return true;
}

// One thread per point: Vinv_j = (V_j + lambda I)^-1, q_j = Vinv gb, Vinv Y_j and, with FP32
// blocks, T_k = W_k Vinv_j for its observations; Y^T Vinv Y and Y^T q go to per-block partials.
template <int DA, int DC, typename Real>
__global__ void __launch_bounds__(kPtThreads) k_point_eliminate(DevState s, double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  using L = Lay<DA, DC, Real>;
  constexpr int DCc = L::DCc;
  constexpr int NV = ElimNV<DC>::NV;
  __shared__ double red[(kPtThreads / 32) * NV];
  const Dims& D = s.d;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  double v[NV];
#pragma unroll
  for (int t = 0; t < NV; ++t) v[t] = 0.0;
  if (j < D.M) {
    const double lam = *s.d_lambda;
    Real vv[L::SV];
    vload(reinterpret_cast<const Real*>(s.p_V) + (size_t)j * L::SV, vv);
    double a[6] = {double(vv[0]) + lam, double(vv[1]), double(vv[2]), double(vv[3]) + lam, double(vv[4]),
                   double(vv[5]) + lam};
    double vi[6] = {0, 0, 0, 0, 0, 0};
    const bool fixB = j < D.nnB;
    if (!fixB && !inv3(a, vi)) {
      *s.d_fail = 1;
      vi[0] = vi[1] = vi[2] = vi[3] = vi[4] = vi[5] = 0.0;
    }
    Real vo[L::SV];
#pragma unroll
    for (int t = 0; t < L::SV; ++t) vo[t] = t < 6 ? Real(vi[t]) : Real(0);
    vstore(reinterpret_cast<Real*>(s.p_Vinv) + (size_t)j * L::SV, vo);
    double gb[4];
    vload(s.p_gb + (size_t)j * 4, gb);
    double q[4] = {0, 0, 0, 0};
#pragma unroll
    for (int r = 0; r < 3; ++r) q[r] = vi[s3(r, 0)] * gb[0] + vi[s3(r, 1)] * gb[1] + vi[s3(r, 2)] * gb[2];
    vstore(s.p_q + (size_t)j * 4, q);
    if (DC > 0) {
      Real yv[L::SY];
      vload(reinterpret_cast<const Real*>(s.p_Y) + (size_t)j * L::SY, yv);
      double YV[3][DCc];
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < DCc; ++c)
          YV[r][c] = vi[s3(r, 0)] * double(yv[c]) + vi[s3(r, 1)] * double(yv[DCc + c]) + vi[s3(r, 2)] * double(yv[2 * DCc + c]);
      Real yo[L::SY];
#pragma unroll
      for (int t = 0; t < L::SY; ++t) yo[t] = Real(0);
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < DCc; ++c) yo[r * DCc + c] = Real(YV[r][c]);
      vstore(reinterpret_cast<Real*>(s.p_YV) + (size_t)j * L::SY, yo);
      int z = 0;
#pragma unroll
      for (int r = 0; r < DCc; ++r)
#pragma unroll
        for (int c = r; c < DCc; ++c, ++z)
          v[z] = double(yv[r]) * YV[0][c] + double(yv[DCc + r]) * YV[1][c] + double(yv[2 * DCc + r]) * YV[2][c];
#pragma unroll
      for (int c = 0; c < DCc; ++c)
        v[nsym(DC) + c] = double(yv[c]) * q[0] + double(yv[DCc + c]) * q[1] + double(yv[2 * DCc + c]) * q[2];
    }
    if constexpr (stores_products<Real>()) {
      for (int k = s.p_ptr[j]; k < s.p_ptr[j + 1]; ++k) {
        float w[L::SW];
        vload(s.o_W + (size_t)k * L::SW, w);
        float t[L::SW];
#pragma unroll
        for (int x = 0; x < L::SW; ++x) t[x] = 0.f;
#pragma unroll
        for (int r = 0; r < DA; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c)
            t[r * 3 + c] = float(double(w[r * 3]) * vi[s3(0, c)] + double(w[r * 3 + 1]) * vi[s3(1, c)] +
                                 double(w[r * 3 + 2]) * vi[s3(2, c)]);
        vstore(s.o_T + (size_t)k * L::SW, t);
      }
    }
  }
  block_reduce<NV, NV>(v, red);
  store_partials(part, v);
}

// One warp per chunk of a camera-pair block's observation pairs: partial sum T_k W_m^T (FP32
// blocks: the stored T_k and W_m; FP64 blocks: A_k^T (B_k Vinv_j B_m^T) A_m).
template <int DA, typename Real>
__device__ __forceinline__ void schur_chunks_body(DevState s, double* __restrict__ part, int bid, int nblk) {
  using L = Lay<DA, 0, Real>;
  using SV = SchurV<DA>;
  const int lane = threadIdx.x & 31;
  const int ch = bid * 4 + (threadIdx.x >> 5);
  if (ch >= s.nch_blk) return;
  Real acc[SV::VP];
#pragma unroll
  for (int t = 0; t < SV::VP; ++t) acc[t] = Real(0);
  const int end = s.bc_end[ch];
  if constexpr (!stores_products<Real>()) {
    // FP64 blocks: T_k W_m^T = A_k^T (B_k Vinv_j B_m^T) A_m, 126 FMAs per pair
    const double* oA = reinterpret_cast<const double*>(s.o_A);
    for (int p = s.bc_beg[ch] + lane; p < end; p += 32) {
      const int k = s.pr_k[p], m = s.pr_m[p];
      const int j = s.o_pt[k];
      double Ak[L::SA], Am[L::SA], Bk[kSB], Bm[kSB], vi[L::SV];
      vload(oA + (size_t)k * L::SA, Ak);
      vload(s.o_B + (size_t)k * kSB, Bk);
      vload(oA + (size_t)m * L::SA, Am);
      vload(s.o_B + (size_t)m * kSB, Bm);
      vload(reinterpret_cast<const double*>(s.p_Vinv) + (size_t)j * L::SV, vi);
      double Q[2][3];   // B_k Vinv_j
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          Q[r][c] = Bk[3 * r] * vi[s3(0, c)] + Bk[3 * r + 1] * vi[s3(1, c)] + Bk[3 * r + 2] * vi[s3(2, c)];
      double Mx[2][2];  // B_k Vinv_j B_m^T
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int t = 0; t < 2; ++t) Mx[r][t] = Q[r][0] * Bm[3 * t] + Q[r][1] * Bm[3 * t + 1] + Q[r][2] * Bm[3 * t + 2];
#pragma unroll
      for (int c = 0; c < DA; ++c) {
        const double n0 = Mx[0][0] * Am[c] + Mx[0][1] * Am[DA + c];
        const double n1 = Mx[1][0] * Am[c] + Mx[1][1] * Am[DA + c];
#pragma unroll
        for (int a = 0; a < DA; ++a) acc[a * DA + c] += Ak[a] * n0 + Ak[DA + a] * n1;
      }
    }
  } else {
  const float* oT = s.o_T;
  const float* oW = s.o_W;
  // FP32 blocks: a lane takes its pairs p and p + 32 in one trip, so both pairs' gathers are in
  // flight together (same summation order as one pair per trip), except with 13 unknowns per
  // camera, whose blocks already fill the register file.
  constexpr int U = DA <= 11 ? 2 : 1;
  for (int p = s.bc_beg[ch] + lane; p < end; p += 32 * U) {
    int k[U], m[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int q = p + 32 * u < end ? p + 32 * u : p;   // a missing second pair re-reads the first
      k[u] = s.pr_k[q];
      m[u] = s.pr_m[q];
    }
    float t[U][L::SW], w[U][L::SW];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      vload(oT + (size_t)k[u] * L::SW, t[u]);
      vload(oW + (size_t)m[u] * L::SW, w[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (u > 0 && p + 32 * u >= end) break;
#pragma unroll
      for (int a = 0; a < DA; ++a)
#pragma unroll
        for (int c = 0; c < DA; ++c)
          acc[a * DA + c] += t[u][a * 3] * w[u][c * 3] + t[u][a * 3 + 1] * w[u][c * 3 + 1] +
                             t[u][a * 3 + 2] * w[u][c * 3 + 2];
    }
  }
  }
  warp_reduce_transpose(acc);
#pragma unroll
  for (int t = 0; t < SV::VP / 32; ++t) part[(size_t)ch * SV::VP + lane * (SV::VP / 32) + t] = double(acc[t]);
}

template <int DA, typename Real>
__global__ void __launch_bounds__(128) k_schur_chunks(DevState s, double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  schur_chunks_body<DA, Real>(s, part, blockIdx.x, gridDim.x);
}

// One warp per camera-pair block (i <= l): S_il = delta_il (U_i + lambda I) - sum of its chunk
// partials, written into the lower triangle of the dense column-major S.
template <int DA, typename Real>
__device__ __forceinline__ void schur_finish_body(DevState s, const double* __restrict__ part, int bid, int nblk,
                                                  bool skip_fixed_diag = false) {
  using L = Lay<DA, 0, Real>;
  using SV = SchurV<DA>;
  constexpr int PER = SV::VP / 32;
  const int lane = threadIdx.x & 31;
  const int b = bid * 4 + (threadIdx.x >> 5);
  if (b >= s.nb) return;
  const int i = s.b_i[b], l = s.b_l[b];
  // beside rhs_finish in one launch, the identity block of a fixed camera is rhs_finish's alone
  if (skip_fixed_diag && i == l && i < s.d.nnA) return;
  double sum[PER];
#pragma unroll
  for (int t = 0; t < PER; ++t) sum[t] = 0.0;
  for (int ch = s.blk_bc_ptr[b]; ch < s.blk_bc_ptr[b + 1]; ++ch)
#pragma unroll
    for (int t = 0; t < PER; ++t) sum[t] += part[(size_t)ch * SV::VP + lane + 32 * t];
  const double lam = *s.d_lambda;
  const Real* cU = reinterpret_cast<const Real*>(s.c_U) + (size_t)i * L::SU;
  const size_t ld = s.ld;
#pragma unroll
  for (int t = 0; t < PER; ++t) {
    const int e = lane + 32 * t;
    if (e >= SV::NV) continue;
    const int a = e / DA, c = e % DA;
    double val = -sum[t];
    if (i == l) val += double(cU[a * DA + c]) + (a == c ? lam : 0.0);
    if (s.Sb) {
      reinterpret_cast<Real*>(s.Sb)[(size_t)b * DA * DA + a * DA + c] = Real(val);
    } else {
      // element (row l*DA + c, col i*DA + a) of the lower triangle holds S_il[a][c]
      s.S[(size_t)(i * DA + a) * ld + (l * DA + c)] = val;
    }
  }
}

template <int DA, typename Real>
__global__ void __launch_bounds__(128) k_schur_finish(DevState s, const double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  schur_finish_body<DA, Real>(s, part, blockIdx.x, gridDim.x);
}

// One warp per chunk of a camera's observations: partial sum_k W_k q_j(k) and sum_k T_k Y_j(k),
// the latter as sum_k W_k (Vinv Y)_j(k) (FP64 blocks: W_k x as A_k^T (B_k x)).
template <int DA, int DC, typename Real>
__device__ __forceinline__ void rhs_chunks_body(DevState s, double* __restrict__ part, int bid, int nblk) {
  using L = Lay<DA, DC, Real>;
  using RV = RhsV<DA, DC>;
  constexpr int DCc = L::DCc;
  const int lane = threadIdx.x & 31;
  const int ch = bid * kCamWarps + (threadIdx.x >> 5);
  if (ch >= s.nch_cam) return;
  double acc[RV::VP];
#pragma unroll
  for (int t = 0; t < RV::VP; ++t) acc[t] = 0.0;
  for (int idx = s.cc_beg[ch] + lane; idx < s.cc_end[ch]; idx += 32) {
    const int k = s.c_obs[idx];
    const int j = s.o_pt[k];
    double q[4];
    vload(s.p_q + (size_t)j * 4, q);
    if constexpr (!stores_products<Real>()) {
      // W_k x = A_k^T (B_k x)
      double A[L::SA], B[kSB];
      vload(reinterpret_cast<const double*>(s.o_A) + (size_t)k * L::SA, A);
      vload(s.o_B + (size_t)k * kSB, B);
      const double bq0 = B[0] * q[0] + B[1] * q[1] + B[2] * q[2];
      const double bq1 = B[3] * q[0] + B[4] * q[1] + B[5] * q[2];
#pragma unroll
      for (int a = 0; a < DA; ++a) acc[a] += A[a] * bq0 + A[DA + a] * bq1;
      if (DC > 0) {
        double yv[L::SY];
        vload(reinterpret_cast<const double*>(s.p_YV) + (size_t)j * L::SY, yv);
#pragma unroll
        for (int c = 0; c < DCc; ++c) {
          const double by0 = B[0] * yv[c] + B[1] * yv[DCc + c] + B[2] * yv[2 * DCc + c];
          const double by1 = B[3] * yv[c] + B[4] * yv[DCc + c] + B[5] * yv[2 * DCc + c];
#pragma unroll
          for (int a = 0; a < DA; ++a) acc[DA + a * DCc + c] += A[a] * by0 + A[DA + a] * by1;
        }
      }
      continue;
    }
    float w[L::SW];
    vload(s.o_W + (size_t)k * L::SW, w);
#pragma unroll
    for (int a = 0; a < DA; ++a) acc[a] += double(w[a * 3]) * q[0] + double(w[a * 3 + 1]) * q[1] + double(w[a * 3 + 2]) * q[2];
    if (DC > 0) {
      // T_k Y_j = W_k (Vinv_j Y_j): the point's Vinv Y is already stored, so no T_k gather
      Real yv[L::SY];
      vload(reinterpret_cast<const Real*>(s.p_YV) + (size_t)j * L::SY, yv);
#pragma unroll
      for (int a = 0; a < DA; ++a)
#pragma unroll
        for (int c = 0; c < DCc; ++c)
          acc[DA + a * DCc + c] += double(w[a * 3]) * double(yv[c]) + double(w[a * 3 + 1]) * double(yv[DCc + c]) +
                                   double(w[a * 3 + 2]) * double(yv[2 * DCc + c]);
    }
  }
  warp_reduce_transpose(acc);
#pragma unroll
  for (int t = 0; t < RV::VP / 32; ++t) part[(size_t)ch * RV::VP + lane * (RV::VP / 32) + t] = acc[t];
}

template <int DA, int DC, typename Real>
__global__ void __launch_bounds__(kCamWarps * 32) k_rhs_chunks(DevState s, double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  rhs_chunks_body<DA, DC, Real>(s, part, blockIdx.x, gridDim.x);
}

// One warp per camera: rhs_i = ga_i - sum W q and the camera/global border X_i - sum T Y into S;
// identity block, zero rhs and zero border for fixed cameras.
template <int DA, int DC, typename Real>
__device__ __forceinline__ void rhs_finish_body(DevState s, const double* __restrict__ cpart, int bid, int nblk) {
  using L = Lay<DA, DC, Real>;
  using RV = RhsV<DA, DC>;
  constexpr int DCc = L::DCc;
  constexpr int PER = RV::VP / 32;
  const Dims& D = s.d;
  const int lane = threadIdx.x & 31;
  const int i = bid * kCamWarps + (threadIdx.x >> 5);
  if (i >= D.N) return;
  const size_t ld = s.ld, rs = s.rhs_stride;
  const int c0 = D.N * DA;
  if (i < D.nnA) {
    for (int t = lane; t < DA * DA; t += 32) {
      const int a = t / DA, c = t % DA;
      if (s.Sb) reinterpret_cast<Real*>(s.Sb)[(size_t)s.diag_blk[i] * DA * DA + t] = Real(a == c ? 1.0 : 0.0);
      else s.S[(size_t)(i * DA + a) * ld + (i * DA + c)] = (a == c) ? 1.0 : 0.0;
    }
    for (int a = lane; a < DA; a += 32) s.rhs[(size_t)(i * DA + a) * rs] = 0.0;
    if (!s.Sb)
      for (int t = lane; t < RV::NX; t += 32) s.S[(size_t)(i * DA + t / DCc) * ld + c0 + t % DCc] = 0.0;
    return;
  }
  double sum[PER];
#pragma unroll
  for (int t = 0; t < PER; ++t) sum[t] = 0.0;
  for (int ch = s.cam_cc_ptr[i]; ch < s.cam_cc_ptr[i + 1]; ++ch)
#pragma unroll
    for (int t = 0; t < PER; ++t) sum[t] += cpart[(size_t)ch * RV::VP + lane + 32 * t];
  const Real* cX = reinterpret_cast<const Real*>(s.c_X) + (size_t)i * L::SX;
#pragma unroll
  for (int t = 0; t < PER; ++t) {
    const int e = lane + 32 * t;
    if (e < DA) {
      s.rhs[(size_t)(i * DA + e) * rs] = s.c_ga[(size_t)i * L::SG + e] - sum[t];
    } else if (e < RV::NV) {
      const int x = e - DA, a = x / DCc, c = x % DCc;
      const double val = (c >= D.nnC) ? double(cX[a * DCc + c]) - sum[t] : 0.0;
      s.S[(size_t)(i * DA + a) * ld + (c0 + c)] = val;  // row c0+c, col i*DA+a
    }
  }
}

template <int DA, int DC, typename Real>
__global__ void __launch_bounds__(kCamWarps * 32) k_rhs_finish(DevState s, const double* __restrict__ cpart) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  rhs_finish_body<DA, DC, Real>(s, cpart, blockIdx.x, gridDim.x);
}

// Global block: S_cc = Z + lambda I - sum_j Y_j^T Vinv_j Y_j, rhs_c = gc - sum_j Y_j^T q_j.
template <int DA, int DC>
__device__ __forceinline__ void global_block_body(DevState s, const double* __restrict__ part, int nbp, int bid, int nblk) {
  constexpr int NV = ElimNV<DC>::NV;
  constexpr int DCc = DC > 0 ? DC : 1;
  __shared__ double red[8 * NV];
  double a[NV];
  fold_partials<NV, NV>(part, nbp, a, red);
  if (threadIdx.x == 0 && DC > 0) {
    const Dims& D = s.d;
    const double lam = *s.d_lambda;
    const int c0 = D.N * DA;
    const size_t ld = s.ld;
    int z = 0;
    for (int r = 0; r < DCc; ++r)
      for (int c = r; c < DCc; ++c, ++z) {
        double val;
        if (r < D.nnC || c < D.nnC) val = (r == c) ? 1.0 : 0.0;
        else val = s.g_Z[r * DCc + c] - a[z] + (r == c ? lam : 0.0);
        s.S[(size_t)(c0 + r) * ld + (c0 + c)] = val;   // row c0+c >= col c0+r
      }
    for (int c = 0; c < DCc; ++c) s.rhs[(size_t)(c0 + c) * s.rhs_stride] = (c < D.nnC) ? 0.0 : s.g_gc[c] - a[nsym(DC) + c];
  }
}

template <int DA, int DC>
__global__ void __launch_bounds__(256) k_global_block(DevState s, const double* __restrict__ part, int nbp) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  global_block_body<DA, DC>(s, part, nbp, blockIdx.x, gridDim.x);
}

// ---- trial step ----------------------------------------------------------------------------

// G lanes per point: db_j = q_j - sum_k T_k^T da_i(k) - (Vinv Y_j) dc; X' = X + db.  With FP64
// blocks the sum is Vinv_j sum_k B_k^T (A_k da_i(k)).
template <int DA, int DC, typename Real>
__device__ __forceinline__ void point_backsub_body(DevState s, double* __restrict__ part, int bid, int nblk) {
  using L = Lay<DA, DC, Real>;
  constexpr int DCc = L::DCc;
  __shared__ double red[(kPtThreads / 32) * 2];
  const Dims& D = s.d;
  constexpr int G = backsub_lanes<Real>();
  const int gt = bid * blockDim.x + threadIdx.x;
  const int j = gt / G, lig = gt % G;
  const bool active = j < D.M && j >= D.nnB;
  double v[2] = {0.0, 0.0};
  double acc[3] = {0, 0, 0};
  const double* x = s.x;
  if (active) {
    // this lane's share of sum_k T_k^T dc_i over the track (FP64 blocks: of sum_k B_k^T A_k dc_i,
    // multiplied by Vinv_j below)
    for (int k = s.p_ptr[j] + lig; k < s.p_ptr[j + 1]; k += G) {
      const int i = s.o_cam[k];
      if constexpr (stores_products<Real>()) {
        float t[L::SW];
        vload(s.o_T + (size_t)k * L::SW, t);
#pragma unroll
        for (int a = 0; a < DA; ++a) {
          const double da = x[i * DA + a];
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[c] += double(t[a * 3 + c]) * da;
        }
      } else {
        double A[L::SA], B[kSB];
        vload(reinterpret_cast<const double*>(s.o_A) + (size_t)k * L::SA, A);
        vload(s.o_B + (size_t)k * kSB, B);
        double ad0 = 0.0, ad1 = 0.0;
#pragma unroll
        for (int a = 0; a < DA; ++a) {
          const double da = x[i * DA + a];
          ad0 += A[a] * da;
          ad1 += A[DA + a] * da;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] += B[c] * ad0 + B[3 + c] * ad1;
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) acc[c] = group_sum<G>(acc[c]);
  if (j < D.M && lig == 0) {
    double db[3] = {0, 0, 0};
    if (active) {
      double q[4];
      vload(s.p_q + (size_t)j * 4, q);
      if constexpr (!stores_products<Real>()) {
        double vi[L::SV];
        vload(reinterpret_cast<const double*>(s.p_Vinv) + (size_t)j * L::SV, vi);
        const double a0 = acc[0], a1 = acc[1], a2 = acc[2];
#pragma unroll
        for (int r = 0; r < 3; ++r) acc[r] = vi[s3(r, 0)] * a0 + vi[s3(r, 1)] * a1 + vi[s3(r, 2)] * a2;
      }
      if (DC > 0) {
        Real yv[L::SY];
        vload(reinterpret_cast<const Real*>(s.p_YV) + (size_t)j * L::SY, yv);
        const int c0 = D.N * DA;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < DCc; ++c) acc[r] += double(yv[r * DCc + c]) * x[c0 + c];
      }
      double gb[4];
      vload(s.p_gb + (size_t)j * 4, gb);
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        db[r] = q[r] - acc[r];
        v[0] += db[r] * db[r];
        v[1] += db[r] * gb[r];
      }
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) s.trial.X[3 * j + r] = s.cur.X[3 * j + r] + db[r];
  }
  block_reduce<2, 2>(v, red);
  store_partials(part, v, bid, nblk);
}

template <int DA, int DC, typename Real>
__global__ void __launch_bounds__(kPtThreads) k_point_backsub(DevState s, double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  point_backsub_body<DA, DC, Real>(s, part, blockIdx.x, gridDim.x);
}

// One thread per camera (plus the globals on thread 0 of block 0): trial parameters.
template <int MODEL, int DA, int DC>
__device__ __forceinline__ void camera_update_body(DevState s, double* __restrict__ part, int bid, int nblk) {
  __shared__ double red[4 * 2];
  const Dims& D = s.d;
  const int i = bid * blockDim.x + threadIdx.x;
  const double* x = s.x;
  double v[2] = {0.0, 0.0};
  if (i < D.N) {
    double R[9], T[3];
#pragma unroll
    for (int t = 0; t < 9; ++t) R[t] = s.cur.R[9 * i + t];
#pragma unroll
    for (int t = 0; t < 3; ++t) T[t] = s.cur.T[3 * i + t];
    double K[9];
    double dist[4] = {0, 0, 0, 0};
    if (MODEL == kModelStd || MODEL == kModelVarying) {   // per-camera K (STEREO has none)
#pragma unroll
      for (int t = 0; t < 9; ++t) K[t] = s.cur.K[9 * i + t];
    }
    if (MODEL == kModelVarying) {
#pragma unroll
      for (int t = 0; t < 4; ++t) dist[t] = s.cur.dist[4 * i + t];
    }
    if (i >= D.nnA) {
      double d[DA];
#pragma unroll
      for (int a = 0; a < DA; ++a) {
        d[a] = x[i * DA + a];
        v[0] += d[a] * d[a];
        v[1] += d[a] * s.c_ga[(size_t)i * Lay<DA, DC>::SG + a];
      }
      T[0] += d[0]; T[1] += d[1]; T[2] += d[2];
      rotate_update(d + 3, R);
      if (MODEL == kModelVarying && DA > 6) {
        double di[7] = {0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int a = 6; a < DA; ++a) di[a - 6] = d[a];
        intrinsic_update(D.mode, di, K, dist, -1.0);
      }
    }
#pragma unroll
    for (int t = 0; t < 9; ++t) s.trial.R[9 * i + t] = R[t];
#pragma unroll
    for (int t = 0; t < 3; ++t) s.trial.T[3 * i + t] = T[t];
    if (MODEL == kModelStd || MODEL == kModelVarying) {
#pragma unroll
      for (int t = 0; t < 9; ++t) s.trial.K[9 * i + t] = K[t];
    }
    if (MODEL == kModelVarying) {
#pragma unroll
      for (int t = 0; t < 4; ++t) s.trial.dist[4 * i + t] = dist[t];
    }
  }
  if (MODEL == kModelCommon && bid == 0 && threadIdx.x == 0) {
    double K[9], dist[4];
    for (int t = 0; t < 9; ++t) K[t] = s.cur.K[t];
    for (int t = 0; t < 4; ++t) dist[t] = s.cur.dist[t];
    if (DC > D.nnC) {
      double di[7] = {0, 0, 0, 0, 0, 0, 0};
      const int c0 = D.N * DA;
      for (int c = 0; c < DC; ++c) {
        di[c] = (c >= D.nnC) ? x[c0 + c] : 0.0;
        v[0] += di[c] * di[c];
        v[1] += di[c] * s.g_gc[c];
      }
      intrinsic_update(D.mode, di, K, dist, D.cached_ar);
    }
    for (int t = 0; t < 9; ++t) s.trial.K[t] = K[t];
    for (int t = 0; t < 4; ++t) s.trial.dist[t] = dist[t];
  }
  block_reduce<2, 2>(v, red);
  store_partials(part, v, bid, nblk);
}

template <int MODEL, int DA, int DC>
__global__ void __launch_bounds__(128) k_camera_update(DevState s, double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  camera_update_body<MODEL, DA, DC>(s, part, blockIdx.x, gridDim.x);
}

// ---- merged launches of independent stages (the LM path) -------------------------------------
// Stages that do not read each other's output run as block ranges of one launch: one kernel
// boundary (drain and fill) less each.  Every block runs the same code on the same data as in the
// stage's own kernel (block index and count of its range), so the results are the same bits.

// Schur chunks (blocks [0, g1)) and reduced-rhs chunks: both read only the elimination's output.
template <int DA, int DC, typename Real>
__global__ void __launch_bounds__(128) k_chunks_merged(DevState s, int g1, int g2) {
  pdl_wait();
  pdl_trigger();
  if ((int)blockIdx.x < g1) schur_chunks_body<DA, Real>(s, s.part_bc, blockIdx.x, g1);
  else rhs_chunks_body<DA, DC, Real>(s, s.part_cc, blockIdx.x - g1, g2);
}

// Schur finish (blocks [0, g1)), rhs / border finish ([g1, g1 + g2)) and, with global
// parameters, the global block (the last block): they write disjoint parts of S and rhs.
template <int DA, int DC, typename Real>
__global__ void __launch_bounds__(128) k_finish_merged(DevState s, int g1, int g2, const double* __restrict__ pelim,
                                                       int nbp) {
  pdl_wait();
  pdl_trigger();
  const int b = blockIdx.x;
  if (b < g1) schur_finish_body<DA, Real>(s, s.part_bc, b, g1, true);
  else if (b < g1 + g2) rhs_finish_body<DA, DC, Real>(s, s.part_cc, b - g1, g2);
  else global_block_body<DA, DC>(s, pelim, nbp, 0, 1);
}

// Camera (and global) update (blocks [0, g1)) and point back-substitution: both read the
// reduced solution and the current parameters and write different parts of the trial ones.
template <int MODEL, int DA, int DC, typename Real>
__global__ void __launch_bounds__(128) k_update_merged(DevState s, int g1, int g2, double* __restrict__ pcam,
                                                       double* __restrict__ ppt) {
  pdl_wait();
  pdl_trigger();
  if ((int)blockIdx.x < g1) camera_update_body<MODEL, DA, DC>(s, pcam, blockIdx.x, g1);
  else point_backsub_body<DA, DC, Real>(s, ppt, blockIdx.x - g1, g2);
}

// One thread per observation: sum |w e|^2 at parameters P, with the stored (frozen) weights or
// with weights recomputed at P.
template <int MODEL>
__global__ void __launch_bounds__(256) k_obs_cost(DevState s, ParamSet P, int recompute_w, double* __restrict__ part) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  __shared__ double red[8];
  const Dims& D = s.d;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double v[1] = {0.0};
  if (k < D.K) {
    const int i = s.o_cam[k], j = s.o_pt[k];
    Cam cam;
    load_cam<MODEL>(cam, P.R, P.T, P.K, P.dist, i);
    if (MODEL == kModelStereo) load_rig(cam, s.rig, s.o_sub[k]);
    const double X[3] = {P.X[3 * j], P.X[3 * j + 1], P.X[3 * j + 2]};
    double XX[3], e[2];
    residual<MODEL>(cam, X, s.o_meas[2 * k], s.o_meas[2 * k + 1], XX, e);
    const double w = recompute_w ? huber_weight(D.thr, e) : s.o_w[k];
    v[0] = w * w * (e[0] * e[0] + e[1] * e[1]);
  }
  block_reduce<1, 1>(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void __launch_bounds__(256) k_trial_finalize(DevState s, const double* __restrict__ pb, int nbp,
                                                        const double* __restrict__ pc, int nbc,
                                                        const double* __restrict__ po, int nbo) {
  pdl_wait();      // the previous stage's writes are visible
  pdl_trigger();   // the next stage may be scheduled once all blocks of this one are resident
  __shared__ double red[8 * 2];
  double a[2], b[2], c[1];
  fold_partials<2, 2>(pb, nbp, a, red);
  fold_partials<2, 2>(pc, nbc, b, red);
  fold_partials<1, 1>(po, nbo, c, red);
  if (threadIdx.x == 0) {
    s.d_trial[0] = c[0];
    s.d_trial[1] = a[0] + b[0];
    s.d_trial[2] = a[1] + b[1];
    s.d_trial[3] = *s.d_fail != 0 ? 1.0 : 0.0;   // every kernel that can fail ran before this one
  }
}

__global__ void __launch_bounds__(256) k_sum_to(const double* __restrict__ po, int nbo, double* out) {
  __shared__ double red[8];
  double c[1];
  fold_partials<1, 1>(po, nbo, c, red);
  if (threadIdx.x == 0) *out = c[0];
}

// ---- host launchers ----------------------------------------------------------------------

inline int cdiv(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// partial-buffer regions (in doubles)
struct PartLayout {
  size_t relin_pt, relin_cam, elim, backsub, camupd, obs;
};

// blocks of a track kernel with `lanes` lanes per point (the partial regions are sized for the most)
inline int lane_blocks(int M, int lanes = kMaxPtLanes) { return cdiv((int64_t)std::max(M, 1) * lanes, kPtThreads); }

template <int DA, int DC>
inline PartLayout part_layout(const DevState& s) {
  PartLayout p;
  const int bl = lane_blocks(s.d.M);
  const int bc = cdiv(std::max(s.d.N, 1), kCamWarps);
  const int bu = cdiv(std::max(s.d.N, 1), 128);
  p.relin_pt = 0;
  p.relin_cam = p.relin_pt + (size_t)bl * RelinNV<DC>::NV;
  p.elim = p.relin_cam + (size_t)bc * 2;
  p.backsub = p.elim + (size_t)bl * ElimNV<DC>::NV;
  p.camupd = p.backsub + (size_t)bl * 2;
  p.obs = p.camupd + (size_t)bu * 2;
  return p;
}

template <int MODEL, int DA, int DC, typename Real>
struct Ops {
  // Launches one stage of the LM iteration (see LmStage in lm.cuh).
  static int stage(DevState& s, int id, int init_lambda, double tau, cudaStream_t st) {
    const PartLayout pl = part_layout<DA, DC>(s);
    const int bp = cdiv(std::max(s.d.M, 1), kPtThreads);                  // one lane per point
    const int bl = lane_blocks(s.d.M, kLinLanes);                          // the linearisation
    const int bb = lane_blocks(s.d.M, backsub_lanes<Real>());              // the back-substitution
    const int bc = cdiv(std::max(s.d.N, 1), kCamWarps);
    const int bu = cdiv(std::max(s.d.N, 1), 128);
    const int bo = cdiv(std::max(s.d.K, 1), 256);
    cudaError_t e = cudaSuccess;
    switch (id) {
      case kStageLinearize:
        e = launch_pdl(k_linearize<MODEL, DA, DC, Real>, dim3(bl), dim3(kPtThreads), 0, st, s, s.part + pl.relin_pt);
        break;
      case kStageCameraChunks:
        if (s.nch_cam == 0) return V3DBA_OK;
        e = launch_pdl(k_camera_chunks<DA, DC, Real>, dim3(cdiv(s.nch_cam, kCamWarps)), dim3(kCamWarps * 32), 0, st, s,
                       s.part_cc);
        break;
      case kStageCameraFinish:
        e = launch_pdl(k_camera_finish<DA, DC, Real>, dim3(bc), dim3(kCamWarps * 32), 0, st, s, (const double*)s.part_cc,
                       s.part + pl.relin_cam);
        break;
      case kStageRelinFinalize:
        e = launch_pdl(k_relin_finalize<DC>, dim3(1), dim3(256), 0, st, s, (const double*)(s.part + pl.relin_pt), bl,
                       (const double*)(s.part + pl.relin_cam), bc, init_lambda, tau);
        break;
      case kStagePointEliminate:
        e = launch_pdl(k_point_eliminate<DA, DC, Real>, dim3(bp), dim3(kPtThreads), 0, st, s, s.part + pl.elim);
        break;
      case kStageSchurChunks:
        if (s.nch_blk == 0) return V3DBA_OK;
        e = launch_pdl(k_schur_chunks<DA, Real>, dim3(cdiv(s.nch_blk, 4)), dim3(128), 0, st, s, s.part_bc);
        break;
      case kStageSchurFinish:
        if (s.nb == 0) return V3DBA_OK;
        e = launch_pdl(k_schur_finish<DA, Real>, dim3(cdiv(s.nb, 4)), dim3(128), 0, st, s, (const double*)s.part_bc);
        break;
      case kStageRhsChunks:
        if (s.nch_cam == 0) return V3DBA_OK;
        e = launch_pdl(k_rhs_chunks<DA, DC, Real>, dim3(cdiv(s.nch_cam, kCamWarps)), dim3(kCamWarps * 32), 0, st, s,
                       s.part_cc);
        break;
      case kStageRhsFinish:
        e = launch_pdl(k_rhs_finish<DA, DC, Real>, dim3(bc), dim3(kCamWarps * 32), 0, st, s, (const double*)s.part_cc);
        break;
      case kStageGlobalBlock:
        if (DC == 0) return V3DBA_OK;
        e = launch_pdl(k_global_block<DA, DC>, dim3(1), dim3(256), 0, st, s, (const double*)(s.part + pl.elim), bp);
        break;
      case kStagePointBacksub:
        e = launch_pdl(k_point_backsub<DA, DC, Real>, dim3(bb), dim3(kPtThreads), 0, st, s, s.part + pl.backsub);
        break;
      case kStageCameraUpdate:
        e = launch_pdl(k_camera_update<MODEL, DA, DC>, dim3(bu), dim3(128), 0, st, s, s.part + pl.camupd);
        break;
      case kStageTrialCost:
        e = launch_pdl(k_obs_cost<MODEL>, dim3(bo), dim3(256), 0, st, s, (ParamSet)s.trial, 0, s.part + pl.obs);
        break;
      case kStageTrialFinalize:
        e = launch_pdl(k_trial_finalize, dim3(1), dim3(256), 0, st, s, (const double*)(s.part + pl.backsub), bb,
                       (const double*)(s.part + pl.camupd), bu, (const double*)(s.part + pl.obs), bo);
        break;
      default:
        return V3DBA_ERR_INVALID_ARGUMENT;
    }
    if (e != cudaSuccess) {
      fprintf(stderr, "v3dba: launch of stage %d failed: %s\n", id, cudaGetErrorString(e));
      cudaGetLastError();
      return V3DBA_ERR_CUDA;
    }
    V3DBA_LAUNCH_CHECK();
    return V3DBA_OK;
  }
  static int run(DevState& s, int first, int last, int init_lambda, double tau, cudaStream_t st) {
    for (int id = first; id <= last; ++id) {
      const int rc = stage(s, id, init_lambda, tau, st);
      if (rc) return rc;
    }
    return V3DBA_OK;
  }
  static int relinearize(DevState& s, bool init_lambda, double tau, cudaStream_t st) {
    return run(s, kStageLinearize, kStageRelinFinalize, init_lambda ? 1 : 0, tau, st);
  }
  static int launched(cudaError_t e) {
    if (e != cudaSuccess) {
      fprintf(stderr, "v3dba: merged launch failed: %s\n", cudaGetErrorString(e));
      cudaGetLastError();
      return V3DBA_ERR_CUDA;
    }
    V3DBA_LAUNCH_CHECK();
    return V3DBA_OK;
  }
  // elimination, then the Schur and rhs chunks in one launch, then the three finishing stages in
  // one launch (the same work as the stages kStagePointEliminate .. kStageGlobalBlock)
  static int build_reduced(DevState& s, cudaStream_t st) {
    int rc = stage(s, kStagePointEliminate, 0, 0.0, st);
    if (rc) return rc;
    const PartLayout pl = part_layout<DA, DC>(s);
    const int g1 = s.nch_blk > 0 ? cdiv(s.nch_blk, 4) : 0, g2 = s.nch_cam > 0 ? cdiv(s.nch_cam, kCamWarps) : 0;
    if (g1 + g2 > 0 && (rc = launched(launch_pdl(k_chunks_merged<DA, DC, Real>, dim3(g1 + g2), dim3(128), 0, st, s,
                                                 g1, g2))))
      return rc;
    const int f1 = s.nb > 0 ? cdiv(s.nb, 4) : 0, f2 = cdiv(std::max(s.d.N, 1), kCamWarps);
    const int bp = cdiv(std::max(s.d.M, 1), kPtThreads);
    return launched(launch_pdl(k_finish_merged<DA, DC, Real>, dim3(f1 + f2 + (DC > 0 ? 1 : 0)), dim3(128), 0, st, s,
                               f1, f2, (const double*)(s.part + pl.elim), bp));
  }
  // camera update and point back-substitution in one launch, then the trial cost and the step
  // statistics (the stages kStagePointBacksub .. kStageTrialFinalize)
  static int finish_trial(DevState& s, cudaStream_t st) {
    const PartLayout pl = part_layout<DA, DC>(s);
    const int bu = cdiv(std::max(s.d.N, 1), 128), bb = lane_blocks(s.d.M, backsub_lanes<Real>());
    int rc = launched(launch_pdl(k_update_merged<MODEL, DA, DC, Real>, dim3(bu + bb), dim3(128), 0, st, s, bu, bb,
                                 s.part + pl.camupd, s.part + pl.backsub));
    if (rc) return rc;
    return run(s, kStageTrialCost, kStageTrialFinalize, 0, 0.0, st);
  }
  static int cost(DevState& s, const ParamSet& P, double* d_out, cudaStream_t st) {
    const PartLayout pl = part_layout<DA, DC>(s);
    const int bo = cdiv(std::max(s.d.K, 1), 256);
    k_obs_cost<MODEL><<<bo, 256, 0, st>>>(s, P, 1, s.part + pl.obs);
    V3DBA_LAUNCH_CHECK();
    k_sum_to<<<1, 256, 0, st>>>(s.part + pl.obs, bo, d_out);
    V3DBA_LAUNCH_CHECK();
    return V3DBA_OK;
  }
  static const LmOps* table() {
    static const LmOps t = {&relinearize, &build_reduced, &finish_trial, &cost, &stage};
    return &t;
  }
};

size_t camera_chunk_values(int DA, int DC) {
  const int nu = DA * (DA + 1) / 2 + DA + DA * DC;
  const int nr = DA + DA * DC;
  return (size_t)round32(std::max(nu, nr));
}
size_t block_chunk_values(int DA) { return (size_t)round32(DA * DA); }

// size (in doubles) of the partial buffer for the given dims
size_t partial_doubles(const DevState& s) {
  const int bc = cdiv(std::max(s.d.N, 1), kCamWarps);
  const int bu = cdiv(std::max(s.d.N, 1), 128);
  const int bo = cdiv(std::max(s.d.K, 1), 256);
  const size_t maxNV = RelinNV<7>::NV;
  const int bl = lane_blocks(s.d.M);
  return (size_t)bl * maxNV + (size_t)bc * 2 + (size_t)bl * ElimNV<7>::NV + (size_t)bl * 2 + (size_t)bu * 2 + bo + 64;
}

template <typename Real>
const LmOps* ops_for(int model, int DA, int DC) {
  if (model == kModelStd) return DA == 6 && DC == 0 ? Ops<kModelStd, 6, 0, Real>::table() : nullptr;
  if (model == kModelStereo) return DA == 6 && DC == 0 ? Ops<kModelStereo, 6, 0, Real>::table() : nullptr;
  if (model == kModelCommon) {
    if (DA != 6) return nullptr;
    switch (DC) {
      case 0: return Ops<kModelCommon, 6, 0, Real>::table();
      case 1: return Ops<kModelCommon, 6, 1, Real>::table();
      case 3: return Ops<kModelCommon, 6, 3, Real>::table();
      case 5: return Ops<kModelCommon, 6, 5, Real>::table();
      case 7: return Ops<kModelCommon, 6, 7, Real>::table();
    }
    return nullptr;
  }
  if (model == kModelVarying) {
    if (DC != 0) return nullptr;
    switch (DA) {
      case 6: return Ops<kModelVarying, 6, 0, Real>::table();
      case 7: return Ops<kModelVarying, 7, 0, Real>::table();
      case 9: return Ops<kModelVarying, 9, 0, Real>::table();
      case 11: return Ops<kModelVarying, 11, 0, Real>::table();
      case 13: return Ops<kModelVarying, 13, 0, Real>::table();
    }
  }
  return nullptr;
}

const LmOps* lm_ops(int model, int DA, int DC, bool fp64) {
  return fp64 ? ops_for<double>(model, DA, DC) : ops_for<float>(model, DA, DC);
}

}  // namespace v3dba
