// Preconditioned conjugate gradients on the reduced camera system, for scenes whose reduced
// system is too large to factor densely (thousands of cameras).
//
// The reference always factors the full damped normal matrix with a sparse LDL^T
// (V3D/src/Math/v3d_optimization.cpp:1096-1145); on a 2,000-camera scene its camera part fills
// in densely.  Here the Schur complement S (camera-pair blocks, dA x dA) is kept block-sparse and
// solved inexactly per LM step: stop at |r| <= tol |b| (tol 1e-6 by default) or after max_iter
// iterations.  The blocks are stored in `Real` (FP32 in mixed mode); vectors, dot products and
// the preconditioners are FP64 arithmetic.
//
// Preconditioners (z = M^-1 r):
//   * block-Jacobi: the inverses of the diagonal camera blocks;
//   * the learned factor: G^T G with G = (I + E) C^-1 (csrc/precond_gnn.cu);
//   * either of them plus the gauge coarse space: + Z (Z^T S Z)^-1 Z^T r.  The columns of Z are
//     the camera parts of the 7 similarity motions of the whole scene (translation, rotation,
//     scale), under which the reprojection cost is invariant: with R_i <- Rodrigues(w) R_i and
//     T_i += dT (v3d_metricbundle.cpp:17-50), a world motion (t, w, s) moves camera i by
//     dT_i = -R_i t + s T_i, w_i = -R_i w.  S Z = lambda Z up to rounding, so these are the
//     smallest eigenvectors of the damped system, which no local preconditioner reaches.
//
// The whole iteration runs in one persistent cooperative kernel: grid-wide barriers separate the
// phases, grid reductions write per-block partials that every block then folds in the same fixed
// order (deterministic), and the stopping test is taken on the device.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "lm.cuh"
#include "precond.cuh"

namespace cg = cooperative_groups;

namespace v3dba {
namespace {

constexpr int kPcgThreads = 256;
constexpr int kPcgWarps = kPcgThreads / 32;
constexpr int kPcgMaxGrid = 4096;   // blocks; sizes the partial-sum buffers
constexpr int kPartStride = 16;     // doubles per block and reduction
constexpr int kGauge = 7;           // similarity gauge of a metric reconstruction
constexpr int kGaugeTri = kGauge * (kGauge + 1) / 2;

struct PcgArgs {
  int N, DA, n;                    // cameras, block size, unknowns (N * DA)
  const int* rp;                   // [N+1] row pointer over both triangles
  const int* rb;                   // block id of each row entry
  const int* rc;                   // column camera of each row entry
  const unsigned char* rt;         // 1 when the stored block is (col, row): use its transpose
  const int* rd;                   // [N] entry of the diagonal block in row i (see PcgState)
  const void* Sb;                  // blocks, dA x dA row-major, Real
  const double* Pinv;              // [N] dA x dA inverse diagonal blocks (block-Jacobi)
  const float* cinv;               // learned: [N] 6 x 6 lower-triangular C_i^-1
  const float* ehat;               // learned: [nb] 6 x 6 blocks E_e C_a^-1 by block id
  const double* frames;            // gauge: [N] R_i (9, row-major) and T_i (3)
  const double* gauge_L;           // gauge: packed lower Cholesky factor of Z^T S Z, [28] = ok
  double* t;                       // learned: G r
  const double* b;                 // rhs (n)
  double* x;                       // solution (n)
  double* r; double* z; double* p; double* p2; double* Ap;
  double* r2;                      // learned: the next residual (double buffer)
  double* part;                    // [2 * gridDim * kPartStride] partials
  double tol;
  int max_iter;
  int* iters_out;
  int* fail;
};

// A dA x dA block of `Real` into registers (16-byte vector loads when the blocks allow it).
template <typename Real, int DA>
__device__ __forceinline__ void load_block(const Real* __restrict__ B, Real (&m)[DA * DA]) {
  if constexpr (std::is_same<Real, float>::value && (DA * DA) % 4 == 0) {
    const float4* B4 = reinterpret_cast<const float4*>(B);
#pragma unroll
    for (int q = 0; q < DA * DA / 4; ++q) {
      const float4 t = __ldg(B4 + q);
      m[4 * q] = t.x; m[4 * q + 1] = t.y; m[4 * q + 2] = t.z; m[4 * q + 3] = t.w;
    }
  } else if constexpr (std::is_same<Real, double>::value && (DA * DA) % 2 == 0) {
    const double2* B2 = reinterpret_cast<const double2*>(B);
#pragma unroll
    for (int q = 0; q < DA * DA / 2; ++q) {
      const double2 t = __ldg(B2 + q);
      m[2 * q] = t.x; m[2 * q + 1] = t.y;
    }
  } else {
#pragma unroll
    for (int q = 0; q < DA * DA; ++q) m[q] = B[q];
  }
}

// acc += B v (or B^T v)
template <typename Real, int DA>
__device__ __forceinline__ void block_mv(const Real (&m)[DA * DA], bool tr, const double (&v)[DA], double (&acc)[DA]) {
  if (tr) {
#pragma unroll
    for (int c = 0; c < DA; ++c)
#pragma unroll
      for (int r = 0; r < DA; ++r) acc[r] += double(m[c * DA + r]) * v[c];
  } else {
#pragma unroll
    for (int r = 0; r < DA; ++r)
#pragma unroll
      for (int c = 0; c < DA; ++c) acc[r] += double(m[r * DA + c]) * v[c];
  }
}

// acc += B v (or B^T v) for a block in memory (large dA: no register copy)
template <typename Real, int DA>
__device__ __forceinline__ void block_mv_mem(const Real* __restrict__ B, bool tr, const double (&v)[DA],
                                             double (&acc)[DA]) {
  if constexpr (DA <= 6) {
    Real m[DA * DA];
    load_block<Real, DA>(B, m);
    block_mv<Real, DA>(m, tr, v, acc);
  } else if (tr) {
    for (int c = 0; c < DA; ++c)
#pragma unroll
      for (int r = 0; r < DA; ++r) acc[r] += double(__ldg(B + c * DA + r)) * v[c];
  } else {
#pragma unroll
    for (int r = 0; r < DA; ++r)
      for (int c = 0; c < DA; ++c) acc[r] += double(__ldg(B + r * DA + c)) * v[c];
  }
}

// Component q of Z_i c (the gauge motion with coefficients c applied to camera i).
__device__ __forceinline__ double gauge_apply(const double* f, const double (&c)[kGauge], int q) {
  if (q < 3) return -(f[q * 3] * c[0] + f[q * 3 + 1] * c[1] + f[q * 3 + 2] * c[2]) + f[9 + q] * c[6];
  const int r = q - 3;
  return -(f[r * 3] * c[3] + f[r * 3 + 1] * c[4] + f[r * 3 + 2] * c[5]);
}

// y += (Z_i^T)_(:, q) v: the contribution of component q of camera i's vector to Z^T v.
__device__ __forceinline__ void gauge_project(const double* f, int q, double v, double* y) {
  if (q < 3) {
    for (int k = 0; k < 3; ++k) y[k] -= f[q * 3 + k] * v;
    y[6] += f[9 + q] * v;
  } else {
    for (int k = 0; k < 3; ++k) y[3 + k] -= f[(q - 3) * 3 + k] * v;
  }
}

// c = (Z^T S Z)^-1 y from its packed Cholesky factor
__device__ __forceinline__ void gauge_solve(const double* L, const double* y, double (&c)[kGauge]) {
  double w[kGauge];
  for (int i = 0; i < kGauge; ++i) {
    double s = y[i];
    for (int k = 0; k < i; ++k) s -= L[i * (i + 1) / 2 + k] * w[k];
    w[i] = s / L[i * (i + 1) / 2 + i];
  }
  for (int i = kGauge - 1; i >= 0; --i) {
    double s = w[i];
    for (int k = i + 1; k < kGauge; ++k) s -= L[k * (k + 1) / 2 + i] * c[k];
    c[i] = s / L[i * (i + 1) / 2 + i];
  }
}

// Grid-wide deterministic sums of NV values: per-block partials, then every block folds them:
// warp 0 reads the partials with its lanes striding over the blocks and combines the lanes by a
// fixed shuffle tree, so every block computes the same sums bit for bit.  The partials
// alternate between two buffers, so one barrier per reduction suffices (a buffer is rewritten
// only two reductions later, after every block has passed the barrier of the reduction in
// between).  Must be called by all threads of all blocks.
template <int NV>
__device__ __forceinline__ void grid_sums(double (&v)[NV], double* part, int& parity, cg::grid_group& grid) {
  static_assert(NV <= kPartStride, "partial stride");
  __shared__ double red[kPcgWarps * kPartStride];
  block_reduce<NV, NV>(v, red);
  double* pb = part + (size_t)parity * gridDim.x * kPartStride;
  if (threadIdx.x == 0)
    for (int t = 0; t < NV; ++t) pb[(size_t)blockIdx.x * kPartStride + t] = v[t];
  grid.sync();
  if (threadIdx.x < 32) {
    double s[NV];
#pragma unroll
    for (int t = 0; t < NV; ++t) s[t] = 0.0;
    for (int bk = threadIdx.x; bk < (int)gridDim.x; bk += 32)
#pragma unroll
      for (int t = 0; t < NV; ++t) s[t] += pb[(size_t)bk * kPartStride + t];
#pragma unroll
    for (int t = 0; t < NV; ++t) s[t] = warp_sum(s[t]);
    if (threadIdx.x == 0)
#pragma unroll
      for (int t = 0; t < NV; ++t) red[t] = s[t];
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < NV; ++t) v[t] = red[t];
  __syncthreads();   // red is reused by the next reduction's block_reduce
  parity ^= 1;
}

// Learned preconditioner, first half: t = G r = (I + E) C^-1 r.  Row i gathers C_i^-1 r_i and
// E_(i,k) C_k^-1 r_k over its lower neighbours k (the transposed entries of its row).
__device__ __forceinline__ void learned_lower_row(const PcgArgs& a, int i, int lane, const double* r, double* t) {
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int e = a.rp[i] + lane; e < a.rd[i]; e += 32) {   // the transposed entries: a prefix of the row
    double v[6];
    const double* rv = r + (size_t)a.rc[e] * 6;
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = rv[c];
    block_mv_mem<float, 6>(a.ehat + (size_t)a.rb[e] * 36, false, v, acc);
  }
  if (lane < 6) {
    const float* Ci = a.cinv + (size_t)i * 36 + lane * 6;
    const double* v = r + (size_t)i * 6;
    for (int c = 0; c <= lane; ++c) acc[lane] += double(Ci[c]) * v[c];
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) acc[q] = warp_sum(acc[q]);
  if (lane < 6) t[(size_t)i * 6 + lane] = acc[lane];
}

// The same first half for the residual of the step being taken, r - alpha Ap, formed on the fly
// from the previous residual and Ap of every row it reads (they are not overwritten in this
// phase: the new residual goes to a second buffer).
__device__ __forceinline__ void learned_lower_row_step(const PcgArgs& a, int i, int lane, const double* r,
                                                       const double* Ap, double alpha, double* t) {
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int e = a.rp[i] + lane; e < a.rd[i]; e += 32) {   // the transposed entries: a prefix of the row
    double v[6];
    const size_t o = (size_t)a.rc[e] * 6;
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = r[o + c] - alpha * Ap[o + c];
    block_mv_mem<float, 6>(a.ehat + (size_t)a.rb[e] * 36, false, v, acc);
  }
  if (lane < 6) {
    const float* Ci = a.cinv + (size_t)i * 36 + lane * 6;
    const size_t o = (size_t)i * 6;
    for (int c = 0; c <= lane; ++c) acc[lane] += double(Ci[c]) * (r[o + c] - alpha * Ap[o + c]);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) acc[q] = warp_sum(acc[q]);
  if (lane < 6) t[(size_t)i * 6 + lane] = acc[lane];
}

// Second half: z = G^T t.  Row i gathers C_i^-T t_i and (E_(l,i) C_i^-1)^T t_l over its upper
// neighbours l (the direct entries of its row).  Returns z_i[lane] on lanes < 6.
__device__ __forceinline__ double learned_upper_row(const PcgArgs& a, int i, int lane, const double* t) {
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  // the direct entries after the diagonal one: a suffix of the row, taken by each lane at the
  // same positions rp[i] + lane + 32 m as in a walk over the whole row (the same sums)
  int e = a.rp[i] + lane;
  const int lo = a.rd[i] + 1;
  if (e < lo) e += (lo - e + 31) / 32 * 32;
  for (; e < a.rp[i + 1]; e += 32) {
    double v[6];
    const double* tv = t + (size_t)a.rc[e] * 6;
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = tv[c];
    block_mv_mem<float, 6>(a.ehat + (size_t)a.rb[e] * 36, true, v, acc);
  }
  if (lane < 6) {
    const float* Ci = a.cinv + (size_t)i * 36;
    const double* v = t + (size_t)i * 6;
    for (int c = lane; c < 6; ++c) acc[lane] += double(Ci[c * 6 + lane]) * v[c];
  }
  double out = 0.0;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const double s = warp_sum(acc[q]);
    if (lane == q) out = s;
  }
  return out;
}

// Block-Jacobi: z_i = Pinv_i r_i with r_i[c] held by lane c; returns z_i[lane] on lanes < DA.
template <int DA>
__device__ __forceinline__ double jacobi_row(const PcgArgs& a, int i, int lane, double ri) {
  double zq = 0.0;
  const double* P = a.Pinv + (size_t)i * DA * DA + (size_t)(lane < DA ? lane : 0) * DA;
#pragma unroll
  for (int c = 0; c < DA; ++c) {
    const double rc = __shfl_sync(0xffffffffu, ri, c);
    zq += P[c] * rc;
  }
  return lane < DA ? zq : 0.0;
}

// Preconditioned conjugate gradients, one cooperative launch.  Warp w owns camera rows
// w, w + nwarps, ...; lane c < dA holds component c of the row's vectors.  Per iteration:
//   A: p = z + beta p_old (own rows; neighbours' p formed on the fly), Ap = S p, sum p.Ap
//                                                                              -- 1 barrier
//   B: x += alpha p, r -= alpha Ap, z_f = fine preconditioner of r, sums r.z_f, r.r and, with
//      the gauge space, y = Z^T r                                              -- 1 barrier
//      (the learned factor needs its lower triangular half first, fed with r - alpha Ap formed
//      on the fly: 1 more barrier; r is double-buffered)
// With the gauge space, z = z_f + Z c with c = (Z^T S Z)^-1 y is never stored: every reader
// forms it from z_f, the camera frames and c (r.z = r.z_f + y.c).  p alternates between two
// buffers so that phase A never overwrites a p_old that a neighbour reads.
template <typename Real, int DA, bool LEARNED, bool GAUGE>
__global__ void __launch_bounds__(kPcgThreads) k_pcg(PcgArgs a) {
  cg::grid_group grid = cg::this_grid();
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kPcgWarps + (threadIdx.x >> 5);
  const int nwarps = gridDim.x * kPcgWarps;
  const int N = a.N;
  int parity = 0;
  double* p_old = a.p;
  double* p_new = a.p2;
  const Real* Sb = reinterpret_cast<const Real*>(a.Sb);
  const bool use_gauge = GAUGE && a.gauge_L[kGaugeTri] > 0.5;
  double gc[kGauge];
#pragma unroll
  for (int k = 0; k < kGauge; ++k) gc[k] = 0.0;

  // z_f of row i from r (fine preconditioner) and the row's partial sums; r_i[lane] given
  auto fine_and_sums = [&](int i, double ri, double (&u)[2 + kGauge]) {
    double zq;
    if constexpr (LEARNED) zq = learned_upper_row(a, i, lane, a.t);
    else zq = jacobi_row<DA>(a, i, lane, ri);
    if (lane < DA) {
      a.z[(size_t)i * DA + lane] = zq;
      u[0] += ri * zq;
      u[1] += ri * ri;
      if (use_gauge && lane < 6) gauge_project(a.frames + (size_t)i * 12, lane, ri, u + 2);
    }
  };
  // r.z = r.z_f + y.c with c = (Z^T S Z)^-1 y
  auto finish_sums = [&](double (&u)[2 + kGauge]) -> double {
    double rzv = u[0];
    if (use_gauge) {
      gauge_solve(a.gauge_L, u + 2, gc);
      for (int k = 0; k < kGauge; ++k) rzv += u[2 + k] * gc[k];
    }
    return rzv;
  };

  // x = 0, r = b, z = M^-1 r
  double u0[2 + kGauge];
#pragma unroll
  for (int k = 0; k < 2 + kGauge; ++k) u0[k] = 0.0;
  if constexpr (LEARNED) {
    for (int i = warp; i < N; i += nwarps)
      if (lane < DA) {
        const size_t q = (size_t)i * DA + lane;
        a.x[q] = 0.0;
        a.r[q] = a.b[q];
      }
    grid.sync();
    for (int i = warp; i < N; i += nwarps) learned_lower_row(a, i, lane, a.r, a.t);
    grid.sync();
    for (int i = warp; i < N; i += nwarps) fine_and_sums(i, lane < DA ? a.r[(size_t)i * DA + lane] : 0.0, u0);
  } else {
    for (int i = warp; i < N; i += nwarps) {
      double ri = 0.0;
      if (lane < DA) {
        const size_t q = (size_t)i * DA + lane;
        a.x[q] = 0.0;
        ri = a.b[q];
        a.r[q] = ri;
      }
      fine_and_sums(i, ri, u0);
    }
  }
  grid_sums<2 + kGauge>(u0, a.part, parity, grid);
  double rz = finish_sums(u0);
  const double bnorm = sqrt(u0[1]);
  int it = 0;
  double beta = 0.0;
  if (bnorm > 0.0) {
    while (it < a.max_iter) {
      const bool first = (it == 0);
      // phase A
      double w[1] = {0.0};
      for (int i = warp; i < N; i += nwarps) {
        double acc[DA];
#pragma unroll
        for (int r = 0; r < DA; ++r) acc[r] = 0.0;
        for (int e = a.rp[i] + lane; e < a.rp[i + 1]; e += 32) {
          const int col = a.rc[e];
          double v[DA];
          const double* zc = a.z + (size_t)col * DA;
          const double* pc = p_old + (size_t)col * DA;
#pragma unroll
          for (int c = 0; c < DA; ++c) v[c] = zc[c];
          if (use_gauge) {
            const double* f = a.frames + (size_t)col * 12;
#pragma unroll
            for (int c = 0; c < 6; ++c) v[c] += gauge_apply(f, gc, c);
          }
          if (!first)
#pragma unroll
            for (int c = 0; c < DA; ++c) v[c] += beta * pc[c];
          block_mv_mem<Real, DA>(Sb + (size_t)a.rb[e] * DA * DA, a.rt[e] != 0, v, acc);
        }
        double api = 0.0;
#pragma unroll
        for (int r = 0; r < DA; ++r) {
          const double s = warp_sum(acc[r]);
          if (lane == r) api = s;
        }
        if (lane < DA) {
          const size_t q = (size_t)i * DA + lane;
          double pi = a.z[q];
          if (use_gauge && lane < 6) pi += gauge_apply(a.frames + (size_t)i * 12, gc, lane);
          if (!first) pi += beta * p_old[q];
          p_new[q] = pi;
          a.Ap[q] = api;
          w[0] += pi * api;
        }
      }
      grid_sums<1>(w, a.part, parity, grid);
      const double pAp = w[0];
      if (!(pAp > 0.0)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) *a.fail = 1;
        break;
      }
      const double alpha = rz / pAp;
      // phase B
      double u[2 + kGauge];
#pragma unroll
      for (int k = 0; k < 2 + kGauge; ++k) u[k] = 0.0;
      if constexpr (LEARNED) {
        for (int i = warp; i < N; i += nwarps) {
          learned_lower_row_step(a, i, lane, a.r, a.Ap, alpha, a.t);
          if (lane < DA) {
            const size_t q = (size_t)i * DA + lane;
            a.x[q] += alpha * p_new[q];
            a.r2[q] = a.r[q] - alpha * a.Ap[q];
          }
        }
        grid.sync();
        double* tr = a.r;
        a.r = a.r2;
        a.r2 = tr;
        for (int i = warp; i < N; i += nwarps) fine_and_sums(i, lane < DA ? a.r[(size_t)i * DA + lane] : 0.0, u);
      } else {
        for (int i = warp; i < N; i += nwarps) {
          double ri = 0.0;
          if (lane < DA) {
            const size_t q = (size_t)i * DA + lane;
            a.x[q] += alpha * p_new[q];
            ri = a.r[q] - alpha * a.Ap[q];
            a.r[q] = ri;
          }
          fine_and_sums(i, ri, u);
        }
      }
      grid_sums<2 + kGauge>(u, a.part, parity, grid);
      ++it;
      if (sqrt(u[1]) <= a.tol * bnorm) break;
      const double rz_new = finish_sums(u);
      beta = rz_new / rz;
      rz = rz_new;
      double* tmp = p_old;
      p_old = p_new;
      p_new = tmp;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *a.iters_out = it;
}

// Gauge coarse matrix Z^T S Z: one thread per camera row accumulates Z_i^T (S Z)_i (28 packed
// values) into its own slot.
template <typename Real>
__global__ void k_gauge_rows(PcgArgs a, double* rows_part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const Real* Sb = reinterpret_cast<const Real*>(a.Sb);
  double W[6][kGauge];
  for (int r = 0; r < 6; ++r)
    for (int k = 0; k < kGauge; ++k) W[r][k] = 0.0;
  for (int e = a.rp[i]; e < a.rp[i + 1]; ++e) {
    const double* f = a.frames + (size_t)a.rc[e] * 12;
    const Real* B = Sb + (size_t)a.rb[e] * 36;
    const bool tr = a.rt[e] != 0;
    for (int k = 0; k < kGauge; ++k) {
      double c[kGauge];
      for (int t = 0; t < kGauge; ++t) c[t] = t == k ? 1.0 : 0.0;
      double v[6];
      for (int q = 0; q < 6; ++q) v[q] = gauge_apply(f, c, q);
      for (int r = 0; r < 6; ++r) {
        double s = 0.0;
        for (int q = 0; q < 6; ++q) s += double(tr ? B[q * 6 + r] : B[r * 6 + q]) * v[q];
        W[r][k] += s;
      }
    }
  }
  const double* f = a.frames + (size_t)i * 12;
  double* out = rows_part + (size_t)i * kGaugeTri;
  for (int k = 0; k < kGauge; ++k) {
    double c[kGauge];
    for (int t = 0; t < kGauge; ++t) c[t] = t == k ? 1.0 : 0.0;
    for (int l = 0; l <= k; ++l) {
      double s = 0.0;
      for (int q = 0; q < 6; ++q) s += gauge_apply(f, c, q) * W[q][l];
      out[k * (k + 1) / 2 + l] = s;
    }
  }
}

// Sums the row slots in camera order and factors Z^T S Z (7 x 7, FP64); L[28] = 1 when it is
// numerically positive definite, else 0 (the solve then runs without the gauge space).
__global__ void k_gauge_factor(const double* __restrict__ rows_part, int N, double* L) {
  __shared__ double A[kGaugeTri];
  const int t = threadIdx.x;
  if (t < kGaugeTri) {
    double s = 0.0;
    for (int i = 0; i < N; ++i) s += rows_part[(size_t)i * kGaugeTri + t];
    A[t] = s;
  }
  __syncthreads();
  if (t != 0) return;
  double dmax = 0.0;
  for (int k = 0; k < kGauge; ++k) dmax = fmax(dmax, A[k * (k + 1) / 2 + k]);
  bool ok = dmax > 0.0;
  for (int j = 0; j < kGauge && ok; ++j) {
    double d = A[j * (j + 1) / 2 + j];
    for (int k = 0; k < j; ++k) d -= L[j * (j + 1) / 2 + k] * L[j * (j + 1) / 2 + k];
    if (!(d > 1e-13 * dmax)) { ok = false; break; }
    const double ljj = sqrt(d);
    L[j * (j + 1) / 2 + j] = ljj;
    for (int r = j + 1; r < kGauge; ++r) {
      double v = A[r * (r + 1) / 2 + j];
      for (int k = 0; k < j; ++k) v -= L[r * (r + 1) / 2 + k] * L[j * (j + 1) / 2 + k];
      L[r * (r + 1) / 2 + j] = v / ljj;
    }
  }
  L[kGaugeTri] = ok ? 1.0 : 0.0;
}

// Camera frames of the gauge space: R_i and T_i, zero for fixed cameras.
__global__ void k_gauge_frames(const double* __restrict__ R, const double* __restrict__ T, int N, int n_fixed,
                               double* frames) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const bool fixed = i < n_fixed;
  for (int q = 0; q < 9; ++q) frames[(size_t)i * 12 + q] = fixed ? 0.0 : R[(size_t)i * 9 + q];
  for (int q = 0; q < 3; ++q) frames[(size_t)i * 12 + 9 + q] = fixed ? 0.0 : T[(size_t)i * 3 + q];
}

// Inverse of each diagonal block (Gauss-Jordan with partial pivoting, FP64), one thread per camera.
template <typename Real>
__global__ void k_pcg_precond(const void* Sb, const int* diag_blk, int N, int DA, double* Pinv, int* fail) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double m[13][26];
  const Real* B = reinterpret_cast<const Real*>(Sb) + (size_t)diag_blk[i] * DA * DA;
  for (int r = 0; r < DA; ++r)
    for (int c = 0; c < 2 * DA; ++c) m[r][c] = c < DA ? double(B[r * DA + c]) : (c - DA == r ? 1.0 : 0.0);
  for (int c = 0; c < DA; ++c) {
    int piv = c;
    for (int r = c + 1; r < DA; ++r)
      if (fabs(m[r][c]) > fabs(m[piv][c])) piv = r;
    if (!(fabs(m[piv][c]) > 0.0)) { *fail = 1; return; }
    if (piv != c)
      for (int t = 0; t < 2 * DA; ++t) { const double tmp = m[c][t]; m[c][t] = m[piv][t]; m[piv][t] = tmp; }
    const double inv = 1.0 / m[c][c];
    for (int t = 0; t < 2 * DA; ++t) m[c][t] *= inv;
    for (int r = 0; r < DA; ++r) {
      if (r == c) continue;
      const double f = m[r][c];
      for (int t = 0; t < 2 * DA; ++t) m[r][t] -= f * m[c][t];
    }
  }
  for (int r = 0; r < DA; ++r)
    for (int c = 0; c < DA; ++c) Pinv[(size_t)i * DA * DA + r * DA + c] = m[r][DA + c];
}

}  // namespace

int pcg_plan(PcgState& ps, const std::vector<int>& b_i, const std::vector<int>& b_l, int N) {
  // row structure over both triangles: row i holds (i, l) for every stored block (i, l) and
  // (i, k) for every stored block (k, i) with k < i (transposed)
  std::vector<std::vector<std::pair<int, int>>> rows(N);   // (column, entry code)
  std::vector<int> diag(N, -1);
  for (size_t b = 0; b < b_i.size(); ++b) {
    const int i = b_i[b], l = b_l[b];
    rows[i].push_back({l, (int)(2 * b)});
    if (l != i) rows[l].push_back({i, (int)(2 * b + 1)});
    else diag[i] = (int)b;
  }
  std::vector<int> rp(1, 0), rb, rc, rd(N, -1);
  std::vector<unsigned char> rt;
  for (int i = 0; i < N; ++i) {
    std::sort(rows[i].begin(), rows[i].end());
    for (auto& e : rows[i]) {
      // sorted by column: transposed entries (columns < i), the diagonal, direct entries
      if (e.first == i) rd[i] = (int)rc.size();
      if ((e.second & 1) != (e.first < i ? 1 : 0)) return V3DBA_ERR_INVALID_INPUT;
      rc.push_back(e.first);
      rb.push_back(e.second / 2);
      rt.push_back((unsigned char)(e.second & 1));
    }
    rp.push_back((int)rc.size());
    if (diag[i] < 0 || rd[i] < 0) return V3DBA_ERR_INVALID_INPUT;
  }
  auto up = [](auto** d, const auto& h) -> int {
    using T = typename std::remove_reference<decltype(h)>::type::value_type;
    if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
    V3DBA_CUDA_TRY(cudaMalloc(d, sizeof(T) * std::max<size_t>(h.size(), 1)));
    if (!h.empty()) V3DBA_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return V3DBA_OK;
  };
  int rc2;
  if ((rc2 = up(&ps.rp, rp)) || (rc2 = up(&ps.rb, rb)) || (rc2 = up(&ps.rc, rc)) || (rc2 = up(&ps.rt, rt)) ||
      (rc2 = up(&ps.rd, rd)) || (rc2 = up(&ps.diag_blk, diag)))
    return rc2;
  return V3DBA_OK;
}

int pcg_alloc(PcgState& ps, int nb, int N, int DA) {
  const size_t n = (size_t)N * DA;
  auto get = [](auto** d, size_t bytes) -> int {
    if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
    V3DBA_CUDA_TRY(cudaMalloc(d, bytes));
    return V3DBA_OK;
  };
  int rc;
  if ((rc = get(&ps.Sb, sizeof(double) * (size_t)std::max(nb, 1) * DA * DA)) ||
      (rc = get(&ps.Pinv, sizeof(double) * (size_t)std::max(N, 1) * DA * DA)) ||
      (rc = get(&ps.vec, sizeof(double) * 8 * std::max<size_t>(n, 1))) ||   // b r z p Ap t p2 r2
      (rc = get(&ps.part, sizeof(double) * 2 * kPartStride * kPcgMaxGrid)) ||
      (rc = get(&ps.gauge_rows, sizeof(double) * kGaugeTri * (size_t)std::max(N, 1))) ||
      (rc = get(&ps.gauge_L, sizeof(double) * (kGaugeTri + 1))) || (rc = get(&ps.iters, sizeof(int))))
    return rc;
  ps.b = ps.vec;
  ps.ready = true;
  return V3DBA_OK;
}

void pcg_free(PcgState& ps) {
  cudaFree(ps.rp); cudaFree(ps.rb); cudaFree(ps.rc); cudaFree(ps.rt); cudaFree(ps.rd); cudaFree(ps.diag_blk);
  cudaFree(ps.Sb); cudaFree(ps.Pinv); cudaFree(ps.vec); cudaFree(ps.part); cudaFree(ps.iters);
  cudaFree(ps.gauge_rows); cudaFree(ps.gauge_L);
  ps = PcgState();
}

int gauge_frames(const double* R, const double* T, int N, int n_fixed, double* frames, cudaStream_t st) {
  if (N <= 0) return V3DBA_OK;
  k_gauge_frames<<<(N + 127) / 128, 128, 0, st>>>(R, T, N, n_fixed, frames);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

namespace {

template <typename Real, int DA>
void* pcg_kernel(bool learned, bool gauge) {
  if constexpr (DA == 6) {
    if (learned) return gauge ? (void*)k_pcg<Real, 6, true, true> : (void*)k_pcg<Real, 6, true, false>;
    if (gauge) return (void*)k_pcg<Real, 6, false, true>;
  }
  return (void*)k_pcg<Real, DA, false, false>;
}

PcgArgs make_args(PcgState& ps, int N, int DA, double tol, int max_iter, double* x, int* d_fail,
                  const PcgPrecond& P) {
  const size_t n = (size_t)N * DA;
  PcgArgs a;
  a.N = N; a.DA = DA; a.n = (int)n;
  a.rp = ps.rp; a.rb = ps.rb; a.rc = ps.rc; a.rt = ps.rt; a.rd = ps.rd; a.Sb = ps.Sb;
  a.Pinv = ps.Pinv; a.b = ps.b; a.x = x;
  a.r = ps.vec + n; a.z = ps.vec + 2 * n; a.p = ps.vec + 3 * n; a.Ap = ps.vec + 4 * n;
  a.t = ps.vec + 5 * n; a.p2 = ps.vec + 6 * n; a.r2 = ps.vec + 7 * n;
  a.cinv = P.cinv;
  a.ehat = P.ehat;
  a.frames = P.frames;
  a.gauge_L = ps.gauge_L;
  a.part = ps.part; a.tol = tol; a.max_iter = max_iter; a.iters_out = ps.iters; a.fail = d_fail;
  return a;
}

}  // namespace

int pcg_solve_precond(PcgState& ps, int N, int DA, bool fp64, double tol, int max_iter, double* x, int* d_fail,
                      cudaStream_t st, const PcgPrecond& P) {
  const bool learned = P.ehat != nullptr && P.cinv != nullptr;
  const bool gauge = P.frames != nullptr;
  if ((learned || gauge) && DA != 6) return V3DBA_ERR_UNSUPPORTED;
  PcgArgs a = make_args(ps, N, DA, tol, max_iter, x, d_fail, P);
  if (!learned) {
    if (fp64) k_pcg_precond<double><<<(N + 127) / 128, 128, 0, st>>>(ps.Sb, ps.diag_blk, N, DA, ps.Pinv, d_fail);
    else k_pcg_precond<float><<<(N + 127) / 128, 128, 0, st>>>(ps.Sb, ps.diag_blk, N, DA, ps.Pinv, d_fail);
    V3DBA_LAUNCH_CHECK();
  }
  if (gauge) {
    if (fp64) k_gauge_rows<double><<<(N + 127) / 128, 128, 0, st>>>(a, ps.gauge_rows);
    else k_gauge_rows<float><<<(N + 127) / 128, 128, 0, st>>>(a, ps.gauge_rows);
    V3DBA_LAUNCH_CHECK();
    k_gauge_factor<<<1, 32, 0, st>>>(ps.gauge_rows, N, ps.gauge_L);
    V3DBA_LAUNCH_CHECK();
  }
  void* fn = nullptr;
  switch (DA) {
    case 6: fn = fp64 ? pcg_kernel<double, 6>(learned, gauge) : pcg_kernel<float, 6>(learned, gauge); break;
    case 7: fn = fp64 ? pcg_kernel<double, 7>(false, false) : pcg_kernel<float, 7>(false, false); break;
    case 9: fn = fp64 ? pcg_kernel<double, 9>(false, false) : pcg_kernel<float, 9>(false, false); break;
    case 11: fn = fp64 ? pcg_kernel<double, 11>(false, false) : pcg_kernel<float, 11>(false, false); break;
    case 13: fn = fp64 ? pcg_kernel<double, 13>(false, false) : pcg_kernel<float, 13>(false, false); break;
    default: return V3DBA_ERR_UNSUPPORTED;
  }
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPcgThreads, 0);
  const int grid = std::max(1, std::min(sms * std::max(per_sm, 1), kPcgMaxGrid));
  void* args[] = {&a};
  V3DBA_CUDA_TRY(cudaLaunchCooperativeKernel(fn, grid, kPcgThreads, args, 0, st));
  note_launches(1);
  return V3DBA_OK;
}

int pcg_solve(PcgState& ps, int N, int DA, bool fp64, double tol, int max_iter, double* x, int* d_fail,
              cudaStream_t st) {
  return pcg_solve_precond(ps, N, DA, fp64, tol, max_iter, x, d_fail, st, PcgPrecond());
}

}  // namespace v3dba
