// Batched bundle adjustment of many small independent problems (triplets, small submodels) in
// one persistent launch.
//
// The reference solves its triplets one after another on one CPU core, 5 LM iterations each
// (SfM/generate_triples/src/generate_triples.cpp:403-415; submodels likewise,
// SfM/generate_submodels_L1/src/generate_submodels_L1.cpp:330-337).  Here one thread block owns
// one problem at a time and runs the whole SparseLevenbergOptimizer::minimize loop
// (V3D/src/Math/v3d_optimization.cpp:719-1250) for it with the reference's semantics: Huber
// weights frozen across a trial, initial lambda = tau * max diagonal, the gradient / update
// stopping tests, the gain ratio, the lambda schedule, the status codes.  Blocks take problems
// from a queue ordered by decreasing size (longest-processing-time first).
//
// Model: StdMetricBundleOptimizer, up to kMaxCams = 4 cameras per problem (reduced system up to
// 24 x 24), any number of points, each point observed by up to kMaxTrack cameras.  Everything
// is FP64.  Per-point quantities are recomputed from the parameters in every pass over the
// points instead of being stored (FLOPs are cheap, shared memory is not): pass REL (weights,
// cost, gradient, max diagonal), pass SCHUR (one 6x6 camera-pair block of the reduced system per
// round, accumulated in registers and folded by a transposing warp reduction -- deterministic,
// no atomics), a warp Cholesky of the reduced system, pass STEP (point back-substitution, trial
// points, trial cost with frozen weights).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "common.cuh"
#include "lm.cuh"
#include "model.cuh"

namespace v3dba {
namespace {

constexpr int kMaxCams = 4;
constexpr int kMaxTrack = 16;
constexpr int kMaxN = 6 * kMaxCams;  // reduced system dimension

struct BatchDev {
  int count = 0;
  // per problem
  int* cam_off = nullptr;   // first camera of the problem
  int* n_cams = nullptr;
  int* pt_off = nullptr;    // first point
  int* n_pts = nullptr;
  int* order = nullptr;     // processing order (decreasing size)
  double* thr = nullptr;    // Huber threshold
  // per camera (current parameters, updated in place)
  double* R = nullptr;      // 9
  double* T = nullptr;      // 3
  double* K = nullptr;      // 9
  // per point
  double* X = nullptr;      // 3 (current, updated in place)
  double* Xt = nullptr;     // 3 (trial)
  int* ptr = nullptr;       // [total points + 1] observations of global point g
  // per observation (point-major inside each problem)
  double* meas = nullptr;   // 2
  unsigned char* cam = nullptr;  // camera index inside the problem
  double* w = nullptr;      // Huber weights of the last linearisation
  // results
  int* status = nullptr;
  int* iterations = nullptr;
  int* rejected = nullptr;
  double* cost = nullptr;       // cost at the last linearisation
  double* init_cost = nullptr;
  double* lambda_out = nullptr;
  unsigned* queue = nullptr;    // work counter
};

struct BatchOpts {
  double tau, grad_thr, upd_thr;
  int max_iter;
};

template <int H, int V>
__device__ __forceinline__ void rt_stage_b(double (&v)[V], int lane, int m) {
#pragma unroll
  for (int t = 0; t < H; ++t) {
    const bool up = (lane & m) != 0;
    const double send = up ? v[t] : v[t + H];
    const double keep = up ? v[t + H] : v[t];
    v[t] = keep + __shfl_xor_sync(0xffffffffu, send, m);
  }
}

// Block-wide deterministic sum of V = 64 values; thread t < 64 returns the total of value t.
template <int NT>
__device__ __forceinline__ double block_sum64(double (&v)[64], double* red /* [NT/32][64] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  rt_stage_b<32>(v, lane, 16);
  rt_stage_b<16>(v, lane, 8);
  rt_stage_b<8>(v, lane, 4);
  rt_stage_b<4>(v, lane, 2);
  rt_stage_b<2>(v, lane, 1);
  red[wid * 64 + 2 * lane] = v[0];
  red[wid * 64 + 2 * lane + 1] = v[1];
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 64)
    for (int w = 0; w < NT / 32; ++w) s += red[w * 64 + threadIdx.x];
  __syncthreads();
  return s;
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_max(v);
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double m = red[0];
  for (int w = 1; w < NT / 32; ++w) m = fmax(m, red[w]);
  __syncthreads();
  return m;
}

struct CamS {
  double R[9], T[3], K[9];
};

// Weighted Jacobian blocks and weighted residual of observation k at (cams, X).
__device__ __forceinline__ void lin_obs(const CamS* cams, const double X[3], const BatchDev& b, int k, double wk,
                                        double A[2][6], double B[2][3], double r[2], double* e_out) {
  const int c = b.cam[k];
  Cam cm;
#pragma unroll
  for (int q = 0; q < 9; ++q) cm.R[q] = cams[c].R[q];
#pragma unroll
  for (int q = 0; q < 3; ++q) cm.T[q] = cams[c].T[q];
#pragma unroll
  for (int q = 0; q < 9; ++q) cm.K[q] = cams[c].K[q];
  cm.d[0] = cm.d[1] = cm.d[2] = cm.d[3] = 0.0;
  double e[2], Cc[2][1];
  linearize_obs<kModelStd, 6, 0>(cm, X, b.meas[2 * k], b.meas[2 * k + 1], 0, 1.0, e, A, B, Cc);
  if (e_out) { e_out[0] = e[0]; e_out[1] = e[1]; }
  r[0] = -wk * e[0];
  r[1] = -wk * e[1];
#pragma unroll
  for (int rr = 0; rr < 2; ++rr) {
#pragma unroll
    for (int q = 0; q < 6; ++q) A[rr][q] *= wk;
#pragma unroll
    for (int q = 0; q < 3; ++q) B[rr][q] *= wk;
  }
}

// (V_j + lambda I)^-1 (packed 00,01,02,11,12,22), gb_j and q = Vinv gb over the point's track.
__device__ __forceinline__ bool point_elim(const CamS* cams, const double X[3], const BatchDev& b, int o0, int n,
                                           double lam, double vi[6], double gb[3], double q[3]) {
  double V[6] = {0, 0, 0, 0, 0, 0};
  gb[0] = gb[1] = gb[2] = 0.0;
  for (int t = 0; t < n; ++t) {
    double A[2][6], B[2][3], r[2];
    lin_obs(cams, X, b, o0 + t, b.w[o0 + t], A, B, r, nullptr);
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
      V[0] += B[rr][0] * B[rr][0]; V[1] += B[rr][0] * B[rr][1]; V[2] += B[rr][0] * B[rr][2];
      V[3] += B[rr][1] * B[rr][1]; V[4] += B[rr][1] * B[rr][2]; V[5] += B[rr][2] * B[rr][2];
#pragma unroll
      for (int c = 0; c < 3; ++c) gb[c] += B[rr][c] * r[rr];
    }
  }
  V[0] += lam; V[3] += lam; V[5] += lam;
  const double c00 = V[3] * V[5] - V[4] * V[4], c01 = V[2] * V[4] - V[1] * V[5], c02 = V[1] * V[4] - V[2] * V[3];
  const double det = V[0] * c00 + V[1] * c01 + V[2] * c02;
  if (!(det != 0.0) || !isfinite(det)) return false;
  const double id = 1.0 / det;
  vi[0] = c00 * id; vi[1] = c01 * id; vi[2] = c02 * id;
  vi[3] = (V[0] * V[5] - V[2] * V[2]) * id;
  vi[4] = (V[1] * V[2] - V[0] * V[4]) * id;
  vi[5] = (V[0] * V[3] - V[1] * V[1]) * id;
  q[0] = vi[0] * gb[0] + vi[1] * gb[1] + vi[2] * gb[2];
  q[1] = vi[1] * gb[0] + vi[3] * gb[1] + vi[4] * gb[2];
  q[2] = vi[2] * gb[0] + vi[4] * gb[1] + vi[5] * gb[2];
  return true;
}

// W = A^T B (6x3) and T = W Vinv of one observation.
__device__ __forceinline__ void wt_of(const double A[2][6], const double B[2][3], const double vi[6], double W[6][3],
                                      double Tm[6][3]) {
#pragma unroll
  for (int a = 0; a < 6; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) W[a][c] = A[0][a] * B[0][c] + A[1][a] * B[1][c];
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    Tm[a][0] = W[a][0] * vi[0] + W[a][1] * vi[1] + W[a][2] * vi[2];
    Tm[a][1] = W[a][0] * vi[1] + W[a][1] * vi[3] + W[a][2] * vi[4];
    Tm[a][2] = W[a][0] * vi[2] + W[a][1] * vi[4] + W[a][2] * vi[5];
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_batched_lm(BatchDev b, BatchOpts o, int first, int last) {
  __shared__ CamS cams[kMaxCams], tcams[kMaxCams];
  __shared__ double S[kMaxN * kMaxN], rhs[kMaxN], da[kMaxN], ga[kMaxN], udiag[kMaxN];
  __shared__ double red[(NT / 32) * 64];
  __shared__ double sc[16];   // scalars: 0 err, 1 lambda, 2 nu, 3 newErr, 4 d2, 5 dg, 6 plen, 7 gmax, 8 maxdiag
  __shared__ int si[8];       // 0 problem, 1 stop, 2 computeDerivatives, 3 fail, 4 accept, 5 status, 6 it, 7 rejected
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) {
      const unsigned slot = atomicAdd(b.queue, 1u);
      si[0] = (first + (int)slot < last) ? b.order[first + slot] : -1;
    }
    __syncthreads();
    const int p = si[0];
    if (p < 0) return;
    const int N = b.n_cams[p], M = b.n_pts[p], c0 = b.cam_off[p], pt0 = b.pt_off[p];
    const double thr = b.thr[p];
    if (tid < N) {
      for (int q = 0; q < 9; ++q) { cams[tid].R[q] = b.R[9 * (c0 + tid) + q]; cams[tid].K[q] = b.K[9 * (c0 + tid) + q]; }
      for (int q = 0; q < 3; ++q) cams[tid].T[q] = b.T[3 * (c0 + tid) + q];
    }
    // cached parameter length (v3d_metricbundle.h:37-45)
    {
      double v[64];
#pragma unroll
      for (int t = 0; t < 64; ++t) v[t] = 0.0;
      for (int j = tid; j < M; j += NT) {
        const double* X = b.X + 3 * (size_t)(pt0 + j);
        v[0] += X[0] * X[0] + X[1] * X[1] + X[2] * X[2];
      }
      if (tid < N) {
        const double* T = b.T + 3 * (size_t)(c0 + tid);
        v[0] += T[0] * T[0] + T[1] * T[1] + T[2] * T[2] + 3.0;
      }
      const double s = block_sum64<NT>(v, red);
      if (tid == 0) {
        sc[6] = sqrt(s);
        sc[1] = 1e-3;   // lambda of a new optimizer object
        sc[2] = 2.0;    // _nu
        si[1] = 0; si[2] = 1; si[5] = V3DBA_STATUS_TIMEOUT; si[7] = 0;
      }
      __syncthreads();
    }
    int it = 0;
    for (it = 0; it < o.max_iter; ++it) {
      if (si[2]) {
        // ---- pass REL: weights, cost, gradient, max diagonal ----
        double v[64];
#pragma unroll
        for (int t = 0; t < 64; ++t) v[t] = 0.0;
        double gbmax = 0.0, vdmax = -1e30;
        for (int j = tid; j < M; j += NT) {
          const int g = pt0 + j;
          const int o0 = b.ptr[g], n = b.ptr[g + 1] - o0;
          const double X[3] = {b.X[3 * (size_t)g], b.X[3 * (size_t)g + 1], b.X[3 * (size_t)g + 2]};
          double V0 = 0, V3 = 0, V5 = 0, gb[3] = {0, 0, 0};
          for (int t = 0; t < n; ++t) {
            const int k = o0 + t;
            double A[2][6], B[2][3], r[2], e[2];
            lin_obs(cams, X, b, k, 1.0, A, B, r, e);
            const double wk = huber_weight(thr, e);
            b.w[k] = wk;
            v[0] += wk * wk * (e[0] * e[0] + e[1] * e[1]);
            r[0] *= wk; r[1] *= wk;
#pragma unroll
            for (int rr = 0; rr < 2; ++rr) {
#pragma unroll
              for (int q = 0; q < 6; ++q) A[rr][q] *= wk;
#pragma unroll
              for (int q = 0; q < 3; ++q) B[rr][q] *= wk;
              V0 += B[rr][0] * B[rr][0];
              V3 += B[rr][1] * B[rr][1];
              V5 += B[rr][2] * B[rr][2];
#pragma unroll
              for (int q = 0; q < 3; ++q) gb[q] += B[rr][q] * r[rr];
            }
            const int c = b.cam[k];
#pragma unroll
            for (int cc = 0; cc < kMaxCams; ++cc) {
              if (cc != c) continue;
#pragma unroll
              for (int a = 0; a < 6; ++a) {
                v[1 + 6 * cc + a] += A[0][a] * r[0] + A[1][a] * r[1];
                v[1 + 24 + 6 * cc + a] += A[0][a] * A[0][a] + A[1][a] * A[1][a];
              }
            }
          }
          if (n > 0) {
            gbmax = fmax(gbmax, fmax(fabs(gb[0]), fmax(fabs(gb[1]), fabs(gb[2]))));
            vdmax = fmax(vdmax, fmax(V0, fmax(V3, V5)));
          }
        }
        const double s = block_sum64<NT>(v, red);
        if (tid == 0) sc[0] = s;
        else if (tid <= 24) ga[tid - 1] = s;
        else if (tid <= 48) udiag[tid - 25] = s;
        const double gm = block_max<NT>(gbmax, red);
        const double vm = block_max<NT>(vdmax, red);
        if (tid == 0) {
          double gmax = gm;
          for (int a = 0; a < 6 * N; ++a) gmax = fmax(gmax, fabs(ga[a]));
          sc[7] = gmax;
          if (gmax < o.grad_thr) { si[5] = V3DBA_STATUS_CONVERGED; si[1] = 1; }
          if (it == 0) {
            if (b.init_cost) b.init_cost[p] = sc[0];
            if (!si[1]) {
              double md = vm;
              for (int a = 0; a < 6 * N; ++a) md = fmax(md, udiag[a]);
              sc[1] = o.tau * md;
            }
          }
        }
        __syncthreads();
        if (si[1]) break;
      }
      // ---- pass SCHUR: one camera-pair block per round ----
      const double lam = sc[1];
      for (int i = 0; i < N; ++i)
        for (int l = i; l < N; ++l) {
          double v[64];
#pragma unroll
          for (int t = 0; t < 64; ++t) v[t] = 0.0;
          for (int j = tid; j < M; j += NT) {
            const int g = pt0 + j;
            const int o0 = b.ptr[g], n = b.ptr[g + 1] - o0;
            const double X[3] = {b.X[3 * (size_t)g], b.X[3 * (size_t)g + 1], b.X[3 * (size_t)g + 2]};
            double vi[6], gb[3], q[3];
            if (!point_elim(cams, X, b, o0, n, lam, vi, gb, q)) continue;
            for (int t = 0; t < n; ++t) {
              if (b.cam[o0 + t] != i) continue;
              double A[2][6], B[2][3], r[2], W[6][3], Tm[6][3];
              lin_obs(cams, X, b, o0 + t, b.w[o0 + t], A, B, r, nullptr);
              wt_of(A, B, vi, W, Tm);
              if (i == l) {
#pragma unroll
                for (int a = 0; a < 6; ++a) {
#pragma unroll
                  for (int c = 0; c < 6; ++c) v[a * 6 + c] += A[0][a] * A[0][c] + A[1][a] * A[1][c];
                  v[36 + a] += A[0][a] * r[0] + A[1][a] * r[1] - (W[a][0] * q[0] + W[a][1] * q[1] + W[a][2] * q[2]);
                }
              }
              for (int u = 0; u < n; ++u) {
                if (b.cam[o0 + u] != l) continue;
                double A2[2][6], B2[2][3], r2[2], W2[6][3], T2[6][3];
                lin_obs(cams, X, b, o0 + u, b.w[o0 + u], A2, B2, r2, nullptr);
                wt_of(A2, B2, vi, W2, T2);
#pragma unroll
                for (int a = 0; a < 6; ++a)
#pragma unroll
                  for (int c = 0; c < 6; ++c)
                    v[a * 6 + c] -= Tm[a][0] * W2[c][0] + Tm[a][1] * W2[c][1] + Tm[a][2] * W2[c][2];
              }
            }
          }
          const double s = block_sum64<NT>(v, red);
          if (tid < 36) {
            // S_il[a][c] is element (6l + c, 6i + a); only the lower triangle is stored
            const int a = tid / 6, c = tid % 6;
            if (i != l || c >= a) S[(6 * l + c) * kMaxN + 6 * i + a] = s + ((i == l && a == c) ? lam : 0.0);
          } else if (tid < 42 && i == l) {
            rhs[6 * i + tid - 36] = s;
          }
          __syncthreads();
        }
      // ---- warp 0: Cholesky of the reduced system and solve ----
      if (tid < 32) {
        const int n6 = 6 * N;
        bool ok = true;
        for (int k = 0; k < n6; ++k) {
          __syncwarp();
          const double d = S[k * kMaxN + k];
          if (!(d > 0.0)) ok = false;
          const double sd = d > 0.0 ? sqrt(d) : 1.0;
          __syncwarp();
          if (tid == 0) S[k * kMaxN + k] = sd;
          for (int r = k + 1 + tid; r < n6; r += 32) S[r * kMaxN + k] /= sd;
          __syncwarp();
          for (int r = k + 1 + tid; r < n6; r += 32)
            for (int c = k + 1; c <= r; ++c) S[r * kMaxN + c] -= S[r * kMaxN + k] * S[c * kMaxN + k];
        }
        __syncwarp();
        if (tid == 0) {
          si[3] = ok ? 0 : 1;
          if (ok) {
            for (int r = 0; r < n6; ++r) {
              double s = rhs[r];
              for (int c = 0; c < r; ++c) s -= S[r * kMaxN + c] * da[c];
              da[r] = s / S[r * kMaxN + r];
            }
            for (int r = n6 - 1; r >= 0; --r) {
              double s = da[r];
              for (int c = r + 1; c < n6; ++c) s -= S[c * kMaxN + r] * da[c];
              da[r] = s / S[r * kMaxN + r];
            }
          }
        }
      }
      __syncthreads();
      if (!si[3]) {
        // trial cameras
        if (tid < N) {
          CamS c = cams[tid];
          const double* d = da + 6 * tid;
          c.T[0] += d[0]; c.T[1] += d[1]; c.T[2] += d[2];
          rotate_update(d + 3, c.R);
          tcams[tid] = c;
        }
        __syncthreads();
        // ---- pass STEP: point back-substitution, trial points, trial cost ----
        double v[64];
#pragma unroll
        for (int t = 0; t < 64; ++t) v[t] = 0.0;
        for (int j = tid; j < M; j += NT) {
          const int g = pt0 + j;
          const int o0 = b.ptr[g], n = b.ptr[g + 1] - o0;
          const double X[3] = {b.X[3 * (size_t)g], b.X[3 * (size_t)g + 1], b.X[3 * (size_t)g + 2]};
          double vi[6], gb[3], q[3];
          double db[3] = {0, 0, 0};
          if (point_elim(cams, X, b, o0, n, lam, vi, gb, q)) {
            double acc[3] = {gb[0], gb[1], gb[2]};
            for (int t = 0; t < n; ++t) {
              double A[2][6], B[2][3], r[2], W[6][3], Tm[6][3];
              lin_obs(cams, X, b, o0 + t, b.w[o0 + t], A, B, r, nullptr);
              wt_of(A, B, vi, W, Tm);
              const double* d = da + 6 * b.cam[o0 + t];
#pragma unroll
              for (int c = 0; c < 3; ++c)
                acc[c] -= W[0][c] * d[0] + W[1][c] * d[1] + W[2][c] * d[2] + W[3][c] * d[3] + W[4][c] * d[4] + W[5][c] * d[5];
            }
            db[0] = vi[0] * acc[0] + vi[1] * acc[1] + vi[2] * acc[2];
            db[1] = vi[1] * acc[0] + vi[3] * acc[1] + vi[4] * acc[2];
            db[2] = vi[2] * acc[0] + vi[4] * acc[1] + vi[5] * acc[2];
            v[1] += db[0] * db[0] + db[1] * db[1] + db[2] * db[2];
            v[2] += db[0] * gb[0] + db[1] * gb[1] + db[2] * gb[2];
          }
          const double Xn[3] = {X[0] + db[0], X[1] + db[1], X[2] + db[2]};
          b.Xt[3 * (size_t)g] = Xn[0];
          b.Xt[3 * (size_t)g + 1] = Xn[1];
          b.Xt[3 * (size_t)g + 2] = Xn[2];
          for (int t = 0; t < n; ++t) {
            const int k = o0 + t;
            const int c = b.cam[k];
            Cam cm;
#pragma unroll
            for (int qq = 0; qq < 9; ++qq) cm.R[qq] = tcams[c].R[qq];
#pragma unroll
            for (int qq = 0; qq < 3; ++qq) cm.T[qq] = tcams[c].T[qq];
#pragma unroll
            for (int qq = 0; qq < 9; ++qq) cm.K[qq] = tcams[c].K[qq];
            double XX[3], e[2];
            residual<kModelStd>(cm, Xn, b.meas[2 * k], b.meas[2 * k + 1], XX, e);
            const double wk = b.w[k];
            v[0] += wk * wk * (e[0] * e[0] + e[1] * e[1]);
          }
        }
        const double s = block_sum64<NT>(v, red);
        if (tid < 3) sc[3 + tid] = s;
        __syncthreads();
        if (tid == 0) {
          double d2 = sc[4], dg = sc[5];
          for (int a = 0; a < 6 * N; ++a) { d2 += da[a] * da[a]; dg += da[a] * ga[a]; }
          sc[4] = d2;
          si[4] = 0;
          if (sqrt(d2) < o.upd_thr * (sc[6] + o.upd_thr)) {
            si[5] = V3DBA_STATUS_SMALL_UPDATE;
            si[1] = 1;
          } else {
            const double rho = (sc[0] - sc[3]) / (sc[1] * d2 + dg);
            si[4] = rho > 0.0 ? 1 : 0;
          }
        }
        __syncthreads();
        if (si[1]) break;
      } else if (tid == 0) {
        si[4] = 0;
      }
      __syncthreads();
      if (si[4]) {
        if (tid < N) cams[tid] = tcams[tid];
        for (int j = tid; j < M; j += NT) {
          const size_t g = pt0 + j;
          b.X[3 * g] = b.Xt[3 * g];
          b.X[3 * g + 1] = b.Xt[3 * g + 1];
          b.X[3 * g + 2] = b.Xt[3 * g + 2];
        }
      }
      if (tid == 0) {
        if (si[4]) {
          const double rho = (sc[0] - sc[3]) / (sc[1] * sc[4] + sc[5]);
          const double r = 2.0 * rho - 1.0;
          double lam2 = sc[1] * fmax(1.0 / 3.0, 1.0 - r * r * r);
          if (lam2 < 1e-10) lam2 = 1e-10;
          sc[1] = lam2;
          sc[2] = 2.0;
          si[2] = 1;
        } else {
          sc[1] *= sc[2];
          sc[2] *= 2.0;
          si[2] = 0;
          si[7]++;
        }
      }
      __syncthreads();
    }
    // write back
    if (tid < N) {
      for (int q = 0; q < 9; ++q) b.R[9 * (c0 + tid) + q] = cams[tid].R[q];
      for (int q = 0; q < 3; ++q) b.T[3 * (c0 + tid) + q] = cams[tid].T[q];
    }
    if (tid == 0) {
      b.status[p] = si[5];
      b.iterations[p] = it;
      b.rejected[p] = si[7];
      b.cost[p] = sc[0];
      b.lambda_out[p] = sc[1];
    }
    __syncthreads();
  }
}

}  // namespace
}  // namespace v3dba

using namespace v3dba;

// ---- host ----------------------------------------------------------------------------------

struct v3dba_batch_s {
  BatchDev d;
  std::vector<void*> allocs;
  std::vector<int> h_cam_off, h_n_cams, h_pt_off, h_n_pts, h_order, h_size;
  int total_cams = 0, total_pts = 0, total_obs = 0;
  double* d_init = nullptr;       // initial R, T, X (for reset)
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int small_threads = 64, large_threads = 128;   // autotuned block sizes
  int split = 0;                  // problems [0, split) of the order use large_threads
};

namespace {

template <typename T>
int balloc(v3dba_batch_t h, T** p, size_t n) {
  // stream-ordered, from the device's pool (which keeps what a destroyed batch freed): a batch
  // created per call does not pay cudaMalloc / cudaFree each time
  void* q = nullptr;
  int rc0 = ensure_pool();
  if (rc0) return rc0;
  if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
  cudaError_t e = cudaMallocAsync(&q, std::max<size_t>(n, 1) * sizeof(T), h->stream);
  if (e != cudaSuccess) { cudaGetLastError(); return V3DBA_ERR_OUT_OF_MEMORY; }
  h->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return V3DBA_OK;
}

template <typename T>
int bupload(v3dba_batch_t h, T** p, const std::vector<T>& v) {
  int rc = balloc(h, p, v.size());
  if (rc) return rc;
  // the host vector outlives the copy: v3dba_batch_create synchronises the stream before returning
  if (!v.empty()) V3DBA_CUDA_TRY(cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
  return V3DBA_OK;
}

void batch_free(v3dba_batch_t h) {
  if (!h) return;
  if (h->stream) {
    for (void* p : h->allocs) cudaFreeAsync(p, h->stream);
    cudaStreamSynchronize(h->stream);
  }
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int launch_range(v3dba_batch_t h, int threads, int first, int last, const BatchOpts& o) {
  if (last <= first) return V3DBA_OK;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  V3DBA_CUDA_TRY(cudaMemsetAsync(h->d.queue, 0, sizeof(unsigned), h->stream));
  int per_sm = 1;
  if (threads == 64) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batched_lm<64>, 64, 0);
  } else if (threads == 128) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batched_lm<128>, 128, 0);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batched_lm<256>, 256, 0);
  }
  const int grid = std::max(1, std::min(last - first, sms * std::max(per_sm, 1)));
  if (threads == 64) k_batched_lm<64><<<grid, 64, 0, h->stream>>>(h->d, o, first, last);
  else if (threads == 128) k_batched_lm<128><<<grid, 128, 0, h->stream>>>(h->d, o, first, last);
  else k_batched_lm<256><<<grid, 256, 0, h->stream>>>(h->d, o, first, last);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

int batch_run(v3dba_batch_t h, const v3dba_options* opts) {
  BatchOpts o;
  o.tau = opts->tau;
  o.grad_thr = opts->gradient_threshold;
  o.upd_thr = opts->update_threshold;
  o.max_iter = opts->max_iterations;
  int rc = launch_range(h, h->large_threads, 0, h->split, o);
  if (rc) return rc;
  return launch_range(h, h->small_threads, h->split, h->d.count, o);
}

}  // namespace

extern "C" {

int v3dba_batch_create(const v3dba_problem* problems, int count, v3dba_batch_t* out) {
  if (!problems || count <= 0 || !out) return V3DBA_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int total_cams = 0, total_pts = 0, total_obs = 0;
  for (int p = 0; p < count; ++p) {
    const v3dba_problem& q = problems[p];
    if (q.model != V3DBA_MODEL_STD) return V3DBA_ERR_UNSUPPORTED;
    if (q.n_cameras <= 0 || q.n_cameras > kMaxCams || q.n_points < 0 || q.n_measurements < 0) return V3DBA_ERR_UNSUPPORTED;
    if (!q.K || !q.R || !q.T || (q.n_points && !q.X) || (q.n_measurements && (!q.measurements || !q.view || !q.point)))
      return V3DBA_ERR_INVALID_ARGUMENT;
    if (!(q.inlier_threshold > 0.0)) return V3DBA_ERR_INVALID_INPUT;
    std::vector<int> cnt(q.n_points, 0);
    for (int k = 0; k < q.n_measurements; ++k) {
      if (q.view[k] < 0 || q.view[k] >= q.n_cameras || q.point[k] < 0 || q.point[k] >= q.n_points) return V3DBA_ERR_INVALID_INPUT;
      if (++cnt[q.point[k]] > kMaxTrack) return V3DBA_ERR_UNSUPPORTED;
      if (!std::isfinite(q.measurements[2 * k]) || !std::isfinite(q.measurements[2 * k + 1])) return V3DBA_ERR_INVALID_INPUT;
    }
    for (int t = 0; t < 9 * q.n_cameras; ++t)
      if (!std::isfinite(q.K[t]) || !std::isfinite(q.R[t])) return V3DBA_ERR_INVALID_INPUT;
    for (int t = 0; t < 3 * q.n_points; ++t)
      if (!std::isfinite(q.X[t])) return V3DBA_ERR_INVALID_INPUT;
    total_cams += q.n_cameras;
    total_pts += q.n_points;
    total_obs += q.n_measurements;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return V3DBA_ERR_NO_DEVICE; }
  v3dba_batch_t h = new (std::nothrow) v3dba_batch_s();
  if (!h) return V3DBA_ERR_OUT_OF_MEMORY;
  h->total_cams = total_cams; h->total_pts = total_pts; h->total_obs = total_obs;
  std::vector<double> R(9 * (size_t)total_cams), T(3 * (size_t)total_cams), K(9 * (size_t)total_cams);
  std::vector<double> X(3 * (size_t)total_pts), meas(2 * (size_t)total_obs), thr(count);
  std::vector<int> ptr(total_pts + 1, 0);
  std::vector<unsigned char> cam(total_obs);
  int co = 0, po = 0, oo = 0;
  for (int p = 0; p < count; ++p) {
    const v3dba_problem& q = problems[p];
    h->h_cam_off.push_back(co); h->h_n_cams.push_back(q.n_cameras);
    h->h_pt_off.push_back(po); h->h_n_pts.push_back(q.n_points);
    h->h_size.push_back(q.n_measurements);
    thr[p] = q.inlier_threshold;
    std::copy(q.R, q.R + 9 * q.n_cameras, R.begin() + 9 * (size_t)co);
    std::copy(q.T, q.T + 3 * q.n_cameras, T.begin() + 3 * (size_t)co);
    std::copy(q.K, q.K + 9 * q.n_cameras, K.begin() + 9 * (size_t)co);
    std::copy(q.X, q.X + 3 * q.n_points, X.begin() + 3 * (size_t)po);
    // point-major observations (stable); inputs already in point order (a triplet stage's, or
    // any BundlePointStructure's) are copied as they are
    bool sorted = true;
    for (int k = 1; k < q.n_measurements && sorted; ++k) sorted = q.point[k] >= q.point[k - 1];
    if (sorted) {
      int k = 0;
      for (int j = 0; j < q.n_points; ++j) {
        ptr[po + j] = oo + k;
        while (k < q.n_measurements && q.point[k] == j) ++k;
      }
      ptr[po + q.n_points] = oo + q.n_measurements;
      std::copy(q.measurements, q.measurements + 2 * (size_t)q.n_measurements, meas.begin() + 2 * (size_t)oo);
      for (int k2 = 0; k2 < q.n_measurements; ++k2) cam[oo + k2] = (unsigned char)q.view[k2];
    } else {
      std::vector<int> c(q.n_points + 1, 0);
      for (int k = 0; k < q.n_measurements; ++k) c[q.point[k] + 1]++;
      for (int j = 0; j < q.n_points; ++j) c[j + 1] += c[j];
      for (int j = 0; j <= q.n_points; ++j) ptr[po + j] = oo + c[j];
      std::vector<int> fill(c.begin(), c.end() - 1);
      for (int k = 0; k < q.n_measurements; ++k) {
        const int dst = oo + fill[q.point[k]]++;
        meas[2 * (size_t)dst] = q.measurements[2 * k];
        meas[2 * (size_t)dst + 1] = q.measurements[2 * k + 1];
        cam[dst] = (unsigned char)q.view[k];
      }
    }
    co += q.n_cameras; po += q.n_points; oo += q.n_measurements;
  }
  ptr[total_pts] = oo;
  // longest-processing-time order
  h->h_order.resize(count);
  std::iota(h->h_order.begin(), h->h_order.end(), 0);
  std::stable_sort(h->h_order.begin(), h->h_order.end(), [&](int a, int b2) { return h->h_size[a] > h->h_size[b2]; });
  h->split = 0;
  int rc;
#define BTRY(x) do { if ((rc = (x)) != V3DBA_OK) { batch_free(h); return rc; } } while (0)
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
    cudaGetLastError();
    batch_free(h);
    return V3DBA_ERR_CUDA;
  }
  h->d.count = count;
  BTRY(bupload(h, &h->d.cam_off, h->h_cam_off));
  BTRY(bupload(h, &h->d.n_cams, h->h_n_cams));
  BTRY(bupload(h, &h->d.pt_off, h->h_pt_off));
  BTRY(bupload(h, &h->d.n_pts, h->h_n_pts));
  BTRY(bupload(h, &h->d.order, h->h_order));
  BTRY(bupload(h, &h->d.thr, thr));
  BTRY(bupload(h, &h->d.R, R));
  BTRY(bupload(h, &h->d.T, T));
  BTRY(bupload(h, &h->d.K, K));
  BTRY(bupload(h, &h->d.X, X));
  BTRY(balloc(h, &h->d.Xt, 3 * (size_t)total_pts));
  BTRY(bupload(h, &h->d.ptr, ptr));
  BTRY(bupload(h, &h->d.meas, meas));
  BTRY(bupload(h, &h->d.cam, cam));
  BTRY(balloc(h, &h->d.w, (size_t)total_obs));
  BTRY(balloc(h, &h->d.status, count));
  BTRY(balloc(h, &h->d.iterations, count));
  BTRY(balloc(h, &h->d.rejected, count));
  BTRY(balloc(h, &h->d.cost, count));
  BTRY(balloc(h, &h->d.init_cost, count));
  BTRY(balloc(h, &h->d.lambda_out, count));
  BTRY(balloc(h, &h->d.queue, 1));
  // the initial parameters (for v3dba_batch_reset), copied on the device
  BTRY(balloc(h, &h->d_init, 9 * (size_t)total_cams + 3 * (size_t)total_cams + 3 * (size_t)total_pts));
  if (cudaMemcpyAsync(h->d_init, h->d.R, sizeof(double) * 9 * total_cams, cudaMemcpyDeviceToDevice, h->stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(h->d_init + 9 * (size_t)total_cams, h->d.T, sizeof(double) * 3 * total_cams,
                      cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess ||
      cudaMemcpyAsync(h->d_init + 12 * (size_t)total_cams, h->d.X, sizeof(double) * 3 * total_pts,
                      cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess) {
    cudaGetLastError();
    batch_free(h);
    return V3DBA_ERR_CUDA;
  }
#undef BTRY
  *out = h;
  return V3DBA_OK;
}

int v3dba_batch_create_flat(int count, const int* n_cameras, const int* n_points, const int* n_measurements,
                            const double* inlier_threshold, const double* K, const double* R, const double* T,
                            const double* X, const double* measurements, const int* view, const int* point,
                            v3dba_batch_t* out) {
  if (count <= 0 || !n_cameras || !n_points || !n_measurements || !inlier_threshold || !K || !R || !T || !out)
    return V3DBA_ERR_INVALID_ARGUMENT;
  std::vector<v3dba_problem> probs((size_t)count);
  size_t co = 0, po = 0, oo = 0;
  for (int p = 0; p < count; ++p) {
    if (n_cameras[p] < 0 || n_points[p] < 0 || n_measurements[p] < 0) return V3DBA_ERR_INVALID_ARGUMENT;
    if ((n_points[p] && !X) || (n_measurements[p] && (!measurements || !view || !point)))
      return V3DBA_ERR_INVALID_ARGUMENT;
    v3dba_problem q;
    std::memset(&q, 0, sizeof(q));
    q.model = V3DBA_MODEL_STD;
    q.n_cameras = n_cameras[p];
    q.n_points = n_points[p];
    q.n_measurements = n_measurements[p];
    q.inlier_threshold = inlier_threshold[p];
    q.K = K + 9 * co;
    q.R = R + 9 * co;
    q.T = T + 3 * co;
    q.X = X ? X + 3 * po : nullptr;
    q.measurements = measurements ? measurements + 2 * oo : nullptr;
    q.view = view ? view + oo : nullptr;
    q.point = point ? point + oo : nullptr;
    probs[p] = q;
    co += (size_t)n_cameras[p];
    po += (size_t)n_points[p];
    oo += (size_t)n_measurements[p];
  }
  return v3dba_batch_create(probs.data(), count, out);
}

int v3dba_batch_destroy(v3dba_batch_t h) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  batch_free(h);
  return V3DBA_OK;
}

int v3dba_batch_reset(v3dba_batch_t h) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  const size_t nc = h->total_cams, np = h->total_pts;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(h->d.R, h->d_init, 9 * nc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(h->d.T, h->d_init + 9 * nc, 3 * nc * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(h->d.X, h->d_init + 12 * nc, 3 * np * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(h->stream));
  return V3DBA_OK;
}

int v3dba_batch_set_schedule(v3dba_batch_t h, int large_threads, int small_threads, int split) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  auto ok = [](int t) { return t == 64 || t == 128 || t == 256; };
  if (!ok(large_threads) || !ok(small_threads) || split < 0 || split > h->d.count) return V3DBA_ERR_INVALID_ARGUMENT;
  h->large_threads = large_threads;
  h->small_threads = small_threads;
  h->split = split;
  return V3DBA_OK;
}

int v3dba_batch_minimize(v3dba_batch_t h, const v3dba_options* opts, v3dba_result* results, double* device_ms) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  v3dba_options o;
  if (opts) o = *opts; else v3dba_default_options(&o);
  V3DBA_CUDA_TRY(cudaEventRecord(h->ev0, h->stream));
  int rc = batch_run(h, &o);
  if (rc) return rc;
  V3DBA_CUDA_TRY(cudaEventRecord(h->ev1, h->stream));
  V3DBA_CUDA_TRY(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  if (device_ms) *device_ms = ms;
  if (results) {
    const int n = h->d.count;
    std::vector<int> st(n), it(n), rj(n);
    std::vector<double> c(n), ic(n), lm(n);
    V3DBA_CUDA_TRY(cudaMemcpy(st.data(), h->d.status, n * sizeof(int), cudaMemcpyDeviceToHost));
    V3DBA_CUDA_TRY(cudaMemcpy(it.data(), h->d.iterations, n * sizeof(int), cudaMemcpyDeviceToHost));
    V3DBA_CUDA_TRY(cudaMemcpy(rj.data(), h->d.rejected, n * sizeof(int), cudaMemcpyDeviceToHost));
    V3DBA_CUDA_TRY(cudaMemcpy(c.data(), h->d.cost, n * sizeof(double), cudaMemcpyDeviceToHost));
    V3DBA_CUDA_TRY(cudaMemcpy(ic.data(), h->d.init_cost, n * sizeof(double), cudaMemcpyDeviceToHost));
    V3DBA_CUDA_TRY(cudaMemcpy(lm.data(), h->d.lambda_out, n * sizeof(double), cudaMemcpyDeviceToHost));
    for (int p = 0; p < n; ++p) {
      v3dba_result& r = results[p];
      std::memset(&r, 0, sizeof(r));
      r.status = st[p]; r.iterations = it[p]; r.n_rejected = rj[p];
      r.cost = c[p]; r.initial_cost = ic[p]; r.lambda = lm[p];
      r.device_ms = ms; r.fp64_from_iteration = -1;
    }
  }
  return V3DBA_OK;
}

int v3dba_batch_get_params(v3dba_batch_t h, int index, double* R, double* T, double* X) {
  if (!h || index < 0 || index >= h->d.count) return V3DBA_ERR_INVALID_ARGUMENT;
  const size_t c0 = h->h_cam_off[index], nc = h->h_n_cams[index];
  const size_t p0 = h->h_pt_off[index], np = h->h_n_pts[index];
  if (R) V3DBA_CUDA_TRY(cudaMemcpy(R, h->d.R + 9 * c0, 9 * nc * sizeof(double), cudaMemcpyDeviceToHost));
  if (T) V3DBA_CUDA_TRY(cudaMemcpy(T, h->d.T + 3 * c0, 3 * nc * sizeof(double), cudaMemcpyDeviceToHost));
  if (X) V3DBA_CUDA_TRY(cudaMemcpy(X, h->d.X + 3 * p0, 3 * np * sizeof(double), cudaMemcpyDeviceToHost));
  return V3DBA_OK;
}

int v3dba_batch_get_all_params(v3dba_batch_t h, double* R, double* T, double* X) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  if (R) V3DBA_CUDA_TRY(cudaMemcpy(R, h->d.R, 9 * (size_t)h->total_cams * sizeof(double), cudaMemcpyDeviceToHost));
  if (T) V3DBA_CUDA_TRY(cudaMemcpy(T, h->d.T, 3 * (size_t)h->total_cams * sizeof(double), cudaMemcpyDeviceToHost));
  if (X) V3DBA_CUDA_TRY(cudaMemcpy(X, h->d.X, 3 * (size_t)h->total_pts * sizeof(double), cudaMemcpyDeviceToHost));
  return V3DBA_OK;
}

int v3dba_batch_autotune(v3dba_batch_t h, const v3dba_options* opts, int* large_threads, int* small_threads,
                         int* split) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  v3dba_options o;
  if (opts) o = *opts; else v3dba_default_options(&o);
  const int n = h->d.count;
  const int cand_threads[2][2] = {{128, 64}, {256, 128}};
  const int splits[4] = {0, n / 8, n / 4, n / 2};
  double best = 1e30;
  int bl = h->large_threads, bs = h->small_threads, bp = h->split;
  for (int c = 0; c < 2; ++c)
    for (int q = 0; q < 4; ++q) {
      const int lt = cand_threads[c][0], st = cand_threads[c][1];
      for (int alt = 0; alt < 2; ++alt) {
        const int small = alt ? lt : st;   // also try one block size for everything
        int rc = v3dba_batch_set_schedule(h, lt, small, splits[q]);
        if (rc) return rc;
        if ((rc = v3dba_batch_reset(h))) return rc;
        double ms = 0.0;
        if ((rc = v3dba_batch_minimize(h, &o, nullptr, &ms))) return rc;
        if (ms < best) { best = ms; bl = lt; bs = small; bp = splits[q]; }
      }
    }
  int rc = v3dba_batch_set_schedule(h, bl, bs, bp);
  if (rc) return rc;
  if ((rc = v3dba_batch_reset(h))) return rc;
  if (large_threads) *large_threads = bl;
  if (small_threads) *small_threads = bs;
  if (split) *split = bp;
  return V3DBA_OK;
}

int v3dba_minimize_batched(const v3dba_problem* problems, int count, const v3dba_options* opts,
                           double* const* K, double* const* R, double* const* T, double* const* dist,
                           double* const* X, v3dba_result* results) {
  (void)K;
  (void)dist;
  v3dba_batch_t h = nullptr;
  int rc = v3dba_batch_create(problems, count, &h);
  if (rc) return rc;
  rc = v3dba_batch_minimize(h, opts, results, nullptr);
  if (rc == V3DBA_OK && (R || T || X)) {
    std::vector<double> Ra(9 * (size_t)h->total_cams), Ta(3 * (size_t)h->total_cams), Xa(3 * (size_t)h->total_pts);
    rc = v3dba_batch_get_all_params(h, Ra.data(), Ta.data(), Xa.data());
    for (int p = 0; rc == V3DBA_OK && p < count; ++p) {
      const size_t c0 = h->h_cam_off[p], nc = h->h_n_cams[p], p0 = h->h_pt_off[p], np = h->h_n_pts[p];
      if (R && R[p]) std::copy(Ra.begin() + 9 * c0, Ra.begin() + 9 * (c0 + nc), R[p]);
      if (T && T[p]) std::copy(Ta.begin() + 3 * c0, Ta.begin() + 3 * (c0 + nc), T[p]);
      if (X && X[p]) std::copy(Xa.begin() + 3 * p0, Xa.begin() + 3 * (p0 + np), X[p]);
    }
  }
  v3dba_batch_destroy(h);
  return rc;
}

}  // extern "C"

// ---- triplet stage ---------------------------------------------------------------------------
//
// The steps either side of the triplet adjustment (SfM/generate_triples/src/generate_triples.cpp:
// 380-415) for all triplets of a call: k_triplet_prepare (one thread per track) triangulates and
// filters, k_triplet_assemble (one block per triplet) applies the survival tests and packs the
// surviving points and measurements point-major into the batch layout, k_batched_lm adjusts every
// accepted triplet, k_triplet_scatter returns each track's point.

namespace v3dba {
namespace {

struct StageDev {
  int n_trk = 0;
  const int* trk_tri = nullptr;     // [n_trk] triplet of each track
  const int* tptr = nullptr;        // [n_trk+1] measurements of each track (global)
  const int* mview = nullptr;       // [n_meas] triple view
  const float* mpos = nullptr;      // [2 n_meas]
  const double* focal = nullptr;    // [3 count]
  const int* trk_off = nullptr;     // [count] first track of each triplet
  const int* n_trk_of = nullptr;    // [count]
  double* Xtri = nullptr;           // [3 n_trk] linear triangulation
  unsigned char* kept = nullptr;    // [n_meas]
  int* keptcnt = nullptr;           // [n_trk] surviving measurements of a surviving track, else 0
  int* slot = nullptr;              // [n_trk] point slot inside its triplet's problem, or -1
  int* verdict = nullptr;           // [count]
  int* n_surv = nullptr;            // [count]
  int* pt_track = nullptr;          // [total point slots]
  double max_err, min_ratio;
  int min_points;
};

// Least squares of the 2K x 3 system A x = b by Householder QR (the algorithm of TNT's QR,
// V3D/include/Math/v3d_linear_tnt.h:1589-1629 and its solve, :1734-1771): column norms by hypot,
// reflector sign from the diagonal, R's diagonal kept apart.  Returns false when rank deficient.
__device__ bool qr_least_squares3(double (*A)[3], double* b, int m, double x[3]) {
  double rdiag[3];
  for (int k = 0; k < 3; ++k) {
    double nrm = 0.0;
    for (int i = k; i < m; ++i) nrm = hypot(nrm, A[i][k]);
    if (nrm != 0.0) {
      if (A[k][k] < 0.0) nrm = -nrm;
      for (int i = k; i < m; ++i) A[i][k] /= nrm;
      A[k][k] += 1.0;
      for (int j = k + 1; j < 3; ++j) {
        double s = 0.0;
        for (int i = k; i < m; ++i) s += A[i][k] * A[i][j];
        s = -s / A[k][k];
        for (int i = k; i < m; ++i) A[i][j] += s * A[i][k];
      }
    }
    rdiag[k] = -nrm;
  }
  if (rdiag[0] == 0.0 || rdiag[1] == 0.0 || rdiag[2] == 0.0) return false;
  for (int k = 0; k < 3; ++k) {
    double s = 0.0;
    for (int i = k; i < m; ++i) s += A[i][k] * b[i];
    s = -s / A[k][k];
    for (int i = k; i < m; ++i) b[i] += s * A[i][k];
  }
  for (int k = 2; k >= 0; --k) {
    b[k] /= rdiag[k];
    for (int i = 0; i < k; ++i) b[i] -= b[k] * A[i][k];
  }
  x[0] = b[0];
  x[1] = b[1];
  x[2] = b[2];
  return true;
}

// One thread per track: triangulateLinear (v3d_mviewutilities.h:260-303) and filterTripleModel
// (generate_triples.cpp:44-81).  The filter mirrors the reference's arithmetic: the projection
// rounded to float, the float difference and sum of squares, the float square root, times the
// view's focal length in double (no fused multiply-adds, so the decision is the host's).
__global__ void __launch_bounds__(128) k_triplet_prepare(BatchDev b, StageDev s) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= s.n_trk) return;
  const int t = s.trk_tri[g];
  const int c0 = b.cam_off[t];
  const int m0 = s.tptr[g], K = s.tptr[g + 1] - m0;
  double A[2 * kMaxTrack][3], rhs[2 * kMaxTrack], X[3];
  for (int q = 0; q < K; ++q) {
    const int v = s.mview[m0 + q];
    const double* R = b.R + 9 * (size_t)(c0 + v);
    const double* T = b.T + 3 * (size_t)(c0 + v);
    const double x = (double)s.mpos[2 * (m0 + q)], y = (double)s.mpos[2 * (m0 + q) + 1];
    for (int c = 0; c < 3; ++c) {
      A[2 * q][c] = __dsub_rn(__dmul_rn(x, R[6 + c]), R[c]);
      A[2 * q + 1][c] = __dsub_rn(__dmul_rn(y, R[6 + c]), R[3 + c]);
    }
    rhs[2 * q] = __dsub_rn(T[0], __dmul_rn(x, T[2]));
    rhs[2 * q + 1] = __dsub_rn(T[1], __dmul_rn(y, T[2]));
  }
  const bool ok = K > 0 && qr_least_squares3(A, rhs, 2 * K, X);
  if (!ok) X[0] = X[1] = X[2] = nan("");
  int cnt = 0;
  for (int q = 0; q < K; ++q) {
    const int v = s.mview[m0 + q];
    const double* R = b.R + 9 * (size_t)(c0 + v);
    const double* T = b.T + 3 * (size_t)(c0 + v);
    double Y[3];
    for (int r = 0; r < 3; ++r) {
      double acc = __dmul_rn(R[3 * r], X[0]);
      acc = __dadd_rn(acc, __dmul_rn(R[3 * r + 1], X[1]));
      acc = __dadd_rn(acc, __dmul_rn(R[3 * r + 2], X[2]));
      Y[r] = __dadd_rn(acc, T[r]);
    }
    const float px = (float)__ddiv_rn(Y[0], Y[2]), py = (float)__ddiv_rn(Y[1], Y[2]);
    const float dx = __fsub_rn(px, s.mpos[2 * (m0 + q)]), dy = __fsub_rn(py, s.mpos[2 * (m0 + q) + 1]);
    const float n = (float)sqrt((double)__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
    const double err = __dmul_rn(s.focal[3 * t + v], (double)n);
    const bool keep = err < s.max_err;   // false for NaN
    s.kept[m0 + q] = keep ? 1 : 0;
    cnt += keep ? 1 : 0;
  }
  s.keptcnt[g] = cnt >= 3 ? cnt : 0;
  s.Xtri[3 * (size_t)g] = X[0];
  s.Xtri[3 * (size_t)g + 1] = X[1];
  s.Xtri[3 * (size_t)g + 2] = X[2];
}

// Exclusive block-wide scan of one int per thread (256 threads); returns the prefix and the
// block total in *total.
__device__ __forceinline__ int block_scan256(int v, int* sm /* [8] */, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sm[wid] = x;
  __syncthreads();
  int base = 0, tot = 0;
  for (int w = 0; w < 8; ++w) {
    if (w < wid) base += sm[w];
    tot += sm[w];
  }
  __syncthreads();
  *total = tot;
  return base + x - v;
}

// One block (256 threads) per triplet: survival tests (generate_triples.cpp:393-398) and the
// bundle problem of the survivors, point-major as BundlePointStructure builds it
// (v3d_mviewutilities.h:136-158).
__global__ void __launch_bounds__(256) k_triplet_assemble(BatchDev b, StageDev s) {
  __shared__ int sm[8];
  const int t = blockIdx.x;
  const int g0 = s.trk_off[t], n = s.n_trk_of[t];
  int surv = 0;
  for (int base = 0; base < n; base += 256) {
    const int g = g0 + base + threadIdx.x;
    int tot;
    block_scan256((base + (int)threadIdx.x < n && s.keptcnt[g] > 0) ? 1 : 0, sm, &tot);
    surv += tot;
  }
  int verdict = V3DBA_TRIPLET_ACCEPTED;
  if (surv < s.min_points) verdict = V3DBA_TRIPLET_TOO_FEW_POINTS;
  else if ((double)surv < s.min_ratio * (double)n) verdict = V3DBA_TRIPLET_POINTS_DROPPED;
  const int pt0 = b.pt_off[t];
  const int ob0 = s.tptr[g0];   // the triplet's measurement range bounds its kept measurements
  if (threadIdx.x == 0) {
    s.verdict[t] = verdict;
    s.n_surv[t] = surv;
    b.n_pts[t] = verdict == V3DBA_TRIPLET_ACCEPTED ? surv : 0;
    b.ptr[pt0] = ob0;
  }
  int q_run = 0, o_run = 0;
  for (int base = 0; base < n; base += 256) {
    const int g = g0 + base + threadIdx.x;
    const bool in = base + (int)threadIdx.x < n;
    const int kc = in ? s.keptcnt[g] : 0;
    const bool sv = kc > 0 && verdict == V3DBA_TRIPLET_ACCEPTED;
    int tq, to;
    const int q = q_run + block_scan256(sv ? 1 : 0, sm, &tq);
    const int o = o_run + block_scan256(sv ? kc : 0, sm, &to);
    if (in) s.slot[g] = sv ? q : -1;
    if (sv) {
      const int p = pt0 + q;
      b.X[3 * (size_t)p] = s.Xtri[3 * (size_t)g];
      b.X[3 * (size_t)p + 1] = s.Xtri[3 * (size_t)g + 1];
      b.X[3 * (size_t)p + 2] = s.Xtri[3 * (size_t)g + 2];
      b.ptr[p + 1] = ob0 + o + kc;
      s.pt_track[p] = g;
      int w = ob0 + o;
      for (int m = s.tptr[g]; m < s.tptr[g + 1]; ++m) {
        if (!s.kept[m]) continue;
        b.meas[2 * (size_t)w] = (double)s.mpos[2 * m];
        b.meas[2 * (size_t)w + 1] = (double)s.mpos[2 * m + 1];
        b.cam[w] = (unsigned char)s.mview[m];
        ++w;
      }
    }
    q_run += tq;
    o_run += to;
  }
}

// One thread per track: the point after the stage.
__global__ void __launch_bounds__(256) k_triplet_scatter(BatchDev b, StageDev s, double* __restrict__ Xout) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= s.n_trk) return;
  const int t = s.trk_tri[g], q = s.slot[g];
  const double* src = (q >= 0) ? b.X + 3 * (size_t)(b.pt_off[t] + q) : s.Xtri + 3 * (size_t)g;
  Xout[3 * (size_t)g] = src[0];
  Xout[3 * (size_t)g + 1] = src[1];
  Xout[3 * (size_t)g + 2] = src[2];
}

// Per-triplet bookkeeping filled on the device: the triplet of every track, the batch layout's
// camera / point offsets, identity intrinsics and the adjustment's threshold.
__global__ void __launch_bounds__(256) k_triplet_setup(BatchDev b, int* __restrict__ trk_tri, const int* __restrict__ trk_off,
                                                       int* __restrict__ n_trk_of, double thr) {
  const int t = blockIdx.x;
  const int g0 = trk_off[t], g1 = trk_off[t + 1];
  for (int g = g0 + threadIdx.x; g < g1; g += blockDim.x) trk_tri[g] = t;
  if (threadIdx.x < 27) b.K[27 * (size_t)t + threadIdx.x] = (threadIdx.x % 9 == 0 || threadIdx.x % 9 == 4 || threadIdx.x % 9 == 8) ? 1.0 : 0.0;
  if (threadIdx.x == 0) {
    b.cam_off[t] = 3 * t;
    b.n_cams[t] = 3;
    b.pt_off[t] = g0 + t;   // one spare point slot per triplet keeps the end pointers apart
    b.thr[t] = thr;
    n_trk_of[t] = g1 - g0;
  }
}

}  // namespace
}  // namespace v3dba

namespace {

// The stage on flat inputs (all triplets concatenated); outputs flat.  See v3dba_triplet_stage_flat.
int triplet_stage_core(int count, const double* R, const double* T, const double* focal, const int32_t* tracks_of,
                       const int32_t* track_ptr, const int32_t* view, const float* pos,
                       const v3dba_triplet_stage_options& o, int32_t* verdict_out, int32_t* npts_out,
                       int32_t* status_out, int32_t* iters_out, double* cost_out, double* R_out, double* T_out,
                       double* X_out, uint8_t* kept_out, double* device_ms) {
  const size_t n_trk = (size_t)tracks_of[count];
  const size_t n_meas = n_trk > 0 ? (size_t)track_ptr[n_trk] : 0;
  if (n_trk > 0x7fffffffull - (size_t)count || n_meas > 0x7fffffffull) return V3DBA_ERR_UNSUPPORTED;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return V3DBA_ERR_NO_DEVICE; }
  // longest-processing-time order of the adjustments (by raw measurement count)
  std::vector<int> size(count), order(count);
  for (int t = 0; t < count; ++t) size[t] = track_ptr[tracks_of[t + 1]] - track_ptr[tracks_of[t]];
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return size[a] > size[c]; });
  const size_t n_slots = n_trk + count;

  PhaseTrace trace("V3DBA_TRACE_STAGE", "v3dba_triplet_stage");
  v3dba_batch_t h = new (std::nothrow) v3dba_batch_s();
  if (!h) return V3DBA_ERR_OUT_OF_MEMORY;
  h->total_cams = 3 * count;
  h->total_pts = (int)n_slots;
  h->total_obs = (int)n_meas;
  int rc;
  Arena ar;
  auto done = [&]() {
    ar.release(h->stream);
    batch_free(h);   // synchronises the stream before destroying it
  };
#define BTRY(x) do { if ((rc = (x)) != V3DBA_OK) { done(); return rc; } } while (0)
#define BCUDA(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { cudaGetLastError(); done(); \
    return _e == cudaErrorMemoryAllocation ? V3DBA_ERR_OUT_OF_MEMORY : V3DBA_ERR_CUDA; } } while (0)
#define BLAUNCH() do { note_launches(1); BCUDA(cudaPeekAtLastError()); } while (0)
#define BUP(dst, src, n) do { if ((n) > 0) BCUDA(cudaMemcpyAsync(dst, src, sizeof(*(src)) * (n), cudaMemcpyHostToDevice, h->stream)); } while (0)
#define BDOWN(dst, src, n) do { if ((n) > 0) BCUDA(cudaMemcpyAsync(dst, src, sizeof(*(src)) * (n), cudaMemcpyDeviceToHost, h->stream)); } while (0)
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
    cudaGetLastError();
    batch_free(h);
    return V3DBA_ERR_CUDA;
  }
  h->d.count = count;
  StageDev s;
  int *d_trk_tri, *d_tptr, *d_trk_off, *d_n_trk_of, *d_view;
  float* d_mpos;
  double* d_focal;
  double* d_Xout;
  ar.add(&h->d.cam_off, count);
  ar.add(&h->d.n_cams, count);
  ar.add(&h->d.pt_off, count);
  ar.add(&h->d.n_pts, count);
  ar.add(&h->d.order, count);
  ar.add(&h->d.thr, count);
  ar.add(&h->d.R, 27 * (size_t)count);
  ar.add(&h->d.T, 9 * (size_t)count);
  ar.add(&h->d.K, 27 * (size_t)count);
  ar.add(&h->d.X, 3 * n_slots);
  ar.add(&h->d.Xt, 3 * n_slots);
  ar.add(&h->d.ptr, n_slots + 1);
  ar.add(&h->d.meas, 2 * n_meas);
  ar.add(&h->d.cam, n_meas);
  ar.add(&h->d.w, n_meas);
  ar.add(&h->d.status, count);
  ar.add(&h->d.iterations, count);
  ar.add(&h->d.rejected, count);
  ar.add(&h->d.cost, count);
  ar.add(&h->d.init_cost, count);
  ar.add(&h->d.lambda_out, count);
  ar.add(&h->d.queue, 1);
  ar.add(&d_trk_tri, n_trk);
  ar.add(&d_tptr, n_trk + 1);
  ar.add(&d_trk_off, (size_t)count + 1);
  ar.add(&d_n_trk_of, count);
  ar.add(&d_view, n_meas);
  ar.add(&d_mpos, 2 * n_meas);
  ar.add(&d_focal, 3 * (size_t)count);
  ar.add(&s.Xtri, 3 * n_trk);
  ar.add(&s.kept, n_meas);
  ar.add(&s.keptcnt, n_trk);
  ar.add(&s.slot, n_trk);
  ar.add(&s.verdict, count);
  ar.add(&s.n_surv, count);
  ar.add(&s.pt_track, n_slots);
  ar.add(&d_Xout, 3 * n_trk);
  BTRY(ar.commit(h->stream));
  trace.mark("alloc", h->stream);
  // inputs: one copy of each caller array
  BUP(h->d.R, R, 27 * (size_t)count);
  BUP(h->d.T, T, 9 * (size_t)count);
  BUP(d_focal, focal, 3 * (size_t)count);
  BUP(d_trk_off, tracks_of, (size_t)count + 1);
  BUP(d_tptr, track_ptr, n_trk + 1);
  BUP(d_view, view, n_meas);
  BUP(d_mpos, pos, 2 * n_meas);
  BUP(h->d.order, order.data(), (size_t)count);
  trace.mark("upload", h->stream);
  s.n_trk = (int)n_trk;
  s.trk_tri = d_trk_tri;
  s.tptr = d_tptr;
  s.mview = d_view;
  s.mpos = d_mpos;
  s.focal = d_focal;
  s.trk_off = d_trk_off;
  s.n_trk_of = d_n_trk_of;
  s.max_err = o.max_reproj_error;
  s.min_ratio = o.min_point_ratio;
  s.min_points = o.min_points;
  BCUDA(cudaEventRecord(h->ev0, h->stream));
  k_triplet_setup<<<count, 256, 0, h->stream>>>(h->d, d_trk_tri, d_trk_off, d_n_trk_of, o.inlier_threshold);
  BLAUNCH();
  if (n_trk > 0) {
    k_triplet_prepare<<<(unsigned)((n_trk + 127) / 128), 128, 0, h->stream>>>(h->d, s);
    BLAUNCH();
  }
  k_triplet_assemble<<<count, 256, 0, h->stream>>>(h->d, s);
  BLAUNCH();
  BatchOpts bo;
  bo.tau = o.tau;
  bo.grad_thr = 1e-10;
  bo.upd_thr = 1e-10;
  bo.max_iter = o.max_iterations;
  BTRY(launch_range(h, 128, 0, count, bo));
  if (n_trk > 0) {
    k_triplet_scatter<<<(unsigned)((n_trk + 255) / 256), 256, 0, h->stream>>>(h->d, s, d_Xout);
    BLAUNCH();
  }
  BCUDA(cudaEventRecord(h->ev1, h->stream));
  trace.mark("kernels", h->stream);
  BDOWN(verdict_out, s.verdict, (size_t)count);
  BDOWN(npts_out, s.n_surv, (size_t)count);
  BDOWN(status_out, h->d.status, (size_t)count);
  BDOWN(iters_out, h->d.iterations, (size_t)count);
  BDOWN(cost_out, h->d.cost, (size_t)count);
  BDOWN(R_out, h->d.R, 27 * (size_t)count);
  BDOWN(T_out, h->d.T, 9 * (size_t)count);
  if (X_out) BDOWN(X_out, d_Xout, 3 * n_trk);
  if (kept_out) BDOWN(kept_out, s.kept, n_meas);
  BCUDA(cudaStreamSynchronize(h->stream));
  trace.mark("download");
  if (device_ms) {
    float ms = 0.f;
    BCUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    *device_ms = ms;
  }
  done();
  trace.mark("free");
#undef BTRY
#undef BCUDA
#undef BLAUNCH
#undef BUP
#undef BDOWN
  return V3DBA_OK;
}

// Shared validation of one triplet's tracks (track_ptr relative to the triplet).
int check_tracks(int n_tracks, const int32_t* track_ptr, const int32_t* view, const float* pos) {
  if (n_tracks < 0 || (n_tracks > 0 && (!track_ptr || !view || !pos))) return V3DBA_ERR_INVALID_ARGUMENT;
  if (n_tracks == 0) return V3DBA_OK;
  if (track_ptr[0] != 0) return V3DBA_ERR_INVALID_INPUT;
  for (int k = 0; k < n_tracks; ++k) {
    const int len = track_ptr[k + 1] - track_ptr[k];
    if (len < 0) return V3DBA_ERR_INVALID_INPUT;
    if (len > kMaxTrack) return V3DBA_ERR_UNSUPPORTED;
  }
  const int nm = track_ptr[n_tracks];
  unsigned bad = 0;
  for (int m = 0; m < nm; ++m) bad |= (unsigned)view[m] > 2u ? 1u : 0u;
  if (bad) return V3DBA_ERR_INVALID_INPUT;
  if (!all_finite_f(pos, 2 * (size_t)nm)) return V3DBA_ERR_INVALID_INPUT;
  return V3DBA_OK;
}

int stage_options(const v3dba_triplet_stage_options* opts, v3dba_triplet_stage_options* o) {
  v3dba_default_triplet_stage_options(o);
  if (opts) *o = *opts;
  if (!(o->inlier_threshold > 0.0) || o->max_iterations < 0 || !(o->tau >= 0.0)) return V3DBA_ERR_INVALID_ARGUMENT;
  return V3DBA_OK;
}

}  // namespace

extern "C" {

void v3dba_default_triplet_stage_options(v3dba_triplet_stage_options* o) {
  if (!o) return;
  o->max_reproj_error = 1.0;
  o->min_points = 50;
  o->min_point_ratio = 0.5;
  o->inlier_threshold = 1.0;
  o->tau = 1e-3;
  o->max_iterations = 5;
}

int v3dba_triplet_stage_flat(int count, const double* R, const double* T, const double* focal, const int32_t* tracks_of,
                             const int32_t* track_ptr, const int32_t* view, const float* pos,
                             const v3dba_triplet_stage_options* opts, int32_t* verdict, int32_t* n_points,
                             int32_t* status, int32_t* iterations, double* cost, double* R_out, double* T_out,
                             double* X_out, uint8_t* kept, double* device_ms) {
  if (count <= 0 || !R || !T || !focal || !tracks_of || !track_ptr || !verdict || !n_points || !status ||
      !iterations || !cost || !R_out || !T_out)
    return V3DBA_ERR_INVALID_ARGUMENT;
  v3dba_triplet_stage_options o;
  int rc = stage_options(opts, &o);
  if (rc) return rc;
  if (!all_finite(R, 27 * (size_t)count) || !all_finite(T, 9 * (size_t)count) || !all_finite(focal, 3 * (size_t)count))
    return V3DBA_ERR_INVALID_INPUT;
  if (tracks_of[0] != 0) return V3DBA_ERR_INVALID_INPUT;
  for (int t = 0; t < count; ++t)
    if (tracks_of[t + 1] < tracks_of[t]) return V3DBA_ERR_INVALID_INPUT;
  const int n_trk = tracks_of[count];
  if (n_trk > 0 && (!view || !pos)) return V3DBA_ERR_INVALID_ARGUMENT;
  if (track_ptr[0] != 0) return V3DBA_ERR_INVALID_INPUT;
  // the global track_ptr is one list: check it in one pass, as one triplet of n_trk tracks
  if ((rc = check_tracks(n_trk, track_ptr, view, pos))) return rc;
  return triplet_stage_core(count, R, T, focal, tracks_of, track_ptr, view, pos, o, verdict, n_points, status,
                            iterations, cost, R_out, T_out, X_out, kept, device_ms);
}

int v3dba_triplet_stage(const v3dba_triplet* trips, int count, const v3dba_triplet_stage_options* opts,
                        v3dba_triplet_result* results, double* const* Xout, uint8_t* const* keptout,
                        double* device_ms) {
  if (!trips || count <= 0 || !results) return V3DBA_ERR_INVALID_ARGUMENT;
  v3dba_triplet_stage_options o;
  int rc = stage_options(opts, &o);
  if (rc) return rc;
  size_t n_trk = 0, n_meas = 0;
  for (int t = 0; t < count; ++t) {
    const v3dba_triplet& q = trips[t];
    if ((rc = check_tracks(q.n_tracks, q.track_ptr, q.view, q.pos))) return rc;
    if (!all_finite(q.R, 27) || !all_finite(q.T, 9) || !all_finite(q.focal, 3)) return V3DBA_ERR_INVALID_INPUT;
    n_trk += q.n_tracks;
    n_meas += q.n_tracks > 0 ? q.track_ptr[q.n_tracks] : 0;
  }
  if (n_trk > 0x7fffffffull - (size_t)count || n_meas > 0x7fffffffull) return V3DBA_ERR_UNSUPPORTED;
  // concatenate
  std::vector<double> R(27 * (size_t)count), T(9 * (size_t)count), focal(3 * (size_t)count);
  std::vector<int32_t> tracks_of((size_t)count + 1), tptr(n_trk + 1), view(n_meas);
  std::vector<float> pos(2 * n_meas);
  size_t g = 0, mm = 0;
  for (int t = 0; t < count; ++t) {
    const v3dba_triplet& q = trips[t];
    std::copy(q.R, q.R + 27, R.begin() + 27 * (size_t)t);
    std::copy(q.T, q.T + 9, T.begin() + 9 * (size_t)t);
    std::copy(q.focal, q.focal + 3, focal.begin() + 3 * (size_t)t);
    tracks_of[t] = (int32_t)g;
    const int nm = q.n_tracks > 0 ? q.track_ptr[q.n_tracks] : 0;
    for (int k = 0; k < q.n_tracks; ++k) tptr[g + k] = (int32_t)mm + q.track_ptr[k];
    if (nm) {
      std::copy(q.view, q.view + nm, view.begin() + mm);
      std::copy(q.pos, q.pos + 2 * nm, pos.begin() + 2 * mm);
    }
    g += q.n_tracks;
    mm += nm;
  }
  tracks_of[count] = (int32_t)g;
  tptr[n_trk] = (int32_t)mm;
  std::vector<int32_t> verdict(count), npts(count), status(count), iters(count);
  std::vector<double> cost(count), Ro(27 * (size_t)count), To(9 * (size_t)count), Xo(3 * n_trk);
  std::vector<uint8_t> kept(n_meas);
  rc = triplet_stage_core(count, R.data(), T.data(), focal.data(), tracks_of.data(), tptr.data(), view.data(),
                          pos.data(), o, verdict.data(), npts.data(), status.data(), iters.data(), cost.data(),
                          Ro.data(), To.data(), Xo.data(), kept.data(), device_ms);
  if (rc) return rc;
  size_t gg = 0, m2 = 0;
  for (int t = 0; t < count; ++t) {
    v3dba_triplet_result& r = results[t];
    r.verdict = verdict[t];
    r.n_tracks = trips[t].n_tracks;
    r.n_points = npts[t];
    const bool acc = verdict[t] == V3DBA_TRIPLET_ACCEPTED;
    r.status = acc ? status[t] : V3DBA_STATUS_TIMEOUT;
    r.iterations = acc ? iters[t] : 0;
    r.cost = acc ? cost[t] : 0.0;
    const double* Rs = acc ? Ro.data() + 27 * (size_t)t : trips[t].R;
    const double* Ts = acc ? To.data() + 9 * (size_t)t : trips[t].T;
    std::copy(Rs, Rs + 27, r.R);
    std::copy(Ts, Ts + 9, r.T);
    const int nt = trips[t].n_tracks, nm = nt > 0 ? trips[t].track_ptr[nt] : 0;
    if (Xout && Xout[t]) std::copy(Xo.begin() + 3 * gg, Xo.begin() + 3 * (gg + nt), Xout[t]);
    if (keptout && keptout[t]) std::copy(kept.begin() + m2, kept.begin() + m2 + nm, keptout[t]);
    gg += nt;
    m2 += nm;
  }
  return V3DBA_OK;
}

}  // extern "C"
