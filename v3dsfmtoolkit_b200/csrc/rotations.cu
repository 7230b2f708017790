// Rotation averaging on the B200: the reference's SparseRotationOptimizer
// (V3D/src/Geometry/v3d_mviewutilities.cpp:470-582), run by refineConsistentRotations (:589-611)
// through SparseLevenbergOptimizer::minimize (V3D/src/Math/v3d_optimization.cpp:719-1250).
//
// The model: for every view pair k' = (i, j) with relative rotation R_ij, two 9-D measurements
// with the same residual e = vec(R_j - R_ij R_i): measurement k' is attached to view i (Jacobian
// of -R_ij R_i (I + [w_i]x)), measurement k' + n_pairs to view j (Jacobian of R_j (I + [w_j]x)).
// The "points" of the reference's optimizer have dimension 0, so its damped normal matrix is
// block diagonal with one 3x3 block per view, and its sparse LDL^T factors every block on its
// own, in natural order (block reordering keeps the columns of a block together).  The step is
// R_i <- R_i Rodrigues(delta_i).
//
// B200 design: the whole LM loop is one persistent cooperative kernel.  The data (relative
// rotations, 72 B per pair, and the rotations, 72 B per view) stay in L2 across iterations; the
// work per iteration is tiny, so the loop is bound by grid-wide barriers.  An iteration costs
// two barriers: (1) every view solves its 3x3 block and writes its trial rotation; (2) the trial
// cost is evaluated by relinearising at the trial rotations (blocks into the spare buffer), so
// that an accepted step needs no separate relinearisation.  Every block folds the per-block
// partial sums in the same fixed order, so every thread takes the same LM decision without a
// broadcast and the results are deterministic.  A warp owns a view's measurement list (built on
// the device by a stable sort of the measurements by view: ascending measurement index, the
// reference's accumulation order).
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "structure.cuh"

namespace cg = cooperative_groups;

namespace v3dba {
namespace {

constexpr int kRotThreads = 256;
constexpr int kRotWarps = kRotThreads / kWarp;
constexpr int kRotPart = 4;   // doubles per block partial

struct RotState {
  int status, iterations, relin, rejected, cur, reached_stop, pad0, pad1;
  double lambda, nu, err0, err;
};

struct RotArgs {
  int N, P, max_iter;
  const double* rel;     // [P][9]
  const int* pairs;      // [P][2]
  const int* vptr;       // [N+1] measurements of each view ...
  const int* vlist;      // [2P]  ... ascending measurement index
  double* R[2];          // [N][9] rotations: R[cur] current, R[cur^1] trial
  double* U[2];          // [N][6] packed 3x3 normal blocks (00 01 02 11 12 22)
  double* g[2];          // [N][3] J^T(-e)
  double* part;          // [2][grid][kRotPart]
  double* trace;         // [max_iter] err per relinearisation
  RotState* state;
  int cur;               // buffer holding the current rotations on entry
  double tau, nu0, gthr, uthr, plen, stop_cost;
};

__device__ __forceinline__ void load9(const double* __restrict__ p, double (&m)[9]) {
#pragma unroll
  for (int t = 0; t < 9; ++t) m[t] = p[t];
}

// Contributions of one measurement to its view's normal block u (00 01 02 11 12 22), gradient
// J^T(-e) and squared residual, accumulated into acc = {u[6], g[3], err}.
__device__ __forceinline__ void accumulate_measurement(const RotArgs& a, const double* __restrict__ R, int k,
                                                       double (&acc)[10]) {
  const bool second = k >= a.P;
  const int q = second ? k - a.P : k;
  const int i = __ldg(a.pairs + 2 * q), j = __ldg(a.pairs + 2 * q + 1);
  double Ri[9];
  load9(R + 9 * (size_t)i, Ri);
  const double* __restrict__ Rj = R + 9 * (size_t)j;
  const double* __restrict__ Rij = a.rel + 9 * (size_t)q;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    // one row of R_ij and R_j at a time keeps the live registers down
    const double m0 = __ldg(Rij + 3 * r), m1 = __ldg(Rij + 3 * r + 1), m2 = __ldg(Rij + 3 * r + 2);
    double p[3], e[3], A[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double rj = Rj[3 * r + c];
      p[c] = m0 * Ri[c] + m1 * Ri[3 + c] + m2 * Ri[6 + c];
      e[c] = rj - p[c];
      A[c] = second ? rj : -p[c];
      acc[9] += e[c] * e[c];
    }
    // rows 3r..3r+2 of the 9x3 Jacobian: [0 -A2 A1], [A2 0 -A0], [-A1 A0 0]
    acc[0] += A[1] * A[1] + A[2] * A[2];
    acc[1] -= A[0] * A[1];
    acc[2] -= A[0] * A[2];
    acc[3] += A[0] * A[0] + A[2] * A[2];
    acc[4] -= A[1] * A[2];
    acc[5] += A[0] * A[0] + A[1] * A[1];
    acc[6] -= A[2] * e[1] - A[1] * e[2];
    acc[7] -= A[0] * e[2] - A[2] * e[0];
    acc[8] -= A[1] * e[0] - A[0] * e[1];
  }
}

// Sum of acc over a group of G lanes (aligned, G a power of two <= 32).  The first step is
// transposed: the lower half of the group keeps values 0-4, the upper half 5-9, so one shuffle
// per value pair; the halves then finish with butterflies.  Afterwards lane 0 of the group holds
// the totals of values 0-4 and lane G/2 those of values 5-9 (each in the same slots of acc).
template <int G>
__device__ __forceinline__ void group_sum(double (&acc)[10], int lane) {
  if (G == 1) return;
  const bool upper = (lane & (G / 2)) != 0;
#pragma unroll
  for (int t = 0; t < 5; ++t) {
    const double send = upper ? acc[t] : acc[5 + t];
    const double got = __shfl_xor_sync(0xffffffffu, send, G / 2);
    if (upper)
      acc[5 + t] += got;
    else
      acc[t] += got;
  }
#pragma unroll
  for (int o = G / 4; o > 0; o >>= 1) {
#pragma unroll
    for (int t = 0; t < 5; ++t) {
      const double mine = upper ? acc[5 + t] : acc[t];
      const double got = __shfl_xor_sync(0xffffffffu, mine, o);
      if (upper)
        acc[5 + t] = mine + got;
      else
        acc[t] = mine + got;
    }
  }
}

// Grid-wide fold of NV values (the first NS summed, the rest max-reduced): per-block partials,
// one barrier, then warp 0 of every block combines the partials in a fixed order.  The
// partials alternate between two buffers (a buffer is rewritten two folds later, after every
// block has passed the barrier in between).
template <int NV, int NS>
__device__ __forceinline__ void grid_fold(double (&v)[NV], double* part, int& parity, cg::grid_group& grid) {
  static_assert(NV <= kRotPart, "partial stride");
  __shared__ double red[kRotWarps * kRotPart];
  block_reduce<NV, NS>(v, red);
  double* pb = part + (size_t)parity * gridDim.x * kRotPart;
  if (threadIdx.x == 0)
#pragma unroll
    for (int t = 0; t < NV; ++t) pb[(size_t)blockIdx.x * kRotPart + t] = v[t];
  grid.sync();
  if (threadIdx.x < kWarp) {
    double s[NV];
#pragma unroll
    for (int t = 0; t < NV; ++t) s[t] = t < NS ? 0.0 : -1e300;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kWarp)
#pragma unroll
      for (int t = 0; t < NV; ++t) {
        const double x = pb[(size_t)b * kRotPart + t];
        s[t] = t < NS ? s[t] + x : (x > s[t] ? x : s[t]);
      }
#pragma unroll
    for (int t = 0; t < NV; ++t) s[t] = t < NS ? warp_sum(s[t]) : warp_max(s[t]);
    if (threadIdx.x == 0)
#pragma unroll
      for (int t = 0; t < NV; ++t) red[t] = s[t];
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < NV; ++t) v[t] = red[t];
  __syncthreads();
  parity ^= 1;
}

// Linearises every view at rotations R into U/g; returns {err, max |g|, max diag U} folded.
// A group of G lanes owns a view and strides over its measurement list.
template <int G>
__device__ __forceinline__ void linearize_all(const RotArgs& a, const double* R, double* U, double* g, double (&out)[3],
                                              int& parity, cg::grid_group& grid) {
  const int lane = threadIdx.x & 31;
  const int sub = lane & (G - 1);
  const int group = (blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int ngroups = (gridDim.x * blockDim.x) / G;
  double err = 0.0, gmax = 0.0, dmax = -1e300;
  // every lane of a warp runs the same number of rounds (shuffles need the full warp)
  const int rounds = (a.N + ngroups - 1) / ngroups;
  for (int r = 0; r < rounds; ++r) {
    const int v = group + r * ngroups;
    double acc[10];
#pragma unroll
    for (int t = 0; t < 10; ++t) acc[t] = 0.0;
    if (v < a.N) {
      const int end = a.vptr[v + 1];
#pragma unroll 2
      for (int t = a.vptr[v] + sub; t < end; t += G) accumulate_measurement(a, R, a.vlist[t], acc);
    }
    group_sum<G>(acc, lane);
    if (v < a.N) {
      if (sub == 0) {
#pragma unroll
        for (int t = 0; t < 5; ++t) U[6 * (size_t)v + t] = acc[t];
        dmax = fmax(dmax, fmax(acc[0], acc[3]));
      }
      if (sub == (G > 1 ? G / 2 : 0)) {
        U[6 * (size_t)v + 5] = acc[5];
#pragma unroll
        for (int t = 0; t < 3; ++t) g[3 * (size_t)v + t] = acc[6 + t];
        err += acc[9];
        gmax = fmax(gmax, fmax(fabs(acc[6]), fmax(fabs(acc[7]), fabs(acc[8]))));
        dmax = fmax(dmax, acc[5]);
      }
    }
  }
  out[0] = err;
  out[1] = gmax;
  out[2] = dmax;
  grid_fold<3, 1>(out, a.part, parity, grid);
}

// (U + lambda I) d = g by the up-looking LDL^T of LDL_numeric / LDL_lsolve / LDL_dsolve /
// LDL_ltsolve (v3d_optimization.cpp:102-230) on one 3x3 block in natural order.  Returns false
// when a pivot is exactly zero (the reference's factorisation failure).
__device__ __forceinline__ bool ldl_solve3(const double* __restrict__ u, double lambda, const double* __restrict__ gv,
                                           double (&d)[3]) {
  const double a00 = u[0] + lambda, a01 = u[1], a02 = u[2];
  const double a11 = u[3] + lambda, a12 = u[4], a22 = u[5] + lambda;
  const double D0 = a00;
  if (D0 == 0.0) return false;
  const double L10 = a01 / D0;
  const double D1 = a11 - L10 * a01;
  if (D1 == 0.0) return false;
  const double y1 = a12 - L10 * a02;
  const double L20 = a02 / D0;
  double D2 = a22 - L20 * a02;
  const double L21 = y1 / D1;
  D2 -= L21 * y1;
  if (D2 == 0.0) return false;
  double x0 = gv[0], x1 = gv[1], x2 = gv[2];
  x1 -= L10 * x0;
  x2 -= L20 * x0;
  x2 -= L21 * x1;
  x0 /= D0;
  x1 /= D1;
  x2 /= D2;
  x1 -= L21 * x2;
  x0 -= L10 * x1;
  x0 -= L20 * x2;
  d[0] = x0;
  d[1] = x1;
  d[2] = x2;
  return true;
}

// Rn = R * Rodrigues(w) (createRotationMatrixRodrigues, V3D/include/Math/v3d_mathutilities.h:
// 162-183: identity for |w| <= 1e-6).
__device__ __forceinline__ void rotate_right(const double* __restrict__ R, const double (&w)[3], double* __restrict__ Rn) {
  const double th = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
  double M[9] = {1.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0};
  if (fabs(th) > 1e-6) {
    const double J[9] = {0.0, -w[2], w[1], w[2], 0.0, -w[0], -w[1], w[0], 0.0};
    double s, c;
    sincos(th, &s, &c);
    const double c1 = s / th, c2 = (1.0 - c) / (th * th);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int col = 0; col < 3; ++col) {
        const double j2 = J[3 * r] * J[col] + J[3 * r + 1] * J[3 + col] + J[3 * r + 2] * J[6 + col];
        M[3 * r + col] += c1 * J[3 * r + col] + c2 * j2;
      }
  }
  double Rv[9];
  load9(R, Rv);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int col = 0; col < 3; ++col)
      Rn[3 * r + col] = Rv[3 * r] * M[col] + Rv[3 * r + 1] * M[3 + col] + Rv[3 * r + 2] * M[6 + col];
}

template <int G>
__global__ void __launch_bounds__(kRotThreads, 2) k_rot_lm(RotArgs a) {
  cg::grid_group grid = cg::this_grid();
  int parity = 0;
  int cur = a.cur, lb = 0;   // rotations / normal-block buffers of the current linearisation
  double lin[3];
  linearize_all<G>(a, a.R[cur], a.U[lb], a.g[lb], lin, parity, grid);
  double err = lin[0], gmax = lin[1];
  const double err0 = err;
  double err_relin = err0;   // err at the last relinearisation (the reported cost)
  double lambda = 0.0, nu = a.nu0;
  int status = V3DBA_STATUS_TIMEOUT, relin = 0, rejected = 0, reached_stop = 0;
  bool compute = true;
  int it = 0;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  for (; it < a.max_iter; ++it) {
    if (compute) {
      if (tid == 0) a.trace[relin] = err;
      ++relin;
      err_relin = err;
      if (gmax < a.gthr) {
        status = V3DBA_STATUS_CONVERGED;
        break;
      }
      if (it == 0) lambda = a.tau * lin[2];
    }
    // (1) damped block solves and trial rotations
    double s[3] = {0.0, 0.0, 0.0};   // |d|^2, d.g, failed blocks
    {
      const double* U = a.U[lb];
      const double* g = a.g[lb];
      const double* Rc = a.R[cur];
      double* Rt = a.R[cur ^ 1];
      for (int v = tid; v < a.N; v += nthreads) {
        double u[6], gv[3], d[3];
#pragma unroll
        for (int t = 0; t < 6; ++t) u[t] = U[6 * (size_t)v + t];
#pragma unroll
        for (int t = 0; t < 3; ++t) gv[t] = g[3 * (size_t)v + t];
        if (!ldl_solve3(u, lambda, gv, d)) {
          s[2] += 1.0;
          continue;
        }
        s[0] += d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        s[1] += d[0] * gv[0] + d[1] * gv[1] + d[2] * gv[2];
        rotate_right(Rc + 9 * (size_t)v, d, Rt + 9 * (size_t)v);
      }
    }
    grid_fold<3, 3>(s, a.part, parity, grid);
    bool accept = false;
    if (s[2] == 0.0) {
      if (sqrt(s[0]) < a.uthr * (a.plen + a.uthr)) {
        status = V3DBA_STATUS_SMALL_UPDATE;
        break;
      }
      // (2) trial cost, relinearised at the trial rotations into the spare block buffers
      double tr[3];
      linearize_all<G>(a, a.R[cur ^ 1], a.U[lb ^ 1], a.g[lb ^ 1], tr, parity, grid);
      const double rho = (err - tr[0]) / (lambda * s[0] + s[1]);
      if (rho > 0.0) {
        accept = true;
        const double r = 2.0 * rho - 1.0;
        lambda *= fmax(1.0 / 3.0, 1.0 - r * r * r);
        if (lambda < 1e-10) lambda = 1e-10;
        nu = 2.0;
        cur ^= 1;
        lb ^= 1;
        err = tr[0];
        gmax = tr[1];
        compute = true;
        if (a.stop_cost > 0.0 && err <= a.stop_cost) {
          reached_stop = 1;
          err_relin = err;
          ++it;
          break;
        }
      }
    }
    if (!accept) {
      ++rejected;
      lambda *= nu;
      nu *= 2.0;
      compute = false;
    }
  }
  if (tid == 0) {
    RotState st;
    st.status = status;
    st.iterations = it;
    st.relin = relin;
    st.rejected = rejected;
    st.cur = cur;
    st.reached_stop = reached_stop;
    st.pad0 = st.pad1 = 0;
    st.lambda = lambda;
    st.nu = nu;
    st.err0 = err0;
    st.err = err_relin;
    *a.state = st;
  }
}

// key of measurement k: the view it is attached to
__global__ void k_rot_keys(const int* __restrict__ pairs, int P, int* __restrict__ keys) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < 2L * P) keys[k] = k < P ? pairs[2 * k] : pairs[2 * (k - P) + 1];
}

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

using RotKernel = void (*)(RotArgs);

RotKernel rot_kernel(int G) {
  switch (G) {
    case 4: return k_rot_lm<4>;
    case 8: return k_rot_lm<8>;
    case 16: return k_rot_lm<16>;
    default: return k_rot_lm<32>;
  }
}

// Lanes per view: the group size that minimises (views per group) x (measurement rounds per
// view + reduction steps) for the grid's lane count and the mean measurements per view.
int pick_group(long n_views, long n_meas, long lanes) {
  int best = 32;
  double best_cost = 1e300;
  const double mean = n_views > 0 ? (double)n_meas / (double)n_views : 0.0;
  for (int G = 4; G <= 32; G *= 2) {
    const long groups = std::max(1L, lanes / G);
    const double seq = std::ceil((double)n_views / (double)groups);
    const double cost = seq * (std::ceil(mean / G) + 0.5 * std::log2((double)G));
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = G;
    }
  }
  return best;
}

}  // namespace
}  // namespace v3dba

using namespace v3dba;

struct v3dba_rotations_s {
  int N = 0, P = 0, full_grid = 1, cur = 0, G = 32;
  double nu = 2.0;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  char* arena = nullptr;
  size_t trace_cap = 0;
  double* trace = nullptr;   // trace buffer (grown on demand, separate from the arena)
  double *rel = nullptr, *R0 = nullptr, *R[2] = {nullptr, nullptr}, *U[2] = {nullptr, nullptr};
  double *g[2] = {nullptr, nullptr}, *part = nullptr;
  int *pairs = nullptr, *vptr = nullptr, *vlist = nullptr;
  RotState* state = nullptr;
};

namespace {

void release(v3dba_rotations h) {
  if (!h) return;
  if (h->arena) cudaFreeAsync(h->arena, h->st);
  if (h->trace) cudaFreeAsync(h->trace, h->st);
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->e0) cudaEventDestroy(h->e0);
  if (h->e1) cudaEventDestroy(h->e1);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

int grid_for(v3dba_rotations h, int G) {
  const long want = std::max(1L, ((long)h->N * G + kRotThreads - 1) / kRotThreads);
  return (int)std::max(1L, std::min((long)h->full_grid, want));
}

int run(v3dba_rotations h, const v3dba_options* o, int max_iter, RotState* out, float* ms) {
  if ((size_t)std::max(max_iter, 1) > h->trace_cap) {
    if (h->trace) cudaFreeAsync(h->trace, h->st);
    h->trace = nullptr;
    h->trace_cap = 0;
    V3DBA_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&h->trace), sizeof(double) * std::max(max_iter, 1), h->st));
    h->trace_cap = (size_t)std::max(max_iter, 1);
  }
  RotArgs a;
  a.N = h->N;
  a.P = h->P;
  a.max_iter = max_iter;
  a.rel = h->rel;
  a.pairs = h->pairs;
  a.vptr = h->vptr;
  a.vlist = h->vlist;
  a.R[0] = h->R[0];
  a.R[1] = h->R[1];
  a.U[0] = h->U[0];
  a.U[1] = h->U[1];
  a.g[0] = h->g[0];
  a.g[1] = h->g[1];
  a.part = h->part;
  a.trace = h->trace;
  a.state = h->state;
  a.cur = h->cur;
  a.tau = o->tau;
  a.nu0 = h->nu;
  a.gthr = o->gradient_threshold;
  a.uthr = o->update_threshold;
  a.plen = std::sqrt(3.0 * h->N);
  a.stop_cost = o->stop_cost;
  void* args[] = {&a};
  V3DBA_CUDA_TRY(cudaEventRecord(h->e0, h->st));
  V3DBA_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)rot_kernel(h->G), grid_for(h, h->G), kRotThreads, args, 0,
                                             h->st));
  note_launches(1);
  V3DBA_CUDA_TRY(cudaEventRecord(h->e1, h->st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(out, h->state, sizeof(RotState), cudaMemcpyDeviceToHost, h->st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(h->st));
  if (ms) V3DBA_CUDA_TRY(cudaEventElapsedTime(ms, h->e0, h->e1));
  h->cur = out->cur;
  return V3DBA_OK;
}

}  // namespace

extern "C" {

int v3dba_rotations_create(int n_views, int n_pairs, const double* relative_rotations, const int32_t* view_pairs,
                           const double* rotations, v3dba_rotations* out) {
  if (!out || n_views < 0 || n_pairs < 0 || (n_pairs > 0 && (!relative_rotations || !view_pairs)) ||
      (n_views > 0 && !rotations))
    return V3DBA_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if ((long)n_pairs * 2 > 0x7fffffffL || (long)n_views * 9 > 0x7fffffffL) return V3DBA_ERR_UNSUPPORTED;
  for (long t = 0; t < 2L * n_pairs; ++t)
    if (view_pairs[t] < 0 || view_pairs[t] >= n_views) return V3DBA_ERR_INVALID_INPUT;
  if (!all_finite(relative_rotations, 9 * (size_t)n_pairs) || !all_finite(rotations, 9 * (size_t)n_views))
    return V3DBA_ERR_INVALID_INPUT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return V3DBA_ERR_NO_DEVICE;
  }
  v3dba_rotations h = new (std::nothrow) v3dba_rotations_s;
  if (!h) return V3DBA_ERR_OUT_OF_MEMORY;
  h->N = n_views;
  h->P = n_pairs;
#define TRY(x)            \
  do {                    \
    int _rc = (x);        \
    if (_rc) {            \
      release(h);         \
      return _rc;         \
    }                     \
  } while (0)
#define CTRY(x)                                                                                        \
  do {                                                                                                 \
    cudaError_t _e = (x);                                                                              \
    if (_e != cudaSuccess) {                                                                           \
      fprintf(stderr, "v3dba: %s failed: %s\n", #x, cudaGetErrorString(_e));                           \
      release(h);                                                                                      \
      return _e == cudaErrorMemoryAllocation ? V3DBA_ERR_OUT_OF_MEMORY : V3DBA_ERR_CUDA;               \
    }                                                                                                  \
  } while (0)
  TRY(ensure_pool());
  CTRY(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  CTRY(cudaEventCreate(&h->e0));
  CTRY(cudaEventCreate(&h->e1));
  int dev = 0, sms = 148, per_sm = 1;
  CTRY(cudaGetDevice(&dev));
  CTRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // occupancy of the instantiations is the same (one register budget); pick the group size for
  // the full grid, then trim the grid to what the views need
  CTRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rot_lm<32>, kRotThreads, 0));
  h->full_grid = sms * std::max(per_sm, 1);
  h->G = pick_group(n_views, 2L * n_pairs, (long)h->full_grid * kRotThreads);
  const size_t N = n_views, P = n_pairs;
  // one arena for every buffer
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += align_up(std::max<size_t>(bytes, 1));
    return at;
  };
  const size_t o_rel = take(72 * P), o_R0 = take(72 * N), o_Ra = take(72 * N), o_Rb = take(72 * N);
  const size_t o_Ua = take(48 * N), o_Ub = take(48 * N), o_ga = take(24 * N), o_gb = take(24 * N);
  const size_t o_part = take(sizeof(double) * 2 * kRotPart * (size_t)h->full_grid);
  const size_t o_pairs = take(8 * P), o_vptr = take(4 * (N + 1)), o_vlist = take(8 * P), o_keys = take(8 * P);
  const size_t o_state = take(sizeof(RotState));
  CTRY(cudaMallocAsync(reinterpret_cast<void**>(&h->arena), off, h->st));
  char* b = h->arena;
  h->rel = reinterpret_cast<double*>(b + o_rel);
  h->R0 = reinterpret_cast<double*>(b + o_R0);
  h->R[0] = reinterpret_cast<double*>(b + o_Ra);
  h->R[1] = reinterpret_cast<double*>(b + o_Rb);
  h->U[0] = reinterpret_cast<double*>(b + o_Ua);
  h->U[1] = reinterpret_cast<double*>(b + o_Ub);
  h->g[0] = reinterpret_cast<double*>(b + o_ga);
  h->g[1] = reinterpret_cast<double*>(b + o_gb);
  h->part = reinterpret_cast<double*>(b + o_part);
  h->pairs = reinterpret_cast<int*>(b + o_pairs);
  h->vptr = reinterpret_cast<int*>(b + o_vptr);
  h->vlist = reinterpret_cast<int*>(b + o_vlist);
  int* keys = reinterpret_cast<int*>(b + o_keys);
  h->state = reinterpret_cast<RotState*>(b + o_state);
  if (P > 0) {
    CTRY(cudaMemcpyAsync(h->rel, relative_rotations, 72 * P, cudaMemcpyHostToDevice, h->st));
    CTRY(cudaMemcpyAsync(h->pairs, view_pairs, 8 * P, cudaMemcpyHostToDevice, h->st));
  }
  if (N > 0) {
    CTRY(cudaMemcpyAsync(h->R0, rotations, 72 * N, cudaMemcpyHostToDevice, h->st));
    CTRY(cudaMemcpyAsync(h->R[0], h->R0, 72 * N, cudaMemcpyDeviceToDevice, h->st));
  }
  if (P > 0) {
    k_rot_keys<<<(unsigned)((2 * P + 255) / 256), 256, 0, h->st>>>(h->pairs, n_pairs, keys);
    {
      note_launches(1);
      cudaError_t e = cudaPeekAtLastError();
      if (e != cudaSuccess) {
        fprintf(stderr, "v3dba: launch failed: %s\n", cudaGetErrorString(e));
        release(h);
        return V3DBA_ERR_CUDA;
      }
    }
  }
  TRY(group_by_key_device(keys, 2 * n_pairs, n_views, h->vlist, h->vptr, h->st));
  CTRY(cudaStreamSynchronize(h->st));
#undef TRY
#undef CTRY
  *out = h;
  return V3DBA_OK;
}

int v3dba_rotations_destroy(v3dba_rotations h) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  release(h);
  return V3DBA_OK;
}

int v3dba_rotations_minimize(v3dba_rotations h, const v3dba_options* opts, v3dba_result* result) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  v3dba_options o;
  v3dba_default_options(&o);
  o.max_iterations = 200;   // SparseRotationOptimizer's constructor (v3d_mviewutilities.cpp:479-484)
  if (opts) o = *opts;
  if (o.max_iterations < 0 || !(o.tau >= 0.0)) return V3DBA_ERR_INVALID_ARGUMENT;
  RotState s;
  float ms = 0.f;
  std::memset(&s, 0, sizeof(s));
  if (h->N == 0) {   // nothing varies: the reference returns CONVERGED without iterating
    s.status = V3DBA_STATUS_CONVERGED;
  } else {
    const int rc = run(h, &o, o.max_iterations, &s, &ms);
    if (rc) return rc;
    h->nu = s.nu;
    if (o.verbosity >= 1 && s.relin > 0) {
      std::vector<double> tr(s.relin);
      if (cudaMemcpy(tr.data(), h->trace, sizeof(double) * s.relin, cudaMemcpyDeviceToHost) == cudaSuccess)
        for (double e : tr) printf("SparseLevenbergOptimizer: |residual|^2 = %.17g\n", e);
    }
  }
  if (result) {
    std::memset(result, 0, sizeof(*result));
    result->status = s.status;
    result->iterations = s.iterations;
    result->n_relinearizations = s.relin;
    result->n_rejected = s.rejected;
    result->initial_cost = s.err0;
    result->cost = s.err;
    result->lambda = s.lambda;
    result->device_ms = ms;
    result->reached_stop_cost = s.reached_stop;
    result->fp64_from_iteration = -1;
  }
  return V3DBA_OK;
}

int v3dba_rotations_get(v3dba_rotations h, double* rotations) {
  if (!h || (h->N > 0 && !rotations)) return V3DBA_ERR_INVALID_ARGUMENT;
  if (h->N == 0) return V3DBA_OK;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(rotations, h->R[h->cur], 72 * (size_t)h->N, cudaMemcpyDeviceToHost, h->st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(h->st));
  return V3DBA_OK;
}

int v3dba_rotations_set(v3dba_rotations h, const double* rotations) {
  if (!h || (h->N > 0 && !rotations)) return V3DBA_ERR_INVALID_ARGUMENT;
  if (!all_finite(rotations, 9 * (size_t)h->N)) return V3DBA_ERR_INVALID_INPUT;
  h->nu = 2.0;
  if (h->N == 0) return V3DBA_OK;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(h->R[h->cur], rotations, 72 * (size_t)h->N, cudaMemcpyHostToDevice, h->st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(h->st));
  return V3DBA_OK;
}

int v3dba_rotations_reset(v3dba_rotations h) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  h->nu = 2.0;
  h->cur = 0;
  if (h->N == 0) return V3DBA_OK;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(h->R[0], h->R0, 72 * (size_t)h->N, cudaMemcpyDeviceToDevice, h->st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(h->st));
  return V3DBA_OK;
}

int v3dba_rotations_set_group(v3dba_rotations h, int group) {
  if (!h || (group != 4 && group != 8 && group != 16 && group != 32)) return V3DBA_ERR_INVALID_ARGUMENT;
  h->G = group;
  return V3DBA_OK;
}

int v3dba_rotations_autotune(v3dba_rotations h, int* group) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  if (h->N > 0) {
    v3dba_options o;
    v3dba_default_options(&o);
    int best = h->G;
    float best_ms = 1e30f;
    for (int G = 4; G <= 32; G *= 2) {
      h->G = G;
      float t_min = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {   // zero iterations: one linearisation sweep, rotations untouched
        RotState s;
        float ms = 0.f;
        const int rc = run(h, &o, 0, &s, &ms);
        if (rc) return rc;
        t_min = std::min(t_min, ms);
      }
      if (t_min < best_ms) {
        best_ms = t_min;
        best = G;
      }
    }
    h->G = best;
  }
  if (group) *group = h->G;
  return V3DBA_OK;
}

int v3dba_rotations_cost(v3dba_rotations h, double* cost) {
  if (!h || !cost) return V3DBA_ERR_INVALID_ARGUMENT;
  *cost = 0.0;
  if (h->N == 0) return V3DBA_OK;
  v3dba_options o;
  v3dba_default_options(&o);
  RotState s;
  const int rc = run(h, &o, 0, &s, nullptr);   // zero iterations: the first linearisation only
  if (rc) return rc;
  *cost = s.err0;
  return V3DBA_OK;
}

int v3dba_refine_consistent_rotations(int n_views, int n_pairs, const double* relative_rotations,
                                      const int32_t* view_pairs, double* rotations, const v3dba_options* opts,
                                      v3dba_result* result) {
  v3dba_rotations h = nullptr;
  int rc = v3dba_rotations_create(n_views, n_pairs, relative_rotations, view_pairs, rotations, &h);
  if (rc) return rc;
  rc = v3dba_rotations_minimize(h, opts, result);
  if (!rc) rc = v3dba_rotations_get(h, rotations);
  v3dba_rotations_destroy(h);
  return rc;
}

}  // extern "C"
