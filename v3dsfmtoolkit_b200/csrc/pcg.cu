// Block-Jacobi preconditioned conjugate gradients on the reduced camera system, for scenes whose
// reduced system is too large to factor densely (thousands of cameras).
//
// The reference always factors the full damped normal matrix with a sparse LDL^T
// (V3D/src/Math/v3d_optimization.cpp:1096-1145); on a 2,000-camera scene its camera part fills
// in densely.  Here the Schur complement S (camera-pair blocks, dA x dA) is kept block-sparse and
// solved inexactly per LM step: stop at |r| <= tol |b| (tol 1e-6 by default) or after max_iter
// iterations.  The blocks are stored in `Real` (FP32 in mixed mode); vectors, dot products and
// the preconditioner (the inverses of the diagonal blocks) are FP64.
//
// The whole iteration runs in one persistent cooperative kernel: grid-wide barriers separate the
// phases, grid reductions write per-block partials that every block then folds in the same fixed
// order (deterministic), and the stopping test is taken on the device.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "lm.cuh"

namespace cg = cooperative_groups;

namespace v3dba {
namespace {

constexpr int kPcgThreads = 256;
constexpr int kPcgWarps = kPcgThreads / 32;

struct PcgArgs {
  int N, DA, n;                    // cameras, block size, unknowns (N * DA)
  const int* rp;                   // [N+1] row pointer over both triangles
  const int* rb;                   // block id of each row entry
  const int* rc;                   // column camera of each row entry
  const unsigned char* rt;         // 1 when the stored block is (col, row): use its transpose
  const void* Sb;                  // blocks, dA x dA row-major, Real
  int fp64;                        // Real is double
  const double* Pinv;              // [N] dA x dA inverse diagonal blocks
  const double* b;                 // rhs (n)
  double* x;                       // solution (n)
  double* r; double* z; double* p; double* Ap;
  double* part;                    // [gridDim * 4] partials
  double tol;
  int max_iter;
  int* iters_out;
  int* fail;
};

template <typename Real>
__device__ __forceinline__ double sb_at(const PcgArgs& a, int blk, int r, int c) {
  return double(reinterpret_cast<const Real*>(a.Sb)[(size_t)blk * a.DA * a.DA + r * a.DA + c]);
}

// y = S v for the camera rows handled by this block (warp per camera row, lanes over entries).
template <typename Real>
__device__ void matvec_rows(const PcgArgs& a, const double* v, double* y) {
  const int lane = threadIdx.x & 31;
  const int warp = blockIdx.x * kPcgWarps + (threadIdx.x >> 5);
  const int nwarps = gridDim.x * kPcgWarps;
  const int DA = a.DA;
  for (int i = warp; i < a.N; i += nwarps) {
    double acc[13];
#pragma unroll
    for (int t = 0; t < 13; ++t) acc[t] = 0.0;
    for (int e = a.rp[i] + lane; e < a.rp[i + 1]; e += 32) {
      const int blk = a.rb[e], col = a.rc[e];
      const bool tr = a.rt[e] != 0;
      const double* vc = v + (size_t)col * DA;
      for (int r = 0; r < DA; ++r) {
        double s = 0.0;
        for (int c = 0; c < DA; ++c) s += (tr ? sb_at<Real>(a, blk, c, r) : sb_at<Real>(a, blk, r, c)) * vc[c];
        acc[r] += s;
      }
    }
    for (int r = 0; r < DA; ++r) {
      const double s = warp_sum(acc[r]);
      if (lane == 0) y[(size_t)i * DA + r] = s;
    }
  }
}

__device__ __forceinline__ void precond_rows(const PcgArgs& a, const double* r, double* z) {
  const int DA = a.DA;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.N; i += gridDim.x * blockDim.x) {
    const double* P = a.Pinv + (size_t)i * DA * DA;
    const double* ri = r + (size_t)i * DA;
    for (int q = 0; q < DA; ++q) {
      double s = 0.0;
      for (int c = 0; c < DA; ++c) s += P[q * DA + c] * ri[c];
      z[(size_t)i * DA + q] = s;
    }
  }
}

// Grid-wide deterministic sums of NV values: per-block partials, then every block folds them in
// block order.  Must be called by all threads of all blocks.
template <int NV>
__device__ void grid_sums(double (&v)[NV], double* part, cg::grid_group& grid) {
  __shared__ double red[kPcgWarps * 4];
  block_reduce<NV, NV>(v, red);
  if (threadIdx.x == 0)
    for (int t = 0; t < NV; ++t) part[(size_t)blockIdx.x * 4 + t] = v[t];
  grid.sync();
  for (int t = 0; t < NV; ++t) v[t] = 0.0;
  for (int bk = 0; bk < (int)gridDim.x; ++bk)
    for (int t = 0; t < NV; ++t) v[t] += part[(size_t)bk * 4 + t];
  grid.sync();   // partials may be overwritten by the next reduction
}

template <typename Real>
__global__ void __launch_bounds__(kPcgThreads) k_pcg(PcgArgs a) {
  cg::grid_group grid = cg::this_grid();
  const size_t n = a.n;
  const size_t gtid = blockIdx.x * (size_t)blockDim.x + threadIdx.x, gstride = (size_t)gridDim.x * blockDim.x;
  // x = 0, r = b, z = M^-1 r, p = z
  for (size_t t = gtid; t < n; t += gstride) { a.x[t] = 0.0; a.r[t] = a.b[t]; }
  grid.sync();
  precond_rows(a, a.r, a.z);
  grid.sync();
  double v[2] = {0.0, 0.0};
  for (size_t t = gtid; t < n; t += gstride) {
    a.p[t] = a.z[t];
    v[0] += a.r[t] * a.z[t];
    v[1] += a.b[t] * a.b[t];
  }
  grid_sums<2>(v, a.part, grid);
  double rz = v[0];
  const double bnorm = sqrt(v[1]);
  int it = 0;
  if (bnorm > 0.0) {
    for (it = 0; it < a.max_iter; ++it) {
      matvec_rows<Real>(a, a.p, a.Ap);
      grid.sync();
      double w[1] = {0.0};
      for (size_t t = gtid; t < n; t += gstride) w[0] += a.p[t] * a.Ap[t];
      grid_sums<1>(w, a.part, grid);
      const double pAp = w[0];
      if (!(pAp > 0.0)) {
        if (gtid == 0) *a.fail = 1;
        break;
      }
      const double alpha = rz / pAp;
      for (size_t t = gtid; t < n; t += gstride) {
        a.x[t] += alpha * a.p[t];
        a.r[t] -= alpha * a.Ap[t];
      }
      grid.sync();
      precond_rows(a, a.r, a.z);
      grid.sync();
      double u[2] = {0.0, 0.0};
      for (size_t t = gtid; t < n; t += gstride) {
        u[0] += a.r[t] * a.z[t];
        u[1] += a.r[t] * a.r[t];
      }
      grid_sums<2>(u, a.part, grid);
      if (sqrt(u[1]) <= a.tol * bnorm) { ++it; break; }
      const double beta = u[0] / rz;
      rz = u[0];
      for (size_t t = gtid; t < n; t += gstride) a.p[t] = a.z[t] + beta * a.p[t];
      grid.sync();
    }
  }
  if (gtid == 0) *a.iters_out = it;
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
  std::vector<int> rp(1, 0), rb, rc;
  std::vector<unsigned char> rt;
  for (int i = 0; i < N; ++i) {
    std::sort(rows[i].begin(), rows[i].end());
    for (auto& e : rows[i]) {
      rc.push_back(e.first);
      rb.push_back(e.second / 2);
      rt.push_back((unsigned char)(e.second & 1));
    }
    rp.push_back((int)rc.size());
    if (diag[i] < 0) return V3DBA_ERR_INVALID_INPUT;
  }
  auto up = [](auto** d, const auto& h) -> int {
    using T = typename std::remove_reference<decltype(h)>::type::value_type;
    V3DBA_CUDA_TRY(cudaMalloc(d, sizeof(T) * std::max<size_t>(h.size(), 1)));
    if (!h.empty()) V3DBA_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
    return V3DBA_OK;
  };
  int rc2;
  if ((rc2 = up(&ps.rp, rp)) || (rc2 = up(&ps.rb, rb)) || (rc2 = up(&ps.rc, rc)) || (rc2 = up(&ps.rt, rt)) ||
      (rc2 = up(&ps.diag_blk, diag)))
    return rc2;
  return V3DBA_OK;
}

int pcg_alloc(PcgState& ps, int nb, int N, int DA) {
  const size_t n = (size_t)N * DA;
  V3DBA_CUDA_TRY(cudaMalloc(&ps.Sb, sizeof(double) * (size_t)std::max(nb, 1) * DA * DA));
  V3DBA_CUDA_TRY(cudaMalloc(&ps.Pinv, sizeof(double) * (size_t)std::max(N, 1) * DA * DA));
  V3DBA_CUDA_TRY(cudaMalloc(&ps.vec, sizeof(double) * 6 * std::max<size_t>(n, 1)));
  V3DBA_CUDA_TRY(cudaMalloc(&ps.part, sizeof(double) * 4 * 4096));
  V3DBA_CUDA_TRY(cudaMalloc(&ps.iters, sizeof(int)));
  ps.b = ps.vec;
  ps.ready = true;
  return V3DBA_OK;
}

void pcg_free(PcgState& ps) {
  cudaFree(ps.rp); cudaFree(ps.rb); cudaFree(ps.rc); cudaFree(ps.rt); cudaFree(ps.diag_blk);
  cudaFree(ps.Sb); cudaFree(ps.Pinv); cudaFree(ps.vec); cudaFree(ps.part); cudaFree(ps.iters);
  ps = PcgState();
}

int pcg_solve(PcgState& ps, int N, int DA, bool fp64, double tol, int max_iter, double* x, int* d_fail,
              cudaStream_t st) {
  const size_t n = (size_t)N * DA;
  if (fp64) k_pcg_precond<double><<<(N + 127) / 128, 128, 0, st>>>(ps.Sb, ps.diag_blk, N, DA, ps.Pinv, d_fail);
  else k_pcg_precond<float><<<(N + 127) / 128, 128, 0, st>>>(ps.Sb, ps.diag_blk, N, DA, ps.Pinv, d_fail);
  V3DBA_LAUNCH_CHECK();
  PcgArgs a;
  a.N = N; a.DA = DA; a.n = (int)n;
  a.rp = ps.rp; a.rb = ps.rb; a.rc = ps.rc; a.rt = ps.rt; a.Sb = ps.Sb; a.fp64 = fp64 ? 1 : 0;
  a.Pinv = ps.Pinv; a.b = ps.b; a.x = x;
  a.r = ps.vec + n; a.z = ps.vec + 2 * n; a.p = ps.vec + 3 * n; a.Ap = ps.vec + 4 * n;
  a.part = ps.part; a.tol = tol; a.max_iter = max_iter; a.iters_out = ps.iters; a.fail = d_fail;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  void* fn = fp64 ? (void*)k_pcg<double> : (void*)k_pcg<float>;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kPcgThreads, 0);
  const int grid = std::max(1, std::min(sms * std::max(per_sm, 1), 4096));
  void* args[] = {&a};
  V3DBA_CUDA_TRY(cudaLaunchCooperativeKernel(fn, grid, kPcgThreads, args, 0, st));
  note_launches(1);
  return V3DBA_OK;
}

}  // namespace v3dba
