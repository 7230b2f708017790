// Tile-sparse dense FP64 Cholesky of the reduced camera system.
//
// Replaces the reference's block-SYMAMD ordering + sparse LDL^T of the full damped normal
// matrix (V3D/src/Math/v3d_optimization.cpp:111-176 numeric factor, :1096-1145 call site,
// :54-98 symbolic).  After the points are eliminated the system is small (n = 6N + dC) and is
// stored dense, column-major, in 64x64 tiles; tiles that are structurally zero in L (found by a
// tile-level symbolic factorisation on the host) are never touched.
//
// Storage: S has n_pad + 64 rows and n_pad columns (ld = n_pad + 64).  Tile row nt holds the
// right-hand side as its first row, so the right-looking factorisation performs the forward
// substitution L y = b on the fly (the rhs row is factored like any other tile row).
//
// Per tile column k:
//   k_chol_panel  : every block factors the diagonal tile in shared memory (block 0 also forms
//                   its triangular inverse for the back-substitution); blocks 1.. solve
//                   X L_kk^T = A_rk for one panel tile each (TRSM).
//   k_chol_update : one block per trailing tile (r, c): A_rc -= L_rk L_ck^T on the FP64 tensor
//                   pipe (DMMA mma.sync m8n8k4 f64).
// Then k_chol_backsolve solves L^T x = y with one block.  A non-positive pivot sets *fail (the
// LM step then fails and lambda is raised, as the reference does on a zero LDL pivot).
#include <algorithm>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "lm.cuh"

namespace v3dba {

constexpr int TB = 64;
constexpr int LDF = 65;   // shared leading dimension of the factor / TRSM tiles
constexpr int LDM = 68;   // shared leading dimension of the DMMA operand tiles

// Right-looking Cholesky of the 64x64 tile in shared memory (column-major, leading dimension
// LDF, lower triangle).  One barrier per column: the trailing update uses the unscaled pivot
// column (A_rc -= A_rj A_cj / A_jj); the columns are scaled at the end.  Returns false on a
// non-positive (or NaN) pivot.
__device__ bool tile_potrf(double* A) {
  const int tid = threadIdx.x;
  const int r = tid & 63, grp = tid >> 6;  // 4 column groups
  bool ok = true;
  for (int j = 0; j < TB; ++j) {
    const double d = A[j * LDF + j];
    if (!(d > 0.0)) ok = false;
    const double inv = (d > 0.0) ? 1.0 / d : 0.0;
    if (r > j) {
      const double arj = A[j * LDF + r] * inv;
      for (int c = j + 1 + grp; c <= r; c += 4) A[c * LDF + r] -= arj * A[j * LDF + c];
    }
    __syncthreads();
  }
  // scale: L_rj = A_rj / sqrt(A_jj); the square roots are taken first so that no thread reads
  // a diagonal entry another thread has already replaced
  __shared__ double dsq[TB];
  if (tid < TB) {
    const double d = A[tid * LDF + tid];
    dsq[tid] = d > 0.0 ? sqrt(d) : 1.0;
  }
  __syncthreads();
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int c = e >> 6, rr = e & 63;
    if (rr > c) A[c * LDF + rr] /= dsq[c];
    else if (rr == c) A[c * LDF + rr] = dsq[c];
  }
  __syncthreads();
  return ok;
}

// X L^T = W for the 64x64 tile W (shared, LDF) given L (shared, LDF, lower).  X overwrites W.
__device__ void tile_trsm(const double* L, double* W) {
  const int tid = threadIdx.x;
  const int m = tid & 63, grp = tid >> 6;
  for (int c = 0; c < TB; ++c) {
    const double xmc = W[c * LDF + m] / L[c * LDF + c];
    for (int c2 = c + 1 + grp; c2 < TB; c2 += 4) W[c2 * LDF + m] -= xmc * L[c * LDF + c2];
    __syncthreads();
    if (grp == 0) W[c * LDF + m] = xmc;
    __syncthreads();
  }
}

// Z = L^-1 (lower) for the 64x64 tile L in shared memory; four threads per column of Z.
__device__ void tile_trinv(const double* L, double* Z) {
  const int tid = threadIdx.x;
  const int c = tid >> 2, part = tid & 3;
  // zero the upper part
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int cc = e >> 6, rr = e & 63;
    if (rr < cc) Z[cc * LDF + rr] = 0.0;
  }
  __syncthreads();
  // every lane runs the same trip count so the quad shuffles stay convergent (c < 64 always)
  if (part == 0) Z[c * LDF + c] = 1.0 / L[c * LDF + c];
  __syncwarp();
  for (int rr = 1; rr < TB; ++rr) {
    double s = 0.0;
    if (rr > c)
      for (int t = c + part; t < rr; t += 4) s += L[t * LDF + rr] * Z[c * LDF + t];
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (rr > c && part == 0) Z[c * LDF + rr] = -s / L[rr * LDF + rr];
    __syncwarp();
  }
  __syncthreads();
}

__global__ void __launch_bounds__(256) k_chol_panel(double* __restrict__ S, int ld, int k,
                                                    const int* __restrict__ rows, int nrows,
                                                    double* __restrict__ ldiag, int* __restrict__ fail) {
  extern __shared__ double sm[];
  double* D = sm;             // diagonal tile -> L_kk
  double* W = sm + TB * LDF;  // panel tile / inverse
  const int tid = threadIdx.x;
  const size_t col0 = (size_t)k * TB;
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int c = e >> 6, r = e & 63;
    D[c * LDF + r] = S[(col0 + c) * ld + col0 + r];
  }
  __syncthreads();
  const bool ok = tile_potrf(D);
  if (blockIdx.x == 0) {
    if (!ok && tid == 0) atomicExch(fail, 1);
    tile_trinv(D, W);
    double* out = ldiag + (size_t)k * TB * TB;
    for (int e = tid; e < TB * TB; e += blockDim.x) {
      const int c = e >> 6, r = e & 63;
      out[c * TB + r] = W[c * LDF + r];
    }
    return;
  }
  const int r0 = rows[blockIdx.x - 1] * TB;
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int c = e >> 6, m = e & 63;
    W[c * LDF + m] = S[(col0 + c) * ld + r0 + m];
  }
  __syncthreads();
  tile_trsm(D, W);
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int c = e >> 6, m = e & 63;
    S[(col0 + c) * ld + r0 + m] = W[c * LDF + m];
  }
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// A_rc -= L_rk L_ck^T for one trailing tile per block (8 warps, each owns 8 rows x 64 columns).
__global__ void __launch_bounds__(256) k_chol_update(double* __restrict__ S, int ld, int k,
                                                     const int* __restrict__ ur, const int* __restrict__ uc) {
  extern __shared__ double sm[];
  double* As = sm;
  double* Bs = sm + TB * LDM;
  const int tid = threadIdx.x;
  const size_t r0 = (size_t)ur[blockIdx.x] * TB, c0 = (size_t)uc[blockIdx.x] * TB, k0 = (size_t)k * TB;
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int t = e >> 6, m = e & 63;
    As[t * LDM + m] = S[(k0 + t) * ld + r0 + m];
    Bs[t * LDM + m] = S[(k0 + t) * ld + c0 + m];
  }
  __syncthreads();
  const int lane = tid & 31, w = tid >> 5;
  const int g = lane >> 2, q = lane & 3;
  double acc[8][2];
#pragma unroll
  for (int nb = 0; nb < 8; ++nb) acc[nb][0] = acc[nb][1] = 0.0;
#pragma unroll 4
  for (int s = 0; s < TB / 4; ++s) {
    const double a = As[(4 * s + q) * LDM + 8 * w + g];
#pragma unroll
    for (int nb = 0; nb < 8; ++nb) {
      const double b = Bs[(4 * s + q) * LDM + 8 * nb + g];
      dmma(acc[nb][0], acc[nb][1], a, b);
    }
  }
  const size_t row = r0 + 8 * w + g;
#pragma unroll
  for (int nb = 0; nb < 8; ++nb)
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const size_t col = c0 + 8 * nb + 2 * q + i;
      S[col * ld + row] -= acc[nb][i];
    }
}

// L^T x = y with one block; y is row n_pad of S, L_kk^-1 tiles in ldiag.
__global__ void __launch_bounds__(256) k_chol_backsolve(const double* __restrict__ S, int ld, int nt, int n_pad,
                                                        const int* __restrict__ pptr, const int* __restrict__ prows,
                                                        const double* __restrict__ ldiag, double* __restrict__ x) {
  __shared__ double red[4][TB];
  __shared__ double v[TB];
  const int tid = threadIdx.x;
  const int col = tid & 63, part = tid >> 6;
  for (int k = nt - 1; k >= 0; --k) {
    const size_t kc = (size_t)k * TB + col;
    double s = 0.0;
    for (int p = pptr[k]; p < pptr[k + 1]; ++p) {
      const int r = prows[p];
      if (r >= nt) continue;
      const double* Lcol = S + kc * ld + (size_t)r * TB;
      const double* xr = x + (size_t)r * TB;
#pragma unroll 4
      for (int m = part * 16; m < part * 16 + 16; ++m) s += Lcol[m] * xr[m];
    }
    red[part][col] = s;
    __syncthreads();
    if (tid < TB) v[tid] = S[kc * ld + n_pad] - (red[0][tid] + red[1][tid] + red[2][tid] + red[3][tid]);
    __syncthreads();
    // x_k = Linv^T v : x[col] = sum_{m >= col} Linv[m][col] v[m]
    const double* Z = ldiag + (size_t)k * TB * TB + (size_t)col * TB;
    double t = 0.0;
#pragma unroll 4
    for (int m = part * 16; m < part * 16 + 16; ++m) t += (m >= col) ? Z[m] * v[m] : 0.0;
    red[part][col] = t;
    __syncthreads();
    if (tid < TB) x[(size_t)k * TB + tid] = red[0][tid] + red[1][tid] + red[2][tid] + red[3][tid];
    __syncthreads();
  }
}

// Clears the pattern tiles of S (padding diagonal 1).  With d_lambda set, block 0 also starts the
// trial: the damping and a cleared failure flag (the work of the trial-setup kernel, one launch
// less per trial).
__global__ void __launch_bounds__(256) k_chol_zero(double* __restrict__ S, int ld, int nt, int n, int n_pad,
                                                   const int* __restrict__ tiles, double lambda,
                                                   double* __restrict__ d_lambda, int* __restrict__ d_fail) {
  pdl_wait();
  pdl_trigger();
  if (d_lambda && blockIdx.x == 0 && threadIdx.x == 0) {
    *d_lambda = lambda;
    *d_fail = 0;
  }
  const int t = tiles[blockIdx.x];
  const int tr = t / (nt + 1) , tc = t % (nt + 1);
  const size_t r0 = (size_t)tr * TB, c0 = (size_t)tc * TB;
  for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
    const int c = e >> 6, r = e & 63;
    const size_t gr = r0 + r, gc = c0 + c;
    S[gc * ld + gr] = (gr == gc && gr >= (size_t)n && gr < (size_t)n_pad) ? 1.0 : 0.0;
  }
}

// ---- host ----------------------------------------------------------------------------------

int tile_chol_plan(TileChol& tc, int n, std::vector<uint8_t>& nz) {
  tile_chol_free(tc);   // a plan retried after a failed one (out of memory) starts clean
  const int nt = (n + TB - 1) / TB;
  tc.n = n;
  tc.nt = nt;
  tc.n_pad = nt * TB;
  tc.ld = tc.n_pad + TB;
  if ((int)nz.size() != nt * nt) return V3DBA_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < nt; ++k) nz[k * nt + k] = 1;
  const std::vector<uint8_t> orig = nz;
  // tile-level symbolic factorisation (fill-in)
  std::vector<int> rows;
  for (int k = 0; k < nt; ++k) {
    rows.clear();
    for (int r = k + 1; r < nt; ++r)
      if (nz[r * nt + k]) rows.push_back(r);
    for (size_t a = 0; a < rows.size(); ++a)
      for (size_t b = 0; b <= a; ++b) nz[rows[a] * nt + rows[b]] = 1;
  }
  tc.h_panel_ptr.assign(1, 0);
  tc.h_panel_rows.clear();
  tc.h_upd_ptr.assign(1, 0);
  tc.h_upd_r.clear();
  tc.h_upd_c.clear();
  tc.h_tiles.clear();
  for (int k = 0; k < nt; ++k) {
    rows.clear();
    for (int r = k + 1; r < nt; ++r)
      if (nz[r * nt + k]) rows.push_back(r);
    rows.push_back(nt);  // the rhs row
    for (int r : rows) tc.h_panel_rows.push_back(r);
    tc.h_panel_ptr.push_back((int)tc.h_panel_rows.size());
    for (size_t a = 0; a < rows.size(); ++a)
      for (size_t b = 0; b <= a; ++b) {
        if (rows[a] == nt && rows[b] == nt) continue;
        tc.h_upd_r.push_back(rows[a]);
        tc.h_upd_c.push_back(rows[b]);
      }
    tc.h_upd_ptr.push_back((int)tc.h_upd_r.size());
  }
  for (int r = 0; r <= nt; ++r)
    for (int c = 0; c < nt && c <= r; ++c)
      if (r == nt || nz[r * nt + c]) tc.h_tiles.push_back(r * (nt + 1) + c);

  auto up = [](int** d, const std::vector<int>& h) -> int {
    if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
    V3DBA_CUDA_TRY(cudaMalloc(d, sizeof(int) * std::max<size_t>(h.size(), 1)));
    if (!h.empty()) V3DBA_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
    return V3DBA_OK;
  };
  int rc;
  if ((rc = up(&tc.d_panel_rows, tc.h_panel_rows))) return rc;
  if ((rc = up(&tc.d_panel_ptr, tc.h_panel_ptr))) return rc;
  if ((rc = up(&tc.d_upd_r, tc.h_upd_r))) return rc;
  if ((rc = up(&tc.d_upd_c, tc.h_upd_c))) return rc;
  if ((rc = up(&tc.d_upd_ptr, tc.h_upd_ptr))) return rc;
  if ((rc = up(&tc.d_tiles, tc.h_tiles))) return rc;
  if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
  V3DBA_CUDA_TRY(cudaMalloc(&tc.d_ldiag, sizeof(double) * (size_t)nt * TB * TB));
  if ((rc = tile_levels_plan(tc, orig))) return rc;
  static bool attr_set = false;
  if (!attr_set) {
    V3DBA_CUDA_TRY(cudaFuncSetAttribute(k_chol_panel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * TB * LDF * sizeof(double))));
    V3DBA_CUDA_TRY(cudaFuncSetAttribute(k_chol_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)(2 * TB * LDM * sizeof(double))));
    attr_set = true;
  }
  return V3DBA_OK;
}

void tile_chol_free(TileChol& tc) {
  cudaFree(tc.d_panel_rows);
  cudaFree(tc.d_panel_ptr);
  cudaFree(tc.d_upd_r);
  cudaFree(tc.d_upd_c);
  cudaFree(tc.d_upd_ptr);
  cudaFree(tc.d_tiles);
  cudaFree(tc.d_ldiag);
  cudaFree(tc.d_lv);
  tc = TileChol();
}

int tile_chol_zero(const TileChol& tc, double* S, double* /*rhs*/, cudaStream_t st) {
  if (tc.h_tiles.empty()) return V3DBA_OK;
  V3DBA_CUDA_TRY(launch_pdl(k_chol_zero, dim3((unsigned)tc.h_tiles.size()), dim3(256), 0, st, S, tc.ld, tc.nt, tc.n,
                            tc.n_pad, (const int*)tc.d_tiles, 0.0, (double*)nullptr, (int*)nullptr));
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

int tile_chol_zero_setup(const TileChol& tc, double* S, double lambda, double* d_lambda, int* d_fail,
                         cudaStream_t st) {
  if (tc.h_tiles.empty()) return V3DBA_ERR_INVALID_ARGUMENT;
  V3DBA_CUDA_TRY(launch_pdl(k_chol_zero, dim3((unsigned)tc.h_tiles.size()), dim3(256), 0, st, S, tc.ld, tc.nt, tc.n,
                            tc.n_pad, (const int*)tc.d_tiles, lambda, d_lambda, d_fail));
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

int tile_chol_solve(const TileChol& tc, double* S, double* x, int* d_fail, cudaStream_t st) {
  if (tc.levels) return chol_levels_solve(tc, S, x, d_fail, st);
  return chol_cluster_solve(tc, S, x, d_fail, st);
}

int tile_chol_solve_multilaunch(const TileChol& tc, double* S, double* x, int* d_fail, cudaStream_t st) {
  const size_t smp = 2 * TB * LDF * sizeof(double), smu = 2 * TB * LDM * sizeof(double);
  for (int k = 0; k < tc.nt; ++k) {
    const int p0 = tc.h_panel_ptr[k], np = tc.h_panel_ptr[k + 1] - p0;
    k_chol_panel<<<1 + np, 256, smp, st>>>(S, tc.ld, k, tc.d_panel_rows + p0, np, tc.d_ldiag, d_fail);
    V3DBA_LAUNCH_CHECK();
    const int u0 = tc.h_upd_ptr[k], nu = tc.h_upd_ptr[k + 1] - u0;
    if (nu > 0) {
      k_chol_update<<<nu, 256, smu, st>>>(S, tc.ld, k, tc.d_upd_r + u0, tc.d_upd_c + u0);
      V3DBA_LAUNCH_CHECK();
    }
  }
  k_chol_backsolve<<<1, 256, 0, st>>>(S, tc.ld, tc.nt, tc.n_pad, tc.d_panel_ptr, tc.d_panel_rows, tc.d_ldiag, x);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

}  // namespace v3dba
