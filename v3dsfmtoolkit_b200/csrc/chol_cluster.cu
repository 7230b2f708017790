// One-launch tile Cholesky of the reduced camera system on a thread-block cluster.
//
// Same factorisation as tile_cholesky.cu (right-looking over 64x64 tiles, rhs carried as tile row
// nt, tiles that are structurally zero in L skipped), but the whole factor + solve runs in ONE
// launch of a cluster: the phases are separated by cluster barriers (barrier.cluster,
// sub-microsecond) instead of kernel boundaries, which removes the launch and drain latency that
// dominates small reduced systems (hundreds to a few thousand unknowns).  Two kernels:
//   k_chol_cluster (8 CTAs) goes column by column in the caller's order;
//   k_chol_levels (16 CTAs where the device allows, else 8) runs the level schedule of
//   chol_order.cu, the independent columns of an elimination-tree level side by side.
// Both use the same diagonal tile factor (cta_factor_tile8).
//
// k_chol_cluster: per tile column k, CTA 0 owns the chain along the diagonal and keeps it in
// shared memory:
//   with Z_k = L_kk^-1 resident it forms the panel tile next to the diagonal,
//   L_{k+1,k} = A_{k+1,k} Z_k^T, publishes it (split cluster barrier: arrive, keep working), applies
//   it to the next diagonal tile (fetched meanwhile) and factors that tile: 8-column blocking,
//   each 8x8 diagonal block factored and inverted by one warp in registers, panels and trailing
//   blocks updated with FP64 tensor-core MMAs (DMMA m8n8k4), Z_{k+1} assembled;
//   CTAs 1.. form the other panel tiles (and the rhs row), L_rk = A_rk Z_k^T, one 64x64x64 DMMA
//   GEMM per tile, then the other trailing tiles, A_rc -= L_rk L_ck^T (DMMA).
// Then the back-substitution L^T x = y (y = the factored rhs row) by CTA 0, with x kept in
// shared memory and Z_kk fetched ahead of the dependent sums.  (Its CTAs are kCluster = 8.)
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "lm.cuh"

namespace cg = cooperative_groups;

namespace v3dba {

namespace {

constexpr int TB = 64;
constexpr int LDT = 68;          // shared leading dimension (bank-conflict free DMMA fragments)
constexpr int kCluster = 8;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// acc(16x16 block of one warp) += sum_t A(m,t) B(t,n), t in [0,K):
//   A(m,t) = A[m*ars + t*acs], B(t,n) = B[t*bks + n*bns].
// Fragment ownership: acc[a][b][i] is element (8a + g, 8b + 2q + i), g = lane/4, q = lane%4.
__device__ __forceinline__ void warp_mma16(double (&acc)[2][2][2], const double* A, int ars, int acs,
                                           const double* B, int bks, int bns, int K) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  for (int s = 0; s < K / 4; ++s) {
    const int t = 4 * s + q;
    const double a0 = A[(g)*ars + t * acs], a1 = A[(8 + g) * ars + t * acs];
    const double b0 = B[t * bks + (g)*bns], b1 = B[t * bks + (8 + g) * bns];
    dmma(acc[0][0][0], acc[0][0][1], a0, b0);
    dmma(acc[0][1][0], acc[0][1][1], a0, b1);
    dmma(acc[1][0][0], acc[1][0][1], a1, b0);
    dmma(acc[1][1][0], acc[1][1][1], a1, b1);
  }
}

__device__ __forceinline__ void acc_zero(double (&acc)[2][2][2]) {
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
}

// 1/sqrt(x) for a positive pivot: the hardware approximation y (rsqrt.approx.ftz.f64, one
// instruction) refined by one step of Householder's third-order iteration for x^(-1/2),
// y <- y (1 + e/2 + 3 e^2 / 8) with e = 1 - x y^2 (the first three terms of the binomial series of
// (1 - e)^(-1/2)), which roughly triples the number of correct bits.  A chain of four dependent
// FP64 operations instead of the six of two Newton-Raphson steps; the whole 64x64 tile factor
// takes ~4 % fewer cycles.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x, y * y, 1.0);
  const double p = fma(0.375, e, 0.5);
  return fma(y * e, p, y);
}

// ---- 8-column blocking -----------------------------------------------------------------------

// acc(8x8 block of one warp) += sum_t A(m,t) B(t,n), t in [0,K), A(m,t) = A[m*ars + t*acs],
// B(t,n) = B[t*bks + n*bns]; acc[i] is element (g, 2q + i), g = lane/4, q = lane%4.
__device__ __forceinline__ void warp_mma8(double (&acc)[2], const double* A, int ars, int acs, const double* B,
                                          int bks, int bns, int K) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  for (int s = 0; s < K / 4; ++s) {
    const int t = 4 * s + q;
    dmma(acc[0], acc[1], A[g * ars + t * acs], B[t * bks + g * bns]);
  }
}

// C(8x8 at C, col-major ldc) = alpha * acc + beta * C
__device__ __forceinline__ void acc_store8(const double (&acc)[2], double* C, int ldc, double alpha, double beta) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    double* p = C + (2 * q + i) * ldc + g;
    *p = alpha * acc[i] + (beta != 0.0 ? beta * *p : 0.0);
  }
}

// Packed position of element (r, c), r >= c, of an 8x8 lower triangle stored column by column.
__host__ __device__ constexpr int pk8(int r, int c) { return c * 8 - (c * (c - 1)) / 2 + (r - c); }

// One warp: Z = L^-1 for the Cholesky factor L of the 8x8 SPD block D (lower triangle read,
// col-major LDT), written to the lower triangle of Zd (the caller zeroes its upper part).  Every
// lane computes the whole factor and inverse in registers from the same broadcast reads: no
// shuffles and no lane waits for another, so the chain from one pivot to the next is one
// reciprocal square root and two dependent FMAs.  Returns false on a non-positive pivot.
__device__ __noinline__ bool warp_chol_inv8(const double* D, double* Zd) {
  double a[36];
#pragma unroll
  for (int c = 0; c < 8; ++c)
#pragma unroll
    for (int r = c; r < 8; ++r) a[pk8(r, c)] = D[c * LDT + r];
  bool ok = true;
  double s[8];
  // right-looking Cholesky, L over a
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const double d = a[pk8(j, j)];
    if (!(d > 0.0)) ok = false;
    const double sj = rsqrt_nr(d > 0.0 ? d : 1.0);
    s[j] = sj;
#pragma unroll
    for (int r = j + 1; r < 8; ++r) a[pk8(r, j)] *= sj;
#pragma unroll
    for (int c = j + 1; c < 8; ++c)
#pragma unroll
      for (int r = c; r < 8; ++r) a[pk8(r, c)] = fma(-a[pk8(r, j)], a[pk8(c, j)], a[pk8(r, c)]);
  }
  // Z = L^-1: Z_cc = 1 / L_cc = s_c, Z_rc = -s_r sum_{t=c}^{r-1} L_rt Z_tc
  double z[36];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    z[pk8(c, c)] = s[c];
#pragma unroll
    for (int r = c + 1; r < 8; ++r) {
      double acc = 0.0;
#pragma unroll
      for (int t = c; t < r; ++t) acc = fma(a[pk8(r, t)], z[pk8(t, c)], acc);
      z[pk8(r, c)] = -acc * s[r];
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int c = 0; c < 8; ++c)
#pragma unroll
      for (int r = c; r < 8; ++r) Zd[c * LDT + r] = z[pk8(r, c)];
  }
  __syncwarp();
  return ok;
}

// CTA (256 threads): Z = L^-1 (full 64x64, zero upper part) into Zs for the Cholesky factor L of
// the 64x64 tile A (shared, col-major LDT, lower triangle valid; A is overwritten).  Blocked by
// 8 columns with lookahead: warp 0 carries the chain of diagonal blocks (the update of the next
// diagonal block by the panel just formed, then its inverse factor, warp_chol_inv8) while warps
// 1..3 and 5..7 apply the other trailing updates (A_ij -= L_ip L_jp^T) and form block row p of Z
// (Z_pj = -Z_pp sum_{t=j}^{p-1} L_pt Z_tj); the panel blocks L_ip = A_ip Z_pp^T are formed by the
// first warps between.  All products are 8x8 DMMA blocks.  Returns false on a non-positive pivot.
__device__ bool cta_factor_tile8(double* A, double* Zs) {
  const int tid = threadIdx.x, w = tid >> 5;
  __shared__ int s_ok8;
  if (tid == 0) s_ok8 = 1;
  // the upper part of Z: column c is zeroed from row 0 to the end of its diagonal block with
  // 16-byte stores (the lower entries of the diagonal block are written by its factor later)
  for (int c = tid >> 2; c < TB; c += blockDim.x >> 2) {
    double2* col = reinterpret_cast<double2*>(Zs + c * LDT);
    for (int r2 = tid & 3; r2 < 4 * (c >> 3) + 4; r2 += 4) col[r2] = make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (w == 0 && !warp_chol_inv8(A, Zs) && (tid & 31) == 0) s_ok8 = 0;
  __syncthreads();
  for (int p = 0; p < 8; ++p) {
    const double* Zpp = Zs + 8 * p * LDT + 8 * p;
    if (p < 7) {
      if (w < 7 - p) {   // panel blocks L_ip = A_ip Z_pp^T
        const int i = p + 1 + w;
        double acc[2] = {0.0, 0.0};
        warp_mma8(acc, A + 8 * p * LDT + 8 * i, 1, LDT, Zpp, LDT, 1, 8);
        __syncwarp();
        acc_store8(acc, A + 8 * p * LDT + 8 * i, LDT, 1.0, 0.0);
      }
      __syncthreads();
    }
    if (w == 0) {
      if (p < 7) {   // the next diagonal block: A_qq -= L_qp L_qp^T, then its inverse factor
        const int q1 = p + 1;
        double acc[2] = {0.0, 0.0};
        warp_mma8(acc, A + 8 * p * LDT + 8 * q1, 1, LDT, A + 8 * p * LDT + 8 * q1, LDT, 1, 8);
        acc_store8(acc, A + 8 * q1 * LDT + 8 * q1, LDT, -1.0, 1.0);
        __syncwarp();
        if (!warp_chol_inv8(A + 8 * q1 * LDT + 8 * q1, Zs + 8 * q1 * LDT + 8 * q1) && (tid & 31) == 0) s_ok8 = 0;
      }
    } else if (w != 4) {
      // Tasks of this iteration, dealt in turn to warps 1..7 except 4 (which shares warp 0's
      // scheduler partition: kept free of DMMA work, the pivot chain runs ~15 % faster): first
      // the trailing blocks (i, j), p+1 <= j <= i < 8, other than (p+1, p+1) (the lower triangle
      // of the trailing block matrix numbered row by row: u -> (ii, jj), ii(ii+1)/2 <= u <
      // (ii+1)(ii+2)/2), then block row p of Z.  Each warp steps straight to its own tasks.
      constexpr int NW = 6;
      const int slot = w < 4 ? w - 1 : w - 2;
      const int m = 7 - p;
      const int n_upd = m * (m + 1) / 2 - 1;
      for (int k = slot; k < n_upd; k += NW) {
        const int u = k + 1;
        int ii = 0;
        while ((ii + 1) * (ii + 2) / 2 <= u) ++ii;
        const int i = p + 1 + ii, j = p + 1 + (u - ii * (ii + 1) / 2);
        double acc[2] = {0.0, 0.0};
        warp_mma8(acc, A + 8 * p * LDT + 8 * i, 1, LDT, A + 8 * p * LDT + 8 * j, LDT, 1, 8);
        acc_store8(acc, A + 8 * j * LDT + 8 * i, LDT, -1.0, 1.0);
      }
      for (int j = ((slot - n_upd) % NW + NW) % NW; j < p; j += NW) {
        double acc[2] = {0.0, 0.0};
        for (int t = j; t < p; ++t)
          warp_mma8(acc, A + 8 * t * LDT + 8 * p, 1, LDT, Zs + 8 * j * LDT + 8 * t, 1, LDT, 8);
        double* Wpj = Zs + 8 * j * LDT + 8 * p;   // the block itself holds W = sum L Z meanwhile
        acc_store8(acc, Wpj, LDT, 1.0, 0.0);
        __syncwarp();
        double acc2[2] = {0.0, 0.0};
        warp_mma8(acc2, Zpp, 1, LDT, Wpj, 1, LDT, 8);
        __syncwarp();
        acc_store8(acc2, Wpj, LDT, -1.0, 0.0);
      }
    }
    __syncthreads();
  }
  return s_ok8 != 0;
}

// CTA: C(64x64) = A B^T for shared tiles A, B (col-major LDT); the result stays in the warps'
// fragments: warp w owns the 16x16 blocks (bi, bj) = (w>>1, 2*(w&1) + {0,1}).
__device__ __forceinline__ void cta_gemm_abt(double (&acc)[2][2][2][2], const double* A, const double* B) {
  const int w = threadIdx.x >> 5;
  const int bi = w >> 1;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int bj = 2 * (w & 1) + h;
    acc_zero(acc[h]);
    // A(m,t) = A[t*LDT + 16 bi + m]; B(t,n) = B(n,t) = B[t*LDT + 16 bj + n]
    warp_mma16(acc[h], A + 16 * bi, 1, LDT, B + 16 * bj, LDT, 1, TB);
  }
}

// CTA: acc += A B^T for shared tiles A, B (col-major LDT), with the same fragment ownership as
// cta_gemm_abt; A is read transposed (A(m,t) = A[m*LDT + t]) when a_t.
__device__ __forceinline__ void cta_gemm_abt_acc(double (&acc)[2][2][2][2], const double* A, bool a_t,
                                                 const double* B) {
  const int w = threadIdx.x >> 5;
  const int bi = w >> 1;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int bj = 2 * (w & 1) + h;
    if (a_t) warp_mma16(acc[h], A + 16 * bi * LDT, LDT, 1, B + 16 * bj, LDT, 1, TB);
    else warp_mma16(acc[h], A + 16 * bi, 1, LDT, B + 16 * bj, LDT, 1, TB);
  }
}

// The lower triangle of a symmetric update: the 10 16x16 blocks (bi >= bj) of acc += A A^T, two
// per warp at most and 3 / 3 / 2 / 2 per scheduler partition (warp w runs on partition w % 4)
// instead of 4 each for the full tile.  kLowerBlk[w][h] = 4 bi + bj, or -1.  Each element is
// summed in the same order as by cta_gemm_abt_acc, so its lower triangle is the same bits.
__constant__ signed char kLowerBlk[8][2] = {{0, 4}, {8, 9}, {12, 13}, {14, 15}, {5, -1}, {10, -1}, {-1, -1}, {-1, -1}};
__device__ __forceinline__ void cta_gemm_aat_lower_acc(double (&acc)[2][2][2][2], const double* A) {
  const int w = threadIdx.x >> 5;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int b = kLowerBlk[w][h];
    if (b < 0) continue;
    const int bi = b >> 2, bj = b & 3;
    warp_mma16(acc[h], A + 16 * bi, 1, LDT, A + 16 * bj, LDT, 1, TB);
  }
}

// Panel product acc += A Z^T with Z = L_jj^-1 lower triangular (col-major LDT): Z^T is upper
// triangular, so output block column bj takes only the first 16 (bj + 1) terms of the inner
// dimension (the skipped k-steps are exact zeros: the same bits as the full product).  Warp w
// owns row block bi = w >> 1 and the block columns {3, 0} (even w) or {2, 1} (odd w), 5 units of
// k-steps each, so every scheduler partition carries 10 units instead of 16.
__device__ __forceinline__ int panel_bj(int w, int h) { return (w & 1) ? 2 - h : 3 * (1 - h); }
__device__ __forceinline__ void cta_gemm_azt_acc(double (&acc)[2][2][2][2], const double* A, bool a_t,
                                                 const double* Z) {
  const int w = threadIdx.x >> 5;
  const int bi = w >> 1;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int bj = panel_bj(w, h);
    const int K = 16 * (bj + 1);
    if (a_t) warp_mma16(acc[h], A + 16 * bi * LDT, LDT, 1, Z + 16 * bj, LDT, 1, K);
    else warp_mma16(acc[h], A + 16 * bi, 1, LDT, Z + 16 * bj, LDT, 1, K);
  }
}

// Tile copy global -> shared with cp.async (16-byte pieces, all in flight at once); the caller
// waits with tile_wait() and a barrier.
__device__ __forceinline__ void load_tile(double* dst, const double* __restrict__ S, size_t ld, size_t r0, size_t c0) {
  for (int e = threadIdx.x; e < TB * TB / 2; e += blockDim.x) {
    const int c = e >> 5, m2 = (e & 31) * 2;
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst + c * LDT + m2);
    const double* g = S + (c0 + c) * ld + r0 + m2;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g));
  }
  asm volatile("cp.async.commit_group;\n" ::);
}
__device__ __forceinline__ void tile_wait() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
// The copies of load_tile without the commit (several tiles in one group).
__device__ __forceinline__ void copy_tile(double* dst, const double* __restrict__ S, size_t ld, size_t r0, size_t c0) {
  for (int e = threadIdx.x; e < TB * TB / 2; e += blockDim.x) {
    const int c = e >> 5, m2 = (e & 31) * 2;
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst + c * LDT + m2);
    const double* g = S + (c0 + c) * ld + r0 + m2;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g));
  }
}
__device__ __forceinline__ void tile_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// Shared memory of k_chol_levels: six 64 x LDT tiles (two sets of input + two operands, so that
// the next phase-1 task's tiles load while the current one computes) and the rhs reduction.
constexpr size_t kLevelsSmem = (6 * TB * LDT + 4 * TB) * sizeof(double);

}  // namespace

// Split cluster barrier: arrive (release: this CTA's writes become visible to the cluster) and
// wait (acquire).  A CTA may do independent work between the two.
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }

__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(256)
    k_chol_cluster(double* __restrict__ S, int ld, int nt, int n_pad, const int* __restrict__ pptr,
                   const int* __restrict__ prows, const int* __restrict__ uptr, const int* __restrict__ ur,
                   const int* __restrict__ uc, double* __restrict__ ldiag, double* __restrict__ x,
                   int* __restrict__ fail, unsigned long long* __restrict__ trace) {
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  extern __shared__ double sm[];
  double* T0 = sm;
  double* T1 = sm + TB * LDT;
  double* T2 = sm + 2 * TB * LDT;   // rank 0 only: the next diagonal tile
  const size_t lds = (size_t)ld;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31, g = lane >> 2, q = lane & 3;

  // global tile at (r0, c0) = acc (op 0) or -= acc (op 1); optionally also into the shared tile
  // Csm (col-major LDT)
  auto store_acc = [&](const double (&acc)[2][2][2][2], size_t r0, size_t c0, int op, double* Csm) {
    const int bi = w >> 1;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int bj = 2 * (w & 1) + h;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int i = 0; i < 2; ++i) {
            const int col = 16 * bj + 8 * b + 2 * q + i, row = 16 * bi + 8 * a + g;
            double* gp = S + (c0 + col) * lds + r0 + row;
            if (op == 0) *gp = acc[h][a][b][i];
            else *gp -= acc[h][a][b][i];
            if (Csm) Csm[col * LDT + row] = acc[h][a][b][i];
          }
    }
  };
  // rank 0: factor the diagonal tile held in T2; Z = L^-1 into T1 (kept for the next panel) and to
  // global (for the other CTAs' panels and the back-substitution)
  auto factor_resident = [&](int k) {
    __syncthreads();
    const bool ok = cta_factor_tile8(T2, T1);
    if (!ok && tid == 0) atomicExch(fail, 1);
    double* Z = ldiag + (size_t)k * TB * TB;
    for (int e = tid; e < TB * TB; e += blockDim.x) Z[e] = T1[(e >> 6) * LDT + (e & 63)];
  };
  // A_rc -= L_rk L_ck^T for one trailing tile
  auto update_tile = [&](int k, int r, int c) {
    const size_t k0 = (size_t)k * TB, r0 = (size_t)r * TB, c0 = (size_t)c * TB;
    __syncthreads();
    load_tile(T0, S, lds, r0, k0);
    if (c0 != r0) load_tile(T1, S, lds, c0, k0);
    tile_wait();
    __syncthreads();
    double acc[2][2][2][2];
    cta_gemm_abt(acc, T0, c0 != r0 ? T1 : T0);
    store_acc(acc, r0, c0, 1, nullptr);
  };
  // optional phase timestamps (ns): trace[(2 k + phase) * kCluster + rank]
  auto stamp = [&](int slot) {
    if (trace != nullptr && tid == 0) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      trace[(size_t)slot * kCluster + rank] = t;
    }
  };
  if (rank == 0) {
    load_tile(T2, S, lds, 0, 0);
    tile_wait();
    factor_resident(0);
  }
  cl.sync();
  // Per tile step k: CTA 0 owns the chain along the diagonal (panel L_{k+1,k} with Z_k resident,
  // the update of the next diagonal tile in shared memory, its factor); CTAs 1.. form the other
  // panel tiles and apply the other trailing updates.  CTA 0 publishes L_{k+1,k} with a split
  // barrier and factors while the others work.
  for (int k = 0; k < nt; ++k) {
    const size_t k0 = (size_t)k * TB;
    const int p0 = pptr[k], np = pptr[k + 1] - p0;
    const bool has_next = k + 1 < nt;
    const bool diag_panel = has_next && np > 0 && prows[p0] == k + 1;   // rows are listed ascending
    stamp(2 * k);
    if (rank == 0) {
      if (has_next) {
        __syncthreads();
        load_tile(T2, S, lds, k0 + TB, k0 + TB);   // the next diagonal tile, fetched meanwhile
        if (diag_panel) {
          load_tile(T0, S, lds, k0 + TB, k0);
          tile_wait();
          __syncthreads();
          double acc[2][2][2][2];
          cta_gemm_abt(acc, T0, T1);              // L_{k+1,k} = A_{k+1,k} Z_k^T
          __syncthreads();                        // T0 is overwritten with L_{k+1,k}
          store_acc(acc, k0 + TB, k0, 0, T0);
        }
      }
      cluster_arrive();                           // L_{k+1,k} is published (release)
      if (has_next) {
        tile_wait();
        __syncthreads();
        if (diag_panel) {                         // A_{k+1,k+1} -= L_{k+1,k} L_{k+1,k}^T in place
          double acc[2][2][2][2];
          cta_gemm_abt(acc, T0, T0);
          const int bi = w >> 1;
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int bj = 2 * (w & 1) + h;
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
              for (int b = 0; b < 2; ++b)
#pragma unroll
                for (int i = 0; i < 2; ++i)
                  T2[(16 * bj + 8 * b + 2 * q + i) * LDT + 16 * bi + 8 * a + g] -= acc[h][a][b][i];
          }
        }
        factor_resident(k + 1);
      }
      cluster_wait();
    } else {
      // B: the other panel tiles L_rk = A_rk Z^T (the rhs row included)
      const int first = diag_panel ? 1 : 0;
      if (np - first > 0) {
        const double* Z = ldiag + (size_t)k * TB * TB;
        __syncthreads();
        for (int e = tid; e < TB * TB / 2; e += blockDim.x) {
          const int c = e >> 5, m2 = (e & 31) * 2;
          const unsigned saddr = (unsigned)__cvta_generic_to_shared(T1 + c * LDT + m2);
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(Z + c * TB + m2));
        }
        asm volatile("cp.async.commit_group;\n" ::);
      }
      for (int t = first + rank - 1; t < np; t += kCluster - 1) {
        const size_t r0 = (size_t)prows[p0 + t] * TB;
        __syncthreads();
        load_tile(T0, S, lds, r0, k0);
        tile_wait();
        __syncthreads();
        double acc[2][2][2][2];
        cta_gemm_abt(acc, T0, T1);
        store_acc(acc, r0, k0, 0, nullptr);
      }
      cluster_arrive();
      cluster_wait();
      stamp(2 * k + 1);
      // C: trailing tiles other than the next diagonal one (CTA 0's)
      const int u0 = uptr[k], nu = uptr[k + 1] - u0;
      int slot = 0;
      for (int t = 0; t < nu; ++t) {
        if (ur[u0 + t] == k + 1 && uc[u0 + t] == k + 1) continue;
        if (slot++ % (kCluster - 1) != rank - 1) continue;
        update_tile(k, ur[u0 + t], uc[u0 + t]);
      }
    }
    cl.sync();
  }

  stamp(2 * nt);
  // back-substitution L^T x = y on CTA 0:  x_k = Z_kk^T (y_k - sum_{r > k} L_rk^T x_r).  The
  // solution stays in shared memory (T1/T2 are free by now) when it fits, and Z_kk is fetched
  // into registers before the dependent sums so that its latency overlaps them.
  if (rank != 0) return;
  double* v = T0;             // 64 entries
  double* part = T0 + 64;     // 8 warps x 64
  const bool xs_ok = n_pad <= 2 * TB * LDT;
  double* xs = xs_ok ? T1 : x;
  for (int k = nt - 1; k >= 0; --k) {
    const size_t k0 = (size_t)k * TB;
    const double* Z = ldiag + (size_t)k * TB * TB;
    double z0[8], z1[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double* zc = Z + (size_t)(8 * w + c) * TB;
      z0[c] = zc[lane];
      z1[c] = zc[32 + lane];
    }
    // warp w handles columns 8w..8w+7 of tile column k; lanes run over rows (coalesced)
    double sums[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) sums[c] = 0.0;
    for (int p = pptr[k]; p < pptr[k + 1]; ++p) {
      const int r = prows[p];
      if (r >= nt) continue;
      const size_t r0 = (size_t)r * TB;
      const double x0 = xs[r0 + lane], x1 = xs[r0 + 32 + lane];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const double* col = S + (k0 + 8 * w + c) * lds + r0;
        sums[c] += col[lane] * x0 + col[32 + lane] * x1;
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double s = warp_sum(sums[c]);
      if (lane == 0) v[8 * w + c] = S[(k0 + 8 * w + c) * lds + n_pad] - s;
    }
    __syncthreads();
    // x_k[col] = sum_m Z[m][col] v[m]  (Z col-major 64x64)
    const double v0 = v[lane], v1 = v[32 + lane];
    double zs[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) zs[c] = warp_sum(z0[c] * v0 + z1[c] * v1);
    if (lane == 0) {
#pragma unroll
      for (int c = 0; c < 8; ++c) part[8 * w + c] = zs[c];
    }
    __syncthreads();
    if (tid < TB) {
      xs[k0 + tid] = part[tid];
      if (xs_ok) x[k0 + tid] = part[tid];
    }
    __syncthreads();
    __threadfence_block();
  }
  stamp(2 * nt + 1);
}

// Pointers into the packed level plan (TileChol::h_lv on the device).
struct LevelPlanPtrs {
  const int *p1ptr, *p1, *p2ptr, *p2, *tr, *tc, *tmode, *tcptr, *ck, *perm, *bptr, *brow, *blptr, *bcol;
  int n_levels;
};

// Level-scheduled tile Cholesky + solve in one launch of a cluster, under the tile order and
// schedule of tile_levels_plan.  Logical tile (r, c) lives at physical tile (perm r, perm c)
// of S; its input, when the assembled tile is the mirrored (perm c, perm r), is read transposed.
// Per level (columns that are independent of each other):
//   phase 1: the columns of the previous level update every tile they reach,
//            A_rc -= sum_k L_rk L_ck^T (one task per target tile, k in a fixed order), and the
//            diagonal tiles of this level, their last updates in, are factored and inverted in
//            shared memory (Z_j = L_jj^-1 to ldiag);
//   phase 2: L_rj = A_rj Z_j^T for the off-diagonal tiles of this level's columns (the rhs row
//            included);
// the tasks of a phase are spread over the CTAs by the host, one cluster barrier after each
// phase.  Every tile is written by one CTA per phase and its updates are summed in a fixed
// order, so the result does not depend on timing.  Then the back-substitution, level by level
// from the top with the columns of a level spread over the CTAs.  The cluster size (8, or 16
// where the device allows it) is the one the plan was made for.
__global__ void __launch_bounds__(256)
    k_chol_levels(double* __restrict__ S, int ld, int nt, int n_pad, LevelPlanPtrs P,
                  double* __restrict__ ldiag, double* __restrict__ x, int* __restrict__ fail,
                  unsigned long long* __restrict__ trace) {
  pdl_wait();      // launched as a dependent of the system's assembly
  pdl_trigger();
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int ranks = (int)cl.num_blocks();   // the cluster size the plan was made for
  extern __shared__ double sm[];
  double* T0 = sm;
  double* T1 = sm + TB * LDT;
  double* T2 = sm + 2 * TB * LDT;
  // phase 1: tile set 0 = (T2 input, T0 and T1 operands), set 1 = the next three tiles
  auto In = [&](int set) { return set ? sm + 5 * TB * LDT : T2; };
  auto Oa = [&](int set) { return set ? sm + 3 * TB * LDT : T0; };
  auto Ob = [&](int set) { return set ? sm + 4 * TB * LDT : T1; };
  const size_t lds = (size_t)ld;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31, g = lane >> 2, q = lane & 3;
  auto stamp = [&](int slot) {
    if (trace != nullptr && tid == 0) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      trace[(size_t)slot * ranks + rank] = t;
    }
  };
  // rhs row of tile column j (at physical column pc0): b_j -= sum_k L_jk y_k (phase 1) and
  // y_j = Z_j b_j (phase 2); thread (group, col) sums every fourth t, groups combined in a fixed
  // order through shared memory
  double* red = sm + 6 * TB * LDT;
  auto rhs_update = [&](size_t pc0, int t) {
    const int col = tid & 63, grp = tid >> 6;
    double acc = 0.0;
    for (int u = P.tcptr[t]; u < P.tcptr[t + 1]; ++u) {
      const size_t pk0 = (size_t)P.perm[P.ck[u]] * TB;
      for (int s = grp; s < TB; s += 4) acc += S[(pk0 + s) * lds + n_pad] * S[(pk0 + s) * lds + pc0 + col];
    }
    red[grp * TB + col] = acc;
    __syncthreads();
    if (tid < TB) {
      double* b = S + (pc0 + tid) * lds + n_pad;
      *b = *b - (((red[tid] + red[TB + tid]) + red[2 * TB + tid]) + red[3 * TB + tid]);
    }
  };
  auto rhs_solve = [&](size_t pc0, int j) {
    const int col = tid & 63, grp = tid >> 6;
    const double* Z = ldiag + (size_t)j * TB * TB;
    double acc = 0.0;
    for (int s = grp; s < TB; s += 4) acc += S[(pc0 + s) * lds + n_pad] * Z[s * TB + col];
    red[grp * TB + col] = acc;
    __syncthreads();
    if (tid < TB) S[(pc0 + tid) * lds + n_pad] = ((red[tid] + red[TB + tid]) + red[2 * TB + tid]) + red[3 * TB + tid];
  };
  // tile row of fragment row a of this thread (the full-tile ownership of cta_gemm_abt_acc)
  auto frag_row = [&](int a) { return 16 * (w >> 1) + 8 * a + g; };

  for (int lv = 0; lv < P.n_levels; ++lv) {
    stamp(2 * lv);
    // The input tile and the first update's operands of the CTA's next task are fetched into the
    // other tile set while the current task computes its last product (tasks of one phase are
    // independent: their targets differ and their operands are panels of earlier levels).
    const int e_end = P.p1ptr[lv * ranks + rank + 1];
    auto issue = [&](int e, int set) -> bool {
      const int t = P.p1[e];
      const int r = P.tr[t], j = P.tc[t], mode = P.tmode[t] & 3;
      if (r == nt) return false;
      const size_t pr0 = (size_t)P.perm[r] * TB, pc0 = (size_t)P.perm[j] * TB;
      if (mode == 1) copy_tile(In(set), S, lds, pr0, pc0);
      else if (mode == 2) copy_tile(In(set), S, lds, pc0, pr0);
      if (P.tcptr[t] < P.tcptr[t + 1]) {
        const size_t pk0 = (size_t)P.perm[P.ck[P.tcptr[t]]] * TB;
        copy_tile(Oa(set), S, lds, pr0, pk0);                 // L_rk
        if (r != j) copy_tile(Ob(set), S, lds, pc0, pk0);     // L_jk
      }
      tile_commit();
      return true;
    };
    bool fetched = false;   // the current task's tiles were issued by the previous one
    int set = 0;
    for (int e = P.p1ptr[lv * ranks + rank]; e < e_end; ++e, set ^= 1) {
      const int t = P.p1[e];
      const int r = P.tr[t], j = P.tc[t], mode = P.tmode[t] & 3;
      const size_t pr0 = (size_t)P.perm[r] * TB, pc0 = (size_t)P.perm[j] * TB;
      const bool diag = r == j, factor = (P.tmode[t] & kLvFactor) != 0;
      __syncthreads();
      if (r == nt) {   // the rhs row: only row 0 of its tiles is nonzero, so each update is a GEMV
        rhs_update(pc0, t);
        fetched = false;
        continue;
      }
      if (!fetched) issue(e, set);
      fetched = false;
      double* Ti = In(set);
      double* Ta = Oa(set);
      double* Tb = Ob(set);
      double acc[2][2][2][2];
#pragma unroll
      for (int h = 0; h < 2; ++h) acc_zero(acc[h]);
      const int u0 = P.tcptr[t], u1 = P.tcptr[t + 1];
      if (u0 == u1) {   // no updates: wait for the input, then fetch the next task's tiles
        tile_wait();
        __syncthreads();
        if (e + 1 < e_end) fetched = issue(e + 1, set ^ 1);
      }
      for (int u = u0; u < u1; ++u) {
        if (u > u0) {
          const size_t pk0 = (size_t)P.perm[P.ck[u]] * TB;
          copy_tile(Ta, S, lds, pr0, pk0);                 // L_rk
          if (!diag) copy_tile(Tb, S, lds, pc0, pk0);      // L_jk
          tile_commit();
        }
        tile_wait();       // only this task's copies are in flight here
        __syncthreads();
        if (u + 1 == u1 && e + 1 < e_end) fetched = issue(e + 1, set ^ 1);
        if (diag) cta_gemm_aat_lower_acc(acc, Ta);   // only the lower triangle of a diagonal tile is read
        else cta_gemm_abt_acc(acc, Ta, false, Tb);
        __syncthreads();
      }
      // the 16x16 block (bi, bj) of fragment set h: the full ownership of cta_gemm_abt_acc, or
      // the lower-triangle table of cta_gemm_aat_lower_acc on a diagonal tile
      auto blk = [&](int h, int& bi, int& bj) -> bool {
        if (!diag) {
          bi = w >> 1;
          bj = 2 * (w & 1) + h;
          return true;
        }
        const int b = kLowerBlk[w][h];
        bi = b >> 2;
        bj = b & 3;
        return b >= 0;
      };
      if (factor) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int bi, bj;
          if (!blk(h, bi, bj)) continue;
#pragma unroll
          for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
              for (int i = 0; i < 2; ++i) Ti[(16 * bj + 8 * b + 2 * q + i) * LDT + 16 * bi + 8 * a + g] -= acc[h][a][b][i];
        }
        __syncthreads();
        const bool ok = cta_factor_tile8(Ti, Ta);   // Z into this set's first operand tile
        if (!ok && tid == 0) atomicExch(fail, 1);
        double* Z = ldiag + (size_t)j * TB * TB;
        for (int f = tid; f < TB * TB; f += blockDim.x) Z[f] = Ta[(f >> 6) * LDT + (f & 63)];
      } else {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          int bi, bj;
          if (!blk(h, bi, bj)) continue;
#pragma unroll
          for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b)
#pragma unroll
              for (int i = 0; i < 2; ++i) {
                const int row = 16 * bi + 8 * a + g, col = 16 * bj + 8 * b + 2 * q + i;
                const double in = mode == 1 ? Ti[col * LDT + row] : mode == 2 ? Ti[row * LDT + col] : 0.0;
                S[(pc0 + col) * lds + pr0 + row] = in - acc[h][a][b][i];
              }
        }
      }
    }
    tile_wait();   // nothing is in flight past the phase (no task is left to prefetch)
    cl.sync();   // arrive.release / wait.acquire at cluster scope: the CTAs' writes are visible
    stamp(2 * lv + 1);
    for (int e = P.p2ptr[lv * ranks + rank]; e < P.p2ptr[lv * ranks + rank + 1]; ++e) {
      const int t = P.p2[e];
      const int r = P.tr[t], j = P.tc[t];
      const size_t pr0 = (size_t)P.perm[r] * TB, pc0 = (size_t)P.perm[j] * TB;
      // an updated tile was written in place at (pr0, pc0); an untouched one is read as assembled
      const bool tr_in = P.tmode[t] == 2;
      __syncthreads();
      if (r == nt) {
        rhs_solve(pc0, j);
        continue;
      }
      if (tr_in) load_tile(T0, S, lds, pc0, pr0);
      else load_tile(T0, S, lds, pr0, pc0);
      const double* Z = ldiag + (size_t)j * TB * TB;
      for (int f = tid; f < TB * TB / 2; f += blockDim.x) {
        const int c = f >> 5, m2 = (f & 31) * 2;
        const unsigned saddr = (unsigned)__cvta_generic_to_shared(T1 + c * LDT + m2);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(Z + c * TB + m2));
      }
      asm volatile("cp.async.commit_group;\n" ::);
      tile_wait();
      __syncthreads();
      double acc[2][2][2][2];
#pragma unroll
      for (int h = 0; h < 2; ++h) acc_zero(acc[h]);
      cta_gemm_azt_acc(acc, T0, tr_in, T1);   // T1 = Z_j, lower triangular
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int bj = panel_bj(w, h);
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int i = 0; i < 2; ++i)
              S[(pc0 + 16 * bj + 8 * b + 2 * q + i) * lds + pr0 + frag_row(a)] = acc[h][a][b][i];
      }
    }
    cl.sync();   // arrive.release / wait.acquire at cluster scope: the CTAs' writes are visible
  }

  stamp(2 * P.n_levels);
  // back-substitution L^T x = y, x_k = Z_k^T (y_k - sum_{r > k} L_rk^T x_r), level by level from
  // the top: the columns of one level are spread over the CTAs (x in global memory, indexed
  // physically), a cluster barrier after each level
  double* v = T0;
  double* part = T0 + 64;
  for (int lv = P.n_levels - 1; lv >= 0; --lv) {
    for (int e = P.blptr[lv * ranks + rank]; e < P.blptr[lv * ranks + rank + 1]; ++e) {
      const int k = P.bcol[e];
      const size_t k0 = (size_t)P.perm[k] * TB;
      const double* Z = ldiag + (size_t)k * TB * TB;
      double z0[8], z1[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const double* zc = Z + (size_t)(8 * w + c) * TB;
        z0[c] = zc[lane];
        z1[c] = zc[32 + lane];
      }
      double sums[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) sums[c] = 0.0;
      for (int p = P.bptr[k]; p < P.bptr[k + 1]; ++p) {
        const size_t r0 = (size_t)P.perm[P.brow[p]] * TB;
        const double x0 = __ldcg(x + r0 + lane), x1 = __ldcg(x + r0 + 32 + lane);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const double* col = S + (k0 + 8 * w + c) * lds + r0;
          sums[c] += col[lane] * x0 + col[32 + lane] * x1;
        }
      }
      __syncthreads();   // v / part of the previous column are consumed
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const double s = warp_sum(sums[c]);
        if (lane == 0) v[8 * w + c] = S[(k0 + 8 * w + c) * lds + n_pad] - s;
      }
      __syncthreads();
      const double v0 = v[lane], v1 = v[32 + lane];
      double zs[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) zs[c] = warp_sum(z0[c] * v0 + z1[c] * v1);
      if (lane == 0) {
#pragma unroll
        for (int c = 0; c < 8; ++c) part[8 * w + c] = zs[c];
      }
      __syncthreads();
      if (tid < TB) x[k0 + tid] = part[tid];
    }
    cl.sync();   // arrive.release / wait.acquire at cluster scope: the CTAs' writes are visible
  }
  stamp(2 * P.n_levels + 1);
}

// Accuracy check of the pivot reciprocal square root (tests): out[2 i] = rsqrt_nr(x_i),
// out[2 i + 1] = rsqrt(x_i) (CUDA's), both evaluated on the device.
__global__ void k_recip_check(const double* __restrict__ x, int n, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = x[i];
  out[2 * i] = rsqrt_nr(v);
  out[2 * i + 1] = rsqrt(v);
}

// Function attributes are set once per device (a process may drive several GPUs).
int chol_cluster_setup() {
  static std::atomic<uint64_t> done_mask{0};
  int dev = 0;
  V3DBA_CUDA_TRY(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (done_mask.load() & bit) return V3DBA_OK;
  V3DBA_CUDA_TRY(cudaFuncSetAttribute(k_chol_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(3 * TB * LDT * sizeof(double))));
  V3DBA_CUDA_TRY(cudaFuncSetAttribute(k_chol_levels, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kLevelsSmem));
  done_mask.fetch_or(bit);
  return V3DBA_OK;
}

int chol_cluster_solve(const TileChol& tc, double* S, double* x, int* d_fail, cudaStream_t st,
                       unsigned long long* trace) {
  int rc = chol_cluster_setup();
  if (rc) return rc;
  const size_t smem = 3 * TB * LDT * sizeof(double);
  k_chol_cluster<<<kCluster, 256, smem, st>>>(S, tc.ld, tc.nt, tc.n_pad, tc.d_panel_ptr, tc.d_panel_rows,
                                              tc.d_upd_ptr, tc.d_upd_r, tc.d_upd_c, tc.d_ldiag, x, d_fail, trace);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

int chol_levels_solve(const TileChol& tc, double* S, double* x, int* d_fail, cudaStream_t st,
                      unsigned long long* trace) {
  if (!tc.levels || !tc.d_lv) return V3DBA_ERR_INVALID_ARGUMENT;
  int rc = chol_cluster_setup();
  if (rc) return rc;
  const int* b = tc.d_lv;
  LevelPlanPtrs P;
  P.p1ptr = b + tc.lv_off[kLvP1Ptr];
  P.p1 = b + tc.lv_off[kLvP1];
  P.p2ptr = b + tc.lv_off[kLvP2Ptr];
  P.p2 = b + tc.lv_off[kLvP2];
  P.tr = b + tc.lv_off[kLvTaskR];
  P.tc = b + tc.lv_off[kLvTaskC];
  P.tmode = b + tc.lv_off[kLvTaskMode];
  P.tcptr = b + tc.lv_off[kLvTaskCPtr];
  P.ck = b + tc.lv_off[kLvCK];
  P.perm = b + tc.lv_off[kLvPerm];
  P.bptr = b + tc.lv_off[kLvBPtr];
  P.brow = b + tc.lv_off[kLvBRow];
  P.blptr = b + tc.lv_off[kLvBLvPtr];
  P.bcol = b + tc.lv_off[kLvBCol];
  P.n_levels = tc.n_levels;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(tc.lv_ranks, 1, 1);
  cfg.blockDim = dim3(256, 1, 1);
  cfg.dynamicSmemBytes = kLevelsSmem;
  cfg.stream = st;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = tc.lv_ranks;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;   // see pdl_wait()
  attr[1].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 2;
  V3DBA_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_chol_levels, S, tc.ld, tc.nt, tc.n_pad, P, tc.d_ldiag, x, d_fail, trace));
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

int chol_levels_ranks() {
  static std::atomic<int> ranks_of[64];   // per device: 0 until decided
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 8;
  }
  std::atomic<int>& cached = ranks_of[dev & 63];
  if (cached.load()) return cached.load();
  int ranks = 8;
  if (chol_cluster_setup() != V3DBA_OK) {
    cudaGetLastError();
    return ranks;
  }
  const size_t smem = kLevelsSmem;
  if (cudaFuncSetAttribute(k_chol_levels, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16, 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 16;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_chol_levels, &cfg) == cudaSuccess && n >= 1) ranks = 16;
  }
  cudaGetLastError();
  cached.store(ranks);
  return ranks;
}

}  // namespace v3dba

extern "C" int v3dba_check_pivot_reciprocals(int n, const double* x, double* out) {
  if (n <= 0 || !x || !out) return V3DBA_ERR_INVALID_ARGUMENT;
  double *dx = nullptr, *dout = nullptr;
  V3DBA_CUDA_TRY(cudaMalloc(&dx, sizeof(double) * n));
  if (cudaMalloc(&dout, sizeof(double) * 2 * n) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dx);
    return V3DBA_ERR_OUT_OF_MEMORY;
  }
  cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
  v3dba::k_recip_check<<<(n + 255) / 256, 256>>>(dx, n, dout);
  v3dba::note_launches(1);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dout);
  return e == cudaSuccess ? V3DBA_OK : V3DBA_ERR_CUDA;
}
