// One-launch tile Cholesky of the reduced camera system on a thread-block cluster.
//
// Same factorisation as tile_cholesky.cu (right-looking over 64x64 tiles, rhs carried as tile row
// nt, tiles that are structurally zero in L skipped), but the whole factor + solve runs in ONE
// launch of an 8-CTA cluster: the phases of a tile step are separated by cluster barriers
// (barrier.cluster, sub-microsecond) instead of kernel boundaries, which removes the launch and
// drain latency that dominates small reduced systems (hundreds to a few thousand unknowns).
//
// Per tile column k, CTA 0 owns the chain along the diagonal and keeps it in shared memory:
//   with Z_k = L_kk^-1 resident it forms the panel tile next to the diagonal,
//   L_{k+1,k} = A_{k+1,k} Z_k^T, publishes it (split cluster barrier: arrive, keep working), applies
//   it to the next diagonal tile (fetched meanwhile) and factors that tile: 16-column blocking,
//   each 16x16 diagonal block factored and inverted by one warp in registers, panels and trailing
//   blocks updated with FP64 tensor-core MMAs (DMMA m8n8k4), Z_{k+1} assembled;
//   CTAs 1.. form the other panel tiles (and the rhs row), L_rk = A_rk Z_k^T, one 64x64x64 DMMA
//   GEMM per tile, then the other trailing tiles, A_rc -= L_rk L_ck^T (DMMA).
// Then the back-substitution L^T x = y (y = the factored rhs row) by CTA 0, with x kept in
// shared memory and Z_kk fetched ahead of the dependent sums.
#include <cooperative_groups.h>

#include <algorithm>
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
constexpr unsigned FULL = 0xffffffffu;

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

// 1/sqrt(x) for a positive pivot: the hardware approximation (rsqrt.approx.ftz.f64, one
// instruction) refined by two Newton-Raphson steps y <- y (1.5 - 0.5 x y^2) in FP64, each of
// which roughly doubles the number of correct bits.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double hx = 0.5 * x;
  y = y * (1.5 - hx * y * y);
  y = y * (1.5 - hx * y * y);
  return y;
}

// One warp: Cholesky of the 16x16 block D (lower, col-major ld LDT) in place and its inverse
// into Z (16x16, col-major, zero upper part).  Returns false on a non-positive pivot.
// Lane c (< 16) owns column c in registers.  At pivot j lane j scales its column by one
// reciprocal square root and stores it to D; after a warp barrier every lane reads that column
// back with broadcast vector loads and applies its rank-1 update.  The inverse is then formed
// column by column (lane c computes Z[:, c]) from broadcast reads of L.
__device__ bool warp_chol_inv16(double* D, double* Z) {
  const int lane = threadIdx.x & 31;
  const int c = lane;                 // owned column (lanes >= 16 own none)
  __shared__ double inv_diag[8][16];  // per-warp reciprocal diagonal of L
  double* invd = inv_diag[threadIdx.x >> 5];
  double a[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) a[r] = (c < 16 && r >= c) ? D[c * LDT + r] : 0.0;
  bool ok = true;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    if (c == j) {
      const double d = a[j];
      const double rs = d > 0.0 ? rsqrt_nr(d) : 1.0;
      if (!(d > 0.0)) ok = false;
      invd[j] = rs;
      a[j] = d * rs;
#pragma unroll
      for (int r = j + 1; r < 16; ++r) a[r] *= rs;
      double2* col = reinterpret_cast<double2*>(D + j * LDT);
#pragma unroll
      for (int r = 0; r < 16; r += 2) col[r / 2] = make_double2(r >= j ? a[r] : 0.0, r + 1 >= j ? a[r + 1] : 0.0);
    }
    __syncwarp();
    if (c > j && c < 16) {
      const double2* col = reinterpret_cast<const double2*>(D + j * LDT);
      double l[16];
#pragma unroll
      for (int r = 0; r < 16; r += 2) {
        const double2 v = col[r / 2];
        l[r] = v.x;
        l[r + 1] = v.y;
      }
      const double m = D[j * LDT + c];
#pragma unroll
      for (int r = j + 1; r < 16; ++r)
        if (r >= c) a[r] -= l[r] * m;
    }
    __syncwarp();
  }
  ok = __all_sync(FULL, ok);
  // Z[:, c]: z[rr] = (delta_{rr,c} - sum_{t<rr} L[rr][t] z[t]) / L[rr][rr]
  if (c < 16) {
    double z[16];
#pragma unroll
    for (int rr = 0; rr < 16; ++rr) {
      double s0 = (rr == c) ? 1.0 : 0.0, s1 = 0.0;
#pragma unroll
      for (int t = 0; t < rr; t += 2) {
        s0 -= D[t * LDT + rr] * z[t];
        if (t + 1 < rr) s1 -= D[(t + 1) * LDT + rr] * z[t + 1];
      }
      z[rr] = (rr >= c) ? (s0 + s1) * invd[rr] : 0.0;
    }
#pragma unroll
    for (int rr = 0; rr < 16; ++rr) Z[c * LDT + rr] = z[rr];
  }
  __syncwarp();
  return ok;
}

// C(16x16 at C, col-major ldc) = alpha * acc + beta * C
__device__ __forceinline__ void acc_store(const double (&acc)[2][2][2], double* C, int ldc, double alpha, double beta) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        double* p = C + (8 * b + 2 * q + i) * ldc + 8 * a + g;
        *p = alpha * acc[a][b][i] + (beta != 0.0 ? beta * *p : 0.0);
      }
}

// CTA (256 threads): factor the 64x64 tile A (shared, col-major LDT, lower triangle valid) in
// place and write Z = L^-1 (full 64x64, zero upper part) into Zs.  Blocked by 16 columns: each
// 16x16 diagonal block is factored and inverted by one warp (warp_chol_inv16); the panel blocks
// (L_ip = A_ip Z_pp^T), the trailing blocks (A_ij -= L_ip L_jp^T) and the off-diagonal blocks of
// Z (Z_ij = -Z_ii sum_t L_it Z_tj, by distance i - j) are 16x16 DMMA products.  Returns false
// on a non-positive pivot.
__device__ bool cta_factor_tile(double* A, double* Zs) {
  const int tid = threadIdx.x, w = tid >> 5;
  __shared__ int s_ok;
  if (tid == 0) s_ok = 1;
  for (int e = tid; e < TB * TB; e += blockDim.x) Zs[(e >> 6) * LDT + (e & 63)] = 0.0;
  __syncthreads();
  for (int p = 0; p < 4; ++p) {
    double* App = A + 16 * p * LDT + 16 * p;
    if (w == 0) {
      const bool ok = warp_chol_inv16(App, Zs + 16 * p * LDT + 16 * p);
      if ((threadIdx.x & 31) == 0 && !ok) s_ok = 0;
    }
    __syncthreads();
    if (w < 3 - p) {
      const int i = p + 1 + w;
      double acc[2][2][2];
      acc_zero(acc);
      const double* Aip = A + 16 * p * LDT + 16 * i;
      const double* Zpp = Zs + 16 * p * LDT + 16 * p;
      warp_mma16(acc, Aip, 1, LDT, Zpp, LDT, 1, 16);   // A_ip Z_pp^T
      __syncwarp();
      acc_store(acc, A + 16 * p * LDT + 16 * i, LDT, 1.0, 0.0);
    }
    __syncthreads();
    {
      int task = 0;
      for (int i = p + 1; i < 4; ++i)
        for (int j = p + 1; j <= i; ++j, ++task) {
          if (task % 8 != w) continue;
          double acc[2][2][2];
          acc_zero(acc);
          warp_mma16(acc, A + 16 * p * LDT + 16 * i, 1, LDT, A + 16 * p * LDT + 16 * j, LDT, 1, 16);
          acc_store(acc, A + 16 * j * LDT + 16 * i, LDT, -1.0, 1.0);
        }
    }
    __syncthreads();
  }
  for (int d = 1; d < 4; ++d) {
    if (w < 4 - d) {
      const int j = w, i = w + d;
      double acc[2][2][2];
      acc_zero(acc);
      for (int t = j; t < i; ++t)
        warp_mma16(acc, A + 16 * t * LDT + 16 * i, 1, LDT, Zs + 16 * j * LDT + 16 * t, 1, LDT, 16);
      double* Wij = Zs + 16 * j * LDT + 16 * i;   // still zero: use it as scratch for W
      acc_store(acc, Wij, LDT, 1.0, 0.0);
      __syncwarp();
      double acc2[2][2][2];
      acc_zero(acc2);
      warp_mma16(acc2, Zs + 16 * i * LDT + 16 * i, 1, LDT, Wij, 1, LDT, 16);
      __syncwarp();
      acc_store(acc2, Wij, LDT, -1.0, 0.0);
    }
    __syncthreads();
  }
  return s_ok != 0;
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
    const bool ok = cta_factor_tile(T2, T1);
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
  __threadfence();
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
      __threadfence();
      cluster_arrive();                           // L_{k+1,k} is published
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
      __threadfence();
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
    __threadfence();
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

int chol_cluster_setup() {
  static bool done = false;
  if (done) return V3DBA_OK;
  V3DBA_CUDA_TRY(cudaFuncSetAttribute(k_chol_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(3 * TB * LDT * sizeof(double))));
  done = true;
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

}  // namespace v3dba
