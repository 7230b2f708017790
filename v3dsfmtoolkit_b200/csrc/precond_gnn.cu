// Learned correction to the block-Jacobi preconditioner of the PCG reduced-camera solve.
//
// The reference has no iterative solver: it factors the damped normal equations with LDL^T
// (V3D/src/Math/v3d_optimization.cpp:1096-1145).  For scenes whose reduced camera system S is
// solved by PCG instead, this file provides a factorised preconditioner M^-1 = G^T G with
//
//   G = (I + E) C^-1,   C_i C_i^T = S_ii (Cholesky of each 6x6 diagonal camera block),
//
// E strictly block-lower on the co-visibility pattern of S.  E = 0 is block-Jacobi.  In the
// normalised coordinates S^ = C^-1 S C^-T = I + F + F^T (F strictly lower) each edge block is
//
//   E_e = -c0 F_e + c1 (F F)_e + c2 (F F^T)_e        (products restricted to the pattern),
//
// the first-order expansion of the factorised sparse approximate inverse (FSAI) of S^ for
// c = (1, 1, 1).  A message-passing network over the camera graph predicts c - 1 per edge from
// the three normalised 6x6 blocks of the edge and four node statistics:
//
//   e0 = relu(We x_e + b), h0 = relu(Wn x_n + b)
//   3 x { e += relu(Wm [h_b, h_a, e] + b);  h += relu(Wh [h, mean_incident(e)] + b) (first two) }
//   c - 1 = Wo e + b                         (Wo = 0 at initialisation: c = 1)
//
// Training minimises L = |P z - z|^2 / (n m) over m Rademacher probes z, P = (I+E) S^ (I+E)^T,
// an estimate of |P - I|_F^2 / n, with hand-written FP32 forward/backward kernels and Adam.
// Inference inside the LM loop runs the hidden layers on BF16 tensor cores (mma.sync m16n8k16,
// FP32 accumulate).  Every reduction over edges or rows is a fixed-order gather (no atomics), so
// results are run-to-run deterministic.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "common.cuh"
#include "lm.cuh"
#include "precond.cuh"

namespace v3dba {
namespace {

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

template <typename T>
int upload_vec(T** d, const std::vector<T>& h) {
  V3DBA_CUDA_TRY(cudaMalloc(d, sizeof(T) * std::max<size_t>(h.size(), 1)));
  if (!h.empty()) V3DBA_CUDA_TRY(cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return V3DBA_OK;
}

}  // namespace

// --------------------------------------------------------------------------------------------
// graph
// --------------------------------------------------------------------------------------------

int gnn_graph_build(GnnGraph& g, int N, const std::vector<int>& b_i, const std::vector<int>& b_l) {
  std::vector<int> ea, eb, eblk;
  for (size_t b = 0; b < b_i.size(); ++b) {
    const int i = std::min(b_i[b], b_l[b]), l = std::max(b_i[b], b_l[b]);
    if (i == l) continue;
    ea.push_back(i);
    eb.push_back(l);
    eblk.push_back((int)b);
  }
  const int ne = (int)ea.size();
  // lower lists (by b, ordered by a) and upper lists (by a, ordered by b)
  std::vector<int> lo_ptr(N + 1, 0), up_ptr(N + 1, 0), lo_e(ne), up_e(ne);
  for (int e = 0; e < ne; ++e) { lo_ptr[eb[e] + 1]++; up_ptr[ea[e] + 1]++; }
  for (int i = 0; i < N; ++i) { lo_ptr[i + 1] += lo_ptr[i]; up_ptr[i + 1] += up_ptr[i]; }
  {
    std::vector<int> fl(lo_ptr.begin(), lo_ptr.end() - 1), fu(up_ptr.begin(), up_ptr.end() - 1);
    for (int e = 0; e < ne; ++e) { lo_e[fl[eb[e]]++] = e; up_e[fu[ea[e]]++] = e; }
    for (int i = 0; i < N; ++i) {
      std::sort(lo_e.begin() + lo_ptr[i], lo_e.begin() + lo_ptr[i + 1], [&](int x, int y) { return ea[x] < ea[y]; });
      std::sort(up_e.begin() + up_ptr[i], up_e.begin() + up_ptr[i + 1], [&](int x, int y) { return eb[x] < eb[y]; });
    }
  }
  // two-hop products of edge (a, b), the lower position (b, a):
  //   (F F)_(b,a)   = sum over a < k < b of F_(b,k) F_(k,a): edges (k, b) and (a, k)
  //   (F F^T)_(b,a) = sum over k < a of F_(b,k) F_(a,k)^T:  edges (k, b) and (k, a)
  std::vector<int> tri_ptr(1, 0), t1, t2;
  std::vector<unsigned char> tt;
  for (int e = 0; e < ne; ++e) {
    const int a = ea[e], b = eb[e];
    int p = up_ptr[a], q = lo_ptr[b];
    while (p < up_ptr[a + 1] && q < lo_ptr[b + 1]) {
      const int kp = eb[up_e[p]], kq = ea[lo_e[q]];
      if (kp < kq) ++p;
      else if (kq < kp) ++q;
      else {
        if (kp < b) { t1.push_back(lo_e[q]); t2.push_back(up_e[p]); tt.push_back(0); }
        ++p; ++q;
      }
    }
    p = lo_ptr[a]; q = lo_ptr[b];
    while (p < lo_ptr[a + 1] && q < lo_ptr[b + 1]) {
      const int kp = ea[lo_e[p]], kq = ea[lo_e[q]];
      if (kp < kq) ++p;
      else if (kq < kp) ++q;
      else { t1.push_back(lo_e[q]); t2.push_back(lo_e[p]); tt.push_back(1); ++p; ++q; }
    }
    tri_ptr.push_back((int)t1.size());
  }
  gnn_graph_free(g);
  g.N = N; g.ne = ne; g.ntri = (int)t1.size();
  int rc;
  if ((rc = upload_vec(&g.ea, ea)) || (rc = upload_vec(&g.eb, eb)) || (rc = upload_vec(&g.eblk, eblk)) ||
      (rc = upload_vec(&g.lo_ptr, lo_ptr)) || (rc = upload_vec(&g.lo_e, lo_e)) || (rc = upload_vec(&g.up_ptr, up_ptr)) ||
      (rc = upload_vec(&g.up_e, up_e)) || (rc = upload_vec(&g.tri_ptr, tri_ptr)) || (rc = upload_vec(&g.tri_1, t1)) ||
      (rc = upload_vec(&g.tri_2, t2)) || (rc = upload_vec(&g.tri_t, tt)))
    return rc;
  return V3DBA_OK;
}

void gnn_graph_free(GnnGraph& g) {
  cudaFree(g.ea); cudaFree(g.eb); cudaFree(g.eblk); cudaFree(g.lo_ptr); cudaFree(g.lo_e); cudaFree(g.up_ptr);
  cudaFree(g.up_e); cudaFree(g.tri_ptr); cudaFree(g.tri_1); cudaFree(g.tri_2); cudaFree(g.tri_t);
  g = GnnGraph();
}

namespace {

// --------------------------------------------------------------------------------------------
// normalisation and input features
// --------------------------------------------------------------------------------------------

// C_i^-1 of the Cholesky factor of each diagonal block (FP64 arithmetic, stored FP32, lower).
template <typename Real>
__global__ void k_gnn_cinv(const Real* __restrict__ Sb, const int* __restrict__ diag_blk, int N, float* cinv,
                           int* fail) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const Real* A = Sb + (size_t)diag_blk[i] * 36;
  double L[6][6], X[6][6];
  bool ok = true;
  for (int j = 0; j < 6; ++j) {
    double d = double(A[j * 6 + j]);
    for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k];
    if (!(d > 0.0)) { ok = false; d = 1.0; }
    L[j][j] = sqrt(d);
    for (int r = j + 1; r < 6; ++r) {
      double v = double(A[r * 6 + j]);
      for (int k = 0; k < j; ++k) v -= L[r][k] * L[j][k];
      L[r][j] = v / L[j][j];
    }
  }
  for (int c = 0; c < 6; ++c) {
    for (int r = 0; r < c; ++r) X[r][c] = 0.0;
    X[c][c] = 1.0 / L[c][c];
    for (int r = c + 1; r < 6; ++r) {
      double v = 0.0;
      for (int k = c; k < r; ++k) v += L[r][k] * X[k][c];
      X[r][c] = -v / L[r][r];
    }
  }
  if (!ok) *fail = 1;
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) cinv[(size_t)i * 36 + r * 6 + c] = float(X[r][c]);
}

// F_e = C_b^-1 S_(b,a) C_a^-T, S_(b,a) the transpose of the stored block (a, b).
template <typename Real>
__global__ void k_gnn_edge_norm(const Real* __restrict__ Sb, GnnGraph g, const float* __restrict__ cinv, float* xe) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.ne) return;
  const Real* B = Sb + (size_t)g.eblk[e] * 36;
  const float* Ca = cinv + (size_t)g.ea[e] * 36;
  const float* Cb = cinv + (size_t)g.eb[e] * 36;
  double T[6][6];
  for (int r = 0; r < 6; ++r)          // T = S_(b,a) C_a^-T:  T[r][c] = sum_k B[k][r] Ca[c][k]
    for (int c = 0; c < 6; ++c) {
      double v = 0.0;
      for (int k = 0; k <= c; ++k) v += double(B[k * 6 + r]) * double(Ca[c * 6 + k]);
      T[r][c] = v;
    }
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) {
      double v = 0.0;
      for (int k = 0; k <= r; ++k) v += double(Cb[r * 6 + k]) * T[k][c];
      xe[(size_t)e * kGnnEdgeIn + r * 6 + c] = float(v);
    }
}

// Two-hop products of every edge: 72 threads per edge, one per output entry (36 of (F F), 36 of
// (F F^T)); the threads of an edge walk its triangles together and share their loads.
__global__ void __launch_bounds__(288) k_gnn_two_hop(GnnGraph g, float* xe) {
  const int e = blockIdx.x * 4 + threadIdx.y;
  if (e >= g.ne) return;
  const int o = threadIdx.x;                 // 0..71
  const int kind = o >= 36 ? 1 : 0;
  const int r = (o % 36) / 6, c = o % 6;
  float acc = 0.f;
  for (int t = g.tri_ptr[e]; t < g.tri_ptr[e + 1]; ++t) {
    if (g.tri_t[t] != kind) continue;
    const float* A = xe + (size_t)g.tri_1[t] * kGnnEdgeIn + r * 6;
    const float* B = xe + (size_t)g.tri_2[t] * kGnnEdgeIn;
    if (kind == 0) {
#pragma unroll
      for (int k = 0; k < 6; ++k) acc += A[k] * B[k * 6 + c];
    } else {
#pragma unroll
      for (int k = 0; k < 6; ++k) acc += A[k] * B[c * 6 + k];
    }
  }
  xe[(size_t)e * kGnnEdgeIn + 36 + o] = acc;
}

__device__ __forceinline__ int node_degree(const GnnGraph& g, int i) {
  return (g.lo_ptr[i + 1] - g.lo_ptr[i]) + (g.up_ptr[i + 1] - g.up_ptr[i]);
}

// Node statistics, one warp per node (lanes over its incident edges).
__global__ void k_gnn_node_feat(GnnGraph g, const float* __restrict__ xe, float* xn) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= g.N) return;
  const int nlo = g.lo_ptr[i + 1] - g.lo_ptr[i];
  const int deg = node_degree(g, i);
  float sum = 0.f, mx = 0.f;
  for (int q = lane; q < deg; q += 32) {
    const int e = q < nlo ? g.lo_e[g.lo_ptr[i] + q] : g.up_e[g.up_ptr[i] + q - nlo];
    const float4* F = reinterpret_cast<const float4*>(xe + (size_t)e * kGnnEdgeIn);
    float v = 0.f;
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const float4 f = F[t];
      v += f.x * f.x + f.y * f.y + f.z * f.z + f.w * f.w;
    }
    sum += v;
    mx = fmaxf(mx, v);
  }
  sum = warp_sum(sum);
  mx = warp_max(mx);
  if (lane == 0) {
    xn[(size_t)i * 4 + 0] = 1.f;
    xn[(size_t)i * 4 + 1] = log1pf((float)deg);
    xn[(size_t)i * 4 + 2] = deg ? sum / deg : 0.f;
    xn[(size_t)i * 4 + 3] = mx;
  }
}

// --------------------------------------------------------------------------------------------
// dense row layers (FP32 training path)
// --------------------------------------------------------------------------------------------

struct Seg {
  const float* src = nullptr;
  const int* idx = nullptr;   // row r reads src row idx[r] (or r when null)
  int ld = 0;
  int width = 0;
};

__device__ __forceinline__ float seg_load(const Seg* seg, int nseg, int row, int k) {
  int s = 0;
  while (s + 1 < nseg && k >= seg[s].width) { k -= seg[s].width; ++s; }
  const int src_row = seg[s].idx ? seg[s].idx[row] : row;
  return seg[s].src[(size_t)src_row * seg[s].ld + k];
}

struct RowGemm {
  int rows = 0, nseg = 0, K = 0, Nout = 0;
  Seg seg[3];
  const float* W = nullptr;   // element (k, c) at W[k * wk + c * wn]
  int wk = 0, wn = 0;
  const float* bias = nullptr;
  const float* resid = nullptr;   // out = resid + act(z)
  float* out = nullptr;
  int ldo = 0;
  float* act_out = nullptr;       // act(z) as well (ld Nout)
  int relu = 0;
};

constexpr int kRgRows = 64;

// out[r, :] = act([segments of row r] W + b) (+ resid), 64 rows per block.
__global__ void __launch_bounds__(256) k_rowgemm(RowGemm g) {
  extern __shared__ float sm[];
  const int Kp = g.K + 1;
  float* in_s = sm;
  float* w_s = sm + kRgRows * Kp;
  const int r0 = blockIdx.x * kRgRows;
  for (int t = threadIdx.x; t < g.K * g.Nout; t += blockDim.x) {
    const int k = t / g.Nout, c = t - k * g.Nout;
    w_s[t] = g.W[(size_t)k * g.wk + (size_t)c * g.wn];
  }
  for (int t = threadIdx.x; t < kRgRows * g.K; t += blockDim.x) {
    const int r = t / g.K, k = t - r * g.K;
    const int row = r0 + r;
    in_s[r * Kp + k] = row < g.rows ? seg_load(g.seg, g.nseg, row, k) : 0.f;
  }
  __syncthreads();
  const int cl = threadIdx.x & 63, rg = threadIdx.x >> 6;
  for (int c0 = 0; c0 < g.Nout; c0 += 64) {
    const int c = c0 + cl;
    if (c >= g.Nout) continue;
    float acc[16];
    const float b = g.bias ? g.bias[c] : 0.f;
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[j] = b;
    for (int k = 0; k < g.K; ++k) {
      const float w = w_s[k * g.Nout + c];
#pragma unroll
      for (int j = 0; j < 16; ++j) acc[j] += in_s[(rg + 4 * j) * Kp + k] * w;
    }
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int row = r0 + rg + 4 * j;
      if (row >= g.rows) continue;
      const float z = g.relu ? fmaxf(acc[j], 0.f) : acc[j];
      if (g.act_out) g.act_out[(size_t)row * g.Nout + c] = z;
      g.out[(size_t)row * g.ldo + c] = g.resid ? g.resid[(size_t)row * g.ldo + c] + z : z;
    }
  }
}

struct WGrad {
  int rows = 0, nseg = 0, K = 0, Nout = 0;
  Seg seg[3];
  const float* D = nullptr;   // [rows x Nout]
  float* part = nullptr;      // [gridDim.x x (K + 1) * Nout]
};

constexpr int kWgRows = 256;
constexpr int kWgPer = 49;   // ceil((3 * 64 + 1) * 64 / 256)

// Partial [W; b] gradients: sum over this block's rows of [x_r, 1]^T D_r.
__global__ void __launch_bounds__(256) k_wgrad(WGrad g) {
  extern __shared__ float sm[];
  const int Kp = g.K + 1;
  float* x_s = sm;
  float* d_s = sm + 32 * Kp;
  const int nout = Kp * g.Nout;
  float acc[kWgPer];
#pragma unroll
  for (int j = 0; j < kWgPer; ++j) acc[j] = 0.f;
  const int rb = blockIdx.x * kWgRows;
  for (int s0 = 0; s0 < kWgRows; s0 += 32) {
    __syncthreads();
    for (int t = threadIdx.x; t < 32 * Kp; t += blockDim.x) {
      const int r = t / Kp, k = t - r * Kp;
      const int row = rb + s0 + r;
      float v = 0.f;
      if (row < g.rows) v = (k == g.K) ? 1.f : seg_load(g.seg, g.nseg, row, k);
      x_s[t] = v;
    }
    for (int t = threadIdx.x; t < 32 * g.Nout; t += blockDim.x) {
      const int r = t / g.Nout, c = t - r * g.Nout;
      const int row = rb + s0 + r;
      d_s[t] = row < g.rows ? g.D[(size_t)row * g.Nout + c] : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kWgPer; ++j) {
      const int o = threadIdx.x + j * 256;
      if (o < nout) {
        const int k = o / g.Nout, c = o - k * g.Nout;
        float a = acc[j];
#pragma unroll 8
        for (int r = 0; r < 32; ++r) a += x_s[r * Kp + k] * d_s[r * g.Nout + c];
        acc[j] = a;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kWgPer; ++j) {
    const int o = threadIdx.x + j * 256;
    if (o < nout) g.part[(size_t)blockIdx.x * nout + o] = acc[j];
  }
}

__global__ void k_wgrad_reduce(const float* __restrict__ part, int nblk, int nout, float* grad) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nout) return;
  float s = 0.f;
  for (int b = 0; b < nblk; ++b) s += part[(size_t)b * nout + o];
  grad[o] = s;
}

// --------------------------------------------------------------------------------------------
// BF16 tensor-core rows (inference): Nout = 64, K padded to a multiple of 16
// --------------------------------------------------------------------------------------------

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// out = act([segments] W + b) (+ resid) for 64-row tiles; Wt is W^T (64 x Kp, bf16, zero
// padded).  Four warps, 16 rows each, eight 16x8 output tiles per warp.
__global__ void __launch_bounds__(128) k_rowgemm_bf16(RowGemm g, const __nv_bfloat16* __restrict__ Wt, int Kp) {
  extern __shared__ __align__(16) unsigned char smb[];
  const int ld = Kp + 8;
  __nv_bfloat16* a_s = reinterpret_cast<__nv_bfloat16*>(smb);
  __nv_bfloat16* b_s = a_s + 64 * ld;
  const int r0 = blockIdx.x * 64;
  // weights: 8 bf16 per 16-byte copy (Kp is a multiple of 16, rows of b_s 16-byte aligned)
  const int kq8 = Kp / 8;
  for (int t = threadIdx.x; t < 64 * kq8; t += blockDim.x) {
    const int n = t / kq8, k = (t - n * kq8) * 8;
    *reinterpret_cast<uint4*>(b_s + n * ld + k) = *reinterpret_cast<const uint4*>(Wt + (size_t)n * Kp + k);
  }
  // inputs: 4 floats per 16-byte load (segment widths and leading dimensions are multiples of 4)
  const int kq4 = Kp / 4;
  for (int t = threadIdx.x; t < 64 * kq4; t += blockDim.x) {
    const int r = t / kq4, k = (t - r * kq4) * 4;
    const int row = r0 + r;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (row < g.rows && k < g.K) {
      int sgi = 0, kk = k;
      while (sgi + 1 < g.nseg && kk >= g.seg[sgi].width) { kk -= g.seg[sgi].width; ++sgi; }
      const Seg& sg = g.seg[sgi];
      const int src_row = sg.idx ? sg.idx[row] : row;
      v = *reinterpret_cast<const float4*>(sg.src + (size_t)src_row * sg.ld + kk);
    }
    __nv_bfloat162 lo = __floats2bfloat162_rn(v.x, v.y), hi = __floats2bfloat162_rn(v.z, v.w);
    uint2 pk;
    pk.x = *reinterpret_cast<uint32_t*>(&lo);
    pk.y = *reinterpret_cast<uint32_t*>(&hi);
    *reinterpret_cast<uint2*>(a_s + r * ld + k) = pk;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  float acc[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
  const __nv_bfloat16* arow0 = a_s + (warp * 16 + gq) * ld;
  const __nv_bfloat16* arow1 = arow0 + 8 * ld;
  for (int k0 = 0; k0 < Kp; k0 += 16) {
    uint32_t af[4];
    af[0] = *reinterpret_cast<const uint32_t*>(arow0 + k0 + 2 * tq);
    af[1] = *reinterpret_cast<const uint32_t*>(arow1 + k0 + 2 * tq);
    af[2] = *reinterpret_cast<const uint32_t*>(arow0 + k0 + 8 + 2 * tq);
    af[3] = *reinterpret_cast<const uint32_t*>(arow1 + k0 + 8 + 2 * tq);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const __nv_bfloat16* brow = b_s + (nt * 8 + gq) * ld + k0;
      uint32_t bf[2];
      bf[0] = *reinterpret_cast<const uint32_t*>(brow + 2 * tq);
      bf[1] = *reinterpret_cast<const uint32_t*>(brow + 8 + 2 * tq);
      mma_bf16_16816(acc[nt], af, bf);
    }
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int row = r0 + warp * 16 + gq + (q >> 1) * 8;
      const int c = nt * 8 + 2 * tq + (q & 1);
      if (row >= g.rows) continue;
      float z = acc[nt][q] + (g.bias ? g.bias[c] : 0.f);
      if (g.relu) z = fmaxf(z, 0.f);
      g.out[(size_t)row * g.ldo + c] = g.resid ? g.resid[(size_t)row * g.ldo + c] + z : z;
    }
}

// --------------------------------------------------------------------------------------------
// graph aggregation
// --------------------------------------------------------------------------------------------

// G_i = mean over the incident edges of E (64 columns).
__global__ void k_gnn_aggregate(GnnGraph g, const float* __restrict__ E, float* G) {
  const int i = blockIdx.x * 4 + (threadIdx.x >> 6), c = threadIdx.x & 63;
  if (i >= g.N) return;
  float s = 0.f;
  for (int q = g.lo_ptr[i]; q < g.lo_ptr[i + 1]; ++q) s += E[(size_t)g.lo_e[q] * kGnnH + c];
  for (int q = g.up_ptr[i]; q < g.up_ptr[i + 1]; ++q) s += E[(size_t)g.up_e[q] * kGnnH + c];
  const int deg = node_degree(g, i);
  G[(size_t)i * kGnnH + c] = deg ? s / deg : 0.f;
}

// dE_e += dG_b / deg_b + dG_a / deg_a (dG with leading dimension ldg).
__global__ void k_gnn_aggregate_bwd(GnnGraph g, const float* __restrict__ dG, int ldg, float* dE) {
  const int e = blockIdx.x * 4 + (threadIdx.x >> 6), c = threadIdx.x & 63;
  if (e >= g.ne) return;
  const int a = g.ea[e], b = g.eb[e];
  const int da = node_degree(g, a), db = node_degree(g, b);
  dE[(size_t)e * kGnnH + c] += dG[(size_t)b * ldg + c] / db + dG[(size_t)a * ldg + c] / da;
}

// dH_i (+)= sum over lower edges (k, i) of dX[e, 0:64] (the h_b part) and over upper edges
// (i, l) of dX[e, 64:128] (the h_a part); dX has 192 columns.
__global__ void k_gnn_scatter_nodes(GnnGraph g, const float* __restrict__ dX, float* dH, int accumulate) {
  const int i = blockIdx.x * 4 + (threadIdx.x >> 6), c = threadIdx.x & 63;
  if (i >= g.N) return;
  float s = 0.f;
  for (int q = g.lo_ptr[i]; q < g.lo_ptr[i + 1]; ++q) s += dX[(size_t)g.lo_e[q] * 3 * kGnnH + c];
  for (int q = g.up_ptr[i]; q < g.up_ptr[i + 1]; ++q) s += dX[(size_t)g.up_e[q] * 3 * kGnnH + kGnnH + c];
  float* o = dH + (size_t)i * kGnnH + c;
  *o = accumulate ? *o + s : s;
}

// dZ = dOut * (A > 0)
__global__ void k_relu_mask(const float* __restrict__ dOut, const float* __restrict__ A, float* dZ, long n) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t < n) dZ[t] = A[t] > 0.f ? dOut[t] : 0.f;
}

// dst[r, c] += src[r * lds + off + c] for 64 columns
__global__ void k_add_cols(float* dst, const float* __restrict__ src, int lds, int off, long rows) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= rows * kGnnH) return;
  const long r = t / kGnnH;
  const int c = (int)(t - r * kGnnH);
  dst[t] += src[r * lds + off + c];
}

// --------------------------------------------------------------------------------------------
// edge blocks, probe loss
// --------------------------------------------------------------------------------------------

__device__ __forceinline__ void edge_block(const float* x, const float* cf, float (&E)[36]) {
  const float c0 = 1.f + cf[0], c1 = 1.f + cf[1], c2 = 1.f + cf[2];
#pragma unroll
  for (int t = 0; t < 36; ++t) E[t] = -c0 * x[t] + c1 * x[36 + t] + c2 * x[72 + t];
}

__global__ void k_gnn_build_E(int ne, const float* __restrict__ xe, const float* __restrict__ coef, float* Em) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  float E[36];
  edge_block(xe + (size_t)e * kGnnEdgeIn, coef + (size_t)e * 3, E);
#pragma unroll
  for (int t = 0; t < 36; ++t) Em[(size_t)e * 36 + t] = E[t];
}

// PCG blocks by block id: E_e C_a^-1.
__global__ void k_gnn_pcg_blocks(GnnGraph g, const float* __restrict__ xe, const float* __restrict__ coef,
                                 const float* __restrict__ cinv, float* ehat) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.ne) return;
  float E[36];
  edge_block(xe + (size_t)e * kGnnEdgeIn, coef + (size_t)e * 3, E);
  const float* Ca = cinv + (size_t)g.ea[e] * 36;
  float* o = ehat + (size_t)g.eblk[e] * 36;
  for (int r = 0; r < 6; ++r)
    for (int c = 0; c < 6; ++c) {
      float v = 0.f;
      for (int k = c; k < 6; ++k) v += E[r * 6 + k] * Ca[k * 6 + c];
      o[r * 6 + c] = v;
    }
}

// Rademacher probe entry (fmix32 finaliser of MurmurHash3 over the entry index and the seed).
__host__ __device__ __forceinline__ float probe_sign(uint32_t seed, uint32_t idx) {
  uint32_t h = idx * 0x9E3779B1u + seed;
  h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13; h *= 0xC2B2AE35u; h ^= h >> 16;
  return (h & 1u) ? 1.f : -1.f;
}

// Probe vectors are [N][6][P] floats.
__global__ void k_probe_fill(float* z, long n, uint32_t seed) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t < n) z[t] = probe_sign(seed, (uint32_t)t);
}

// out_a = in_a + sum over upper edges (a, b) of E_e^T in_b
__global__ void k_apply_IEt(GnnGraph g, const float* __restrict__ Em, const float* __restrict__ in, float* out) {
  const int i = blockIdx.x * (blockDim.x / kGnnProbes) + threadIdx.x / kGnnProbes, p = threadIdx.x % kGnnProbes;
  if (i >= g.N) return;
  float acc[6];
  for (int r = 0; r < 6; ++r) acc[r] = in[((size_t)i * 6 + r) * kGnnProbes + p];
  for (int q = g.up_ptr[i]; q < g.up_ptr[i + 1]; ++q) {
    const int e = g.up_e[q], b = g.eb[e];
    const float* E = Em + (size_t)e * 36;
    float v[6];
    for (int k = 0; k < 6; ++k) v[k] = in[((size_t)b * 6 + k) * kGnnProbes + p];
    for (int r = 0; r < 6; ++r)
      for (int k = 0; k < 6; ++k) acc[r] += E[k * 6 + r] * v[k];
  }
  for (int r = 0; r < 6; ++r) out[((size_t)i * 6 + r) * kGnnProbes + p] = acc[r];
}

// out_b = in_b + sum over lower edges (a, b) of E_e in_a
__global__ void k_apply_IE(GnnGraph g, const float* __restrict__ Em, const float* __restrict__ in, float* out) {
  const int i = blockIdx.x * (blockDim.x / kGnnProbes) + threadIdx.x / kGnnProbes, p = threadIdx.x % kGnnProbes;
  if (i >= g.N) return;
  float acc[6];
  for (int r = 0; r < 6; ++r) acc[r] = in[((size_t)i * 6 + r) * kGnnProbes + p];
  for (int q = g.lo_ptr[i]; q < g.lo_ptr[i + 1]; ++q) {
    const int e = g.lo_e[q], a = g.ea[e];
    const float* E = Em + (size_t)e * 36;
    float v[6];
    for (int k = 0; k < 6; ++k) v[k] = in[((size_t)a * 6 + k) * kGnnProbes + p];
    for (int r = 0; r < 6; ++r)
      for (int k = 0; k < 6; ++k) acc[r] += E[r * 6 + k] * v[k];
  }
  for (int r = 0; r < 6; ++r) out[((size_t)i * 6 + r) * kGnnProbes + p] = acc[r];
}

// out = S^ in = in + F in (lower edges) + F^T in (upper edges)
__global__ void k_apply_Shat(GnnGraph g, const float* __restrict__ xe, const float* __restrict__ in, float* out) {
  const int i = blockIdx.x * (blockDim.x / kGnnProbes) + threadIdx.x / kGnnProbes, p = threadIdx.x % kGnnProbes;
  if (i >= g.N) return;
  float acc[6];
  for (int r = 0; r < 6; ++r) acc[r] = in[((size_t)i * 6 + r) * kGnnProbes + p];
  for (int q = g.lo_ptr[i]; q < g.lo_ptr[i + 1]; ++q) {
    const int e = g.lo_e[q], a = g.ea[e];
    const float* F = xe + (size_t)e * kGnnEdgeIn;
    float v[6];
    for (int k = 0; k < 6; ++k) v[k] = in[((size_t)a * 6 + k) * kGnnProbes + p];
    for (int r = 0; r < 6; ++r)
      for (int k = 0; k < 6; ++k) acc[r] += F[r * 6 + k] * v[k];
  }
  for (int q = g.up_ptr[i]; q < g.up_ptr[i + 1]; ++q) {
    const int e = g.up_e[q], b = g.eb[e];
    const float* F = xe + (size_t)e * kGnnEdgeIn;
    float v[6];
    for (int k = 0; k < 6; ++k) v[k] = in[((size_t)b * 6 + k) * kGnnProbes + p];
    for (int r = 0; r < 6; ++r)
      for (int k = 0; k < 6; ++k) acc[r] += F[k * 6 + r] * v[k];
  }
  for (int r = 0; r < 6; ++r) out[((size_t)i * 6 + r) * kGnnProbes + p] = acc[r];
}

// d = 2 scale (p - z); per-block partial sums of (p - z)^2 (FP64).
__global__ void k_probe_resid(const float* __restrict__ P, const float* __restrict__ Z, float* dP, long n, float scale2,
                              double* part) {
  __shared__ double red[256];
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double s = 0.0;
  if (t < n) {
    const float r = P[t] - Z[t];
    dP[t] = scale2 * r;
    s = double(r) * r;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_sum_partials(const double* __restrict__ part, int n, double scale, double* out, int accumulate) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int b = 0; b < n; ++b) s += part[b];
  *out = accumulate ? *out + scale * s : scale * s;
}

// dL/dcoef of each edge from dE_e = sum_p (dp_b w_a^T + z_b dy_a^T).
__global__ void k_gnn_dcoef(GnnGraph g, const float* __restrict__ xe, const float* __restrict__ dP,
                            const float* __restrict__ Wv, const float* __restrict__ Z, const float* __restrict__ dY,
                            float* dcoef) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= g.ne) return;
  const int a = g.ea[e], b = g.eb[e];
  const float* x = xe + (size_t)e * kGnnEdgeIn;
  float d0 = 0.f, d1 = 0.f, d2 = 0.f;
  for (int r = 0; r < 6; ++r) {
    const float* dpb = dP + ((size_t)b * 6 + r) * kGnnProbes;
    const float* zb = Z + ((size_t)b * 6 + r) * kGnnProbes;
    for (int c = 0; c < 6; ++c) {
      const float* wa = Wv + ((size_t)a * 6 + c) * kGnnProbes;
      const float* dya = dY + ((size_t)a * 6 + c) * kGnnProbes;
      float dE = 0.f;
#pragma unroll
      for (int p = 0; p < kGnnProbes; ++p) dE += dpb[p] * wa[p] + zb[p] * dya[p];
      d0 -= dE * x[r * 6 + c];
      d1 += dE * x[36 + r * 6 + c];
      d2 += dE * x[72 + r * 6 + c];
    }
  }
  dcoef[(size_t)e * 3 + 0] = d0;
  dcoef[(size_t)e * 3 + 1] = d1;
  dcoef[(size_t)e * 3 + 2] = d2;
}

__global__ void k_adam(float* w, const float* __restrict__ grad, float* m, float* v, int n, float lr, float b1, float b2,
                       float c1, float c2, float eps) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gq = grad[t];
  const float mq = b1 * m[t] + (1.f - b1) * gq;
  const float vq = b2 * v[t] + (1.f - b2) * gq * gq;
  m[t] = mq;
  v[t] = vq;
  w[t] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}

// W (K x 64 row-major, fp32) -> W^T (64 x Kp, bf16, zero padded)
__global__ void k_pack_bf16(const float* __restrict__ W, int K, int Kp, __nv_bfloat16* Wt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= kGnnH * Kp) return;
  const int n = t / Kp, k = t - n * Kp;
  Wt[t] = __float2bfloat16_rn(k < K ? W[(size_t)k * kGnnH + n] : 0.f);
}

}  // namespace

int gnn_features(const GnnGraph& g, const void* Sb, bool fp64, const int* diag_blk, float* cinv, float* xe, float* xn,
                 int* d_fail, cudaStream_t st) {
  const int N = g.N, ne = g.ne;
  if (reinterpret_cast<uintptr_t>(xe) & 15) return V3DBA_ERR_UNSUPPORTED;   // 16-byte loads of edge rows
  if (fp64) k_gnn_cinv<double><<<cdiv(N, 128), 128, 0, st>>>((const double*)Sb, diag_blk, N, cinv, d_fail);
  else k_gnn_cinv<float><<<cdiv(N, 128), 128, 0, st>>>((const float*)Sb, diag_blk, N, cinv, d_fail);
  V3DBA_LAUNCH_CHECK();
  if (ne > 0) {
    if (fp64) k_gnn_edge_norm<double><<<cdiv(ne, 128), 128, 0, st>>>((const double*)Sb, g, cinv, xe);
    else k_gnn_edge_norm<float><<<cdiv(ne, 128), 128, 0, st>>>((const float*)Sb, g, cinv, xe);
    V3DBA_LAUNCH_CHECK();
    k_gnn_two_hop<<<cdiv(ne, 4), dim3(72, 4), 0, st>>>(g, xe);
    V3DBA_LAUNCH_CHECK();
  }
  k_gnn_node_feat<<<cdiv(N, 8), 256, 0, st>>>(g, xe, xn);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

}  // namespace v3dba

using namespace v3dba;

// ---------------------------------------------------------------------------------------------
// model
// ---------------------------------------------------------------------------------------------

namespace {

template <typename T>
int grow(T** p, size_t& cap, size_t need) {
  if (need <= cap && *p) return V3DBA_OK;
  cudaFree(*p);
  *p = nullptr;
  cap = std::max<size_t>(need, 1);
  V3DBA_CUDA_TRY(cudaMalloc(p, sizeof(T) * cap));
  return V3DBA_OK;
}

}  // namespace

struct v3dba_precond_model_s {
  float* w = nullptr;
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  int adam_t = 0;
  __nv_bfloat16* wt = nullptr;   // packed W^T of the 64-wide layers (ein, m0-2, h0-1)
  bool packed = false;
  cudaStream_t st = nullptr;
  // activations (training keeps every layer), grown to the largest system seen
  size_t cpart = 0, cdpart = 0;
  size_t c_e[24] = {}, c_n[24] = {};   // capacities of the buffers below
  float* E[4] = {};      // edge states e0..e3 [ne x 64]
  float* A[3] = {};      // relu outputs of the edge updates
  float* H[3] = {};      // node states h0..h2 [N x 64]
  float* Gm[2] = {};     // mean aggregates
  float* Cn[2] = {};     // relu outputs of the node updates
  float* coef = nullptr; // [ne x 3]
  float* dcoef = nullptr;
  float* Em = nullptr;   // [ne x 36]
  float* dE = nullptr;
  float* dZ = nullptr;
  float* dX = nullptr;   // [ne x 192]
  float* dH = nullptr;
  float* dZn = nullptr;
  float* dXn = nullptr;  // [N x 128]
  float* vz = nullptr;   // probe vectors [N x 6 x P]
  float* vy = nullptr;
  float* vw = nullptr;
  float* vp = nullptr;
  float* vdp = nullptr;
  float* vdw = nullptr;
  float* vdy = nullptr;
  float* part = nullptr;
  double* dpart = nullptr;
  double* d_loss = nullptr;
};

namespace {

constexpr int kPackK[6] = {112, 192, 192, 192, 128, 128};   // ein, m0, m1, m2, h0, h1

size_t pack_offset(int layer) {
  size_t o = 0;
  for (int l = 0; l < layer; ++l) o += (size_t)kGnnH * kPackK[l];
  return o;
}

int model_reserve(v3dba_precond_model_s* m, int N, int ne) {
  int rc;
  size_t k = 0;
  auto ge = [&](float** p, size_t per) { return grow(p, m->c_e[k++], (size_t)std::max(ne, 1) * per); };
  for (int l = 0; l < 4; ++l) if ((rc = ge(&m->E[l], kGnnH))) return rc;
  for (int l = 0; l < 3; ++l) if ((rc = ge(&m->A[l], kGnnH))) return rc;
  if ((rc = ge(&m->coef, 3)) || (rc = ge(&m->dcoef, 3)) || (rc = ge(&m->Em, 36)) || (rc = ge(&m->dE, kGnnH)) ||
      (rc = ge(&m->dZ, kGnnH)) || (rc = ge(&m->dX, 3 * kGnnH)))
    return rc;
  k = 0;
  auto gn = [&](float** p, size_t per) { return grow(p, m->c_n[k++], (size_t)std::max(N, 1) * per); };
  for (int l = 0; l < 3; ++l) if ((rc = gn(&m->H[l], kGnnH))) return rc;
  for (int l = 0; l < 2; ++l) if ((rc = gn(&m->Gm[l], kGnnH)) || (rc = gn(&m->Cn[l], kGnnH))) return rc;
  if ((rc = gn(&m->dH, kGnnH)) || (rc = gn(&m->dZn, kGnnH)) || (rc = gn(&m->dXn, 2 * kGnnH))) return rc;
  const size_t pv = 6 * kGnnProbes;
  if ((rc = gn(&m->vz, pv)) || (rc = gn(&m->vy, pv)) || (rc = gn(&m->vw, pv)) || (rc = gn(&m->vp, pv)) ||
      (rc = gn(&m->vdp, pv)) || (rc = gn(&m->vdw, pv)) || (rc = gn(&m->vdy, pv)))
    return rc;
  const size_t nblk = (size_t)cdiv(std::max(ne, N), kWgRows);
  if ((rc = grow(&m->part, m->cpart, nblk * (3 * kGnnH + 1) * kGnnH))) return rc;
  const size_t nv = (size_t)N * 6 * kGnnProbes;
  if ((rc = grow(&m->dpart, m->cdpart, (size_t)cdiv(nv, 256) + 1))) return rc;
  return V3DBA_OK;
}

Seg seg(const float* src, const int* idx, int ld, int width) {
  Seg s;
  s.src = src; s.idx = idx; s.ld = ld; s.width = width;
  return s;
}

int rowgemm(cudaStream_t st, int rows, std::initializer_list<Seg> in, const float* W, int wk, int wn, const float* bias,
            int Nout, float* out, int ldo, const float* resid, float* act_out, bool relu) {
  if (rows <= 0) return V3DBA_OK;
  RowGemm g;
  g.rows = rows;
  for (const Seg& s : in) { g.seg[g.nseg++] = s; g.K += s.width; }
  g.W = W; g.wk = wk; g.wn = wn; g.bias = bias; g.Nout = Nout; g.out = out; g.ldo = ldo; g.resid = resid;
  g.act_out = act_out; g.relu = relu ? 1 : 0;
  const size_t smem = sizeof(float) * ((size_t)kRgRows * (g.K + 1) + (size_t)g.K * Nout);
  k_rowgemm<<<cdiv(rows, kRgRows), 256, smem, st>>>(g);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

int rowgemm_bf16(v3dba_precond_model_s* m, cudaStream_t st, int rows, std::initializer_list<Seg> in, int layer,
                 const float* bias, float* out, const float* resid, bool relu) {
  if (rows <= 0) return V3DBA_OK;
  RowGemm g;
  g.rows = rows;
  for (const Seg& s : in) {
    // the kernel stages its inputs with 16-byte loads
    if ((reinterpret_cast<uintptr_t>(s.src) & 15) || (s.ld & 3) || (s.width & 3)) return V3DBA_ERR_UNSUPPORTED;
    g.seg[g.nseg++] = s;
    g.K += s.width;
  }
  g.bias = bias; g.Nout = kGnnH; g.out = out; g.ldo = kGnnH; g.resid = resid; g.relu = relu ? 1 : 0;
  const int Kp = kPackK[layer];
  const size_t smem = sizeof(__nv_bfloat16) * 2 * 64 * (size_t)(Kp + 8);
  k_rowgemm_bf16<<<cdiv(rows, 64), 128, smem, st>>>(g, m->wt + pack_offset(layer), Kp);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

int wgrad(v3dba_precond_model_s* m, cudaStream_t st, int rows, std::initializer_list<Seg> in, const float* D, int Nout,
          float* grad) {
  WGrad g;
  g.rows = rows;
  for (const Seg& s : in) { g.seg[g.nseg++] = s; g.K += s.width; }
  g.Nout = Nout; g.D = D; g.part = m->part;
  const int nout = (g.K + 1) * Nout;
  if (rows <= 0) {
    V3DBA_CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(float) * nout, st));
    return V3DBA_OK;
  }
  const int nblk = cdiv(rows, kWgRows);
  const size_t smem = sizeof(float) * (32 * (size_t)(g.K + 1) + 32 * (size_t)Nout);
  k_wgrad<<<nblk, 256, smem, st>>>(g);
  V3DBA_LAUNCH_CHECK();
  k_wgrad_reduce<<<cdiv(nout, 256), 256, 0, st>>>(m->part, nblk, nout, grad);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

int set_smem_limits() {
  static bool done = false;
  if (done) return V3DBA_OK;
  V3DBA_CUDA_TRY(cudaFuncSetAttribute(k_rowgemm, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
  V3DBA_CUDA_TRY(cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  V3DBA_CUDA_TRY(cudaFuncSetAttribute(k_rowgemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
  done = true;
  return V3DBA_OK;
}

int pack_weights(v3dba_precond_model_s* m, cudaStream_t st) {
  if (m->packed) return V3DBA_OK;
  const int off[6] = {GnnLayout::ein, GnnLayout::m0, GnnLayout::m0 + GnnLayout::msz, GnnLayout::m0 + 2 * GnnLayout::msz,
                      GnnLayout::h0, GnnLayout::h0 + GnnLayout::hsz};
  const int K[6] = {kGnnEdgeIn, 3 * kGnnH, 3 * kGnnH, 3 * kGnnH, 2 * kGnnH, 2 * kGnnH};
  for (int l = 0; l < 6; ++l) {
    k_pack_bf16<<<cdiv(kGnnH * kPackK[l], 256), 256, 0, st>>>(m->w + off[l], K[l], kPackK[l], m->wt + pack_offset(l));
    V3DBA_LAUNCH_CHECK();
  }
  m->packed = true;
  return V3DBA_OK;
}

// Forward pass over one system.  train: FP32 kernels keeping every activation; else BF16
// inference of the 64-wide layers with in-place state updates (each block reads only its own
// rows of the state it updates).  Writes m->coef.
int gnn_forward(v3dba_precond_model_s* m, const GnnGraph& g, const float* xe, const float* xn, bool train,
                cudaStream_t st) {
  int rc;
  if ((rc = set_smem_limits()) || (rc = model_reserve(m, g.N, g.ne))) return rc;
  const int N = g.N, ne = g.ne;
  const float* w = m->w;
  auto W = [&](int off) { return w + off; };
  auto Bm = [&](int off, int K, int Nout) { return w + off + (size_t)K * Nout; };
  const int msz = GnnLayout::msz, hsz = GnnLayout::hsz;
  if (!train && (rc = pack_weights(m, st))) return rc;
  float* Ecur = m->E[0];
  float* Hcur = m->H[0];
  if (train) {
    if ((rc = rowgemm(st, ne, {seg(xe, nullptr, kGnnEdgeIn, kGnnEdgeIn)}, W(GnnLayout::ein), kGnnH, 1,
                      Bm(GnnLayout::ein, kGnnEdgeIn, kGnnH), kGnnH, m->E[0], kGnnH, nullptr, nullptr, true)))
      return rc;
  } else if ((rc = rowgemm_bf16(m, st, ne, {seg(xe, nullptr, kGnnEdgeIn, kGnnEdgeIn)}, 0,
                                Bm(GnnLayout::ein, kGnnEdgeIn, kGnnH), m->E[0], nullptr, true))) {
    return rc;
  }
  if ((rc = rowgemm(st, N, {seg(xn, nullptr, kGnnNodeIn, kGnnNodeIn)}, W(GnnLayout::nin), kGnnH, 1,
                    Bm(GnnLayout::nin, kGnnNodeIn, kGnnH), kGnnH, m->H[0], kGnnH, nullptr, nullptr, true)))
    return rc;
  for (int l = 0; l < 3; ++l) {
    const int mo = GnnLayout::m0 + l * msz;
    float* Enext = train ? m->E[l + 1] : Ecur;
    const Seg in_m[3] = {seg(Hcur, g.eb, kGnnH, kGnnH), seg(Hcur, g.ea, kGnnH, kGnnH), seg(Ecur, nullptr, kGnnH, kGnnH)};
    if (train) {
      if ((rc = rowgemm(st, ne, {in_m[0], in_m[1], in_m[2]}, W(mo), kGnnH, 1, Bm(mo, 3 * kGnnH, kGnnH), kGnnH, Enext,
                        kGnnH, Ecur, m->A[l], true)))
        return rc;
    } else if ((rc = rowgemm_bf16(m, st, ne, {in_m[0], in_m[1], in_m[2]}, 1 + l, Bm(mo, 3 * kGnnH, kGnnH), Enext, Ecur,
                                  true))) {
      return rc;
    }
    Ecur = Enext;
    if (l < 2) {
      const int ho = GnnLayout::h0 + l * hsz;
      if (N > 0) {
        k_gnn_aggregate<<<cdiv(N, 4), 256, 0, st>>>(g, Ecur, m->Gm[l]);
        V3DBA_LAUNCH_CHECK();
      }
      float* Hnext = train ? m->H[l + 1] : Hcur;
      const Seg in_h[2] = {seg(Hcur, nullptr, kGnnH, kGnnH), seg(m->Gm[l], nullptr, kGnnH, kGnnH)};
      if (train) {
        if ((rc = rowgemm(st, N, {in_h[0], in_h[1]}, W(ho), kGnnH, 1, Bm(ho, 2 * kGnnH, kGnnH), kGnnH, Hnext, kGnnH,
                          Hcur, m->Cn[l], true)))
          return rc;
      } else if ((rc = rowgemm_bf16(m, st, N, {in_h[0], in_h[1]}, 4 + l, Bm(ho, 2 * kGnnH, kGnnH), Hnext, Hcur, true))) {
        return rc;
      }
      Hcur = Hnext;
    }
  }
  return rowgemm(st, ne, {seg(Ecur, nullptr, kGnnH, kGnnH)}, W(GnnLayout::out), kGnnOut, 1,
                 Bm(GnnLayout::out, kGnnH, kGnnOut), kGnnOut, m->coef, kGnnOut, nullptr, nullptr, false);
}

// Probe loss of the current coefficients and dL/dcoef; loss (scaled) to *d_out (accumulate).
int probe_loss(v3dba_precond_model_s* m, const GnnGraph& g, const float* xe, uint32_t seed, double* d_out,
               bool accumulate, cudaStream_t st) {
  const int N = g.N, ne = g.ne;
  const long nv = (long)N * 6 * kGnnProbes;
  if (ne > 0) {
    k_gnn_build_E<<<cdiv(ne, 128), 128, 0, st>>>(ne, xe, m->coef, m->Em);
    V3DBA_LAUNCH_CHECK();
  }
  k_probe_fill<<<cdiv(nv, 256), 256, 0, st>>>(m->vz, nv, seed);
  V3DBA_LAUNCH_CHECK();
  const int nb = cdiv(N, 256 / kGnnProbes);
  k_apply_IEt<<<nb, 256, 0, st>>>(g, m->Em, m->vz, m->vy);
  V3DBA_LAUNCH_CHECK();
  k_apply_Shat<<<nb, 256, 0, st>>>(g, xe, m->vy, m->vw);
  V3DBA_LAUNCH_CHECK();
  k_apply_IE<<<nb, 256, 0, st>>>(g, m->Em, m->vw, m->vp);
  V3DBA_LAUNCH_CHECK();
  const double scale = 1.0 / ((double)N * 6 * kGnnProbes);
  const int np = cdiv(nv, 256);
  k_probe_resid<<<np, 256, 0, st>>>(m->vp, m->vz, m->vdp, nv, (float)(2.0 * scale), m->dpart);
  V3DBA_LAUNCH_CHECK();
  k_sum_partials<<<1, 32, 0, st>>>(m->dpart, np, scale, d_out, accumulate ? 1 : 0);
  V3DBA_LAUNCH_CHECK();
  k_apply_IEt<<<nb, 256, 0, st>>>(g, m->Em, m->vdp, m->vdw);
  V3DBA_LAUNCH_CHECK();
  k_apply_Shat<<<nb, 256, 0, st>>>(g, xe, m->vdw, m->vdy);
  V3DBA_LAUNCH_CHECK();
  if (ne > 0) {
    k_gnn_dcoef<<<cdiv(ne, 128), 128, 0, st>>>(g, xe, m->vdp, m->vw, m->vz, m->vdy, m->dcoef);
    V3DBA_LAUNCH_CHECK();
  }
  return V3DBA_OK;
}

// Backward pass from m->dcoef into m->grad (every weight written).
int gnn_backward(v3dba_precond_model_s* m, const GnnGraph& g, const float* xe, const float* xn, cudaStream_t st) {
  const int N = g.N, ne = g.ne;
  const int msz = GnnLayout::msz, hsz = GnnLayout::hsz;
  float* gr = m->grad;
  int rc;
  auto mask = [&](const float* dOut, const float* A, float* dZ, long n) -> int {
    if (n <= 0) return V3DBA_OK;
    k_relu_mask<<<cdiv(n, 256), 256, 0, st>>>(dOut, A, dZ, n);
    V3DBA_LAUNCH_CHECK();
    return V3DBA_OK;
  };
  // output layer
  if ((rc = wgrad(m, st, ne, {seg(m->E[3], nullptr, kGnnH, kGnnH)}, m->dcoef, kGnnOut, gr + GnnLayout::out))) return rc;
  if ((rc = rowgemm(st, ne, {seg(m->dcoef, nullptr, kGnnOut, kGnnOut)}, m->w + GnnLayout::out, 1, kGnnOut, nullptr,
                    kGnnH, m->dE, kGnnH, nullptr, nullptr, false)))
    return rc;
  for (int l = 2; l >= 0; --l) {
    if (l < 2) {
      const int ho = GnnLayout::h0 + l * hsz;
      if ((rc = mask(m->dH, m->Cn[l], m->dZn, (long)N * kGnnH))) return rc;
      if ((rc = wgrad(m, st, N, {seg(m->H[l], nullptr, kGnnH, kGnnH), seg(m->Gm[l], nullptr, kGnnH, kGnnH)}, m->dZn,
                      kGnnH, gr + ho)))
        return rc;
      if ((rc = rowgemm(st, N, {seg(m->dZn, nullptr, kGnnH, kGnnH)}, m->w + ho, 1, kGnnH, nullptr, 2 * kGnnH, m->dXn,
                        2 * kGnnH, nullptr, nullptr, false)))
        return rc;
      if (N > 0) {
        k_add_cols<<<cdiv((long)N * kGnnH, 256), 256, 0, st>>>(m->dH, m->dXn, 2 * kGnnH, 0, N);
        V3DBA_LAUNCH_CHECK();
      }
      if (ne > 0) {
        k_gnn_aggregate_bwd<<<cdiv(ne, 4), 256, 0, st>>>(g, m->dXn + kGnnH, 2 * kGnnH, m->dE);
        V3DBA_LAUNCH_CHECK();
      }
    }
    const int mo = GnnLayout::m0 + l * msz;
    if ((rc = mask(m->dE, m->A[l], m->dZ, (long)ne * kGnnH))) return rc;
    if ((rc = wgrad(m, st, ne,
                    {seg(m->H[l], g.eb, kGnnH, kGnnH), seg(m->H[l], g.ea, kGnnH, kGnnH), seg(m->E[l], nullptr, kGnnH, kGnnH)},
                    m->dZ, kGnnH, gr + mo)))
      return rc;
    if ((rc = rowgemm(st, ne, {seg(m->dZ, nullptr, kGnnH, kGnnH)}, m->w + mo, 1, kGnnH, nullptr, 3 * kGnnH, m->dX,
                      3 * kGnnH, nullptr, nullptr, false)))
      return rc;
    if (ne > 0) {
      k_add_cols<<<cdiv((long)ne * kGnnH, 256), 256, 0, st>>>(m->dE, m->dX, 3 * kGnnH, 2 * kGnnH, ne);
      V3DBA_LAUNCH_CHECK();
    }
    if (N > 0) {
      k_gnn_scatter_nodes<<<cdiv(N, 4), 256, 0, st>>>(g, m->dX, m->dH, l < 2 ? 1 : 0);
      V3DBA_LAUNCH_CHECK();
    }
  }
  // inputs
  if ((rc = mask(m->dE, m->E[0], m->dZ, (long)ne * kGnnH))) return rc;
  if ((rc = wgrad(m, st, ne, {seg(xe, nullptr, kGnnEdgeIn, kGnnEdgeIn)}, m->dZ, kGnnH, gr + GnnLayout::ein))) return rc;
  if ((rc = mask(m->dH, m->H[0], m->dZn, (long)N * kGnnH))) return rc;
  return wgrad(m, st, N, {seg(xn, nullptr, kGnnNodeIn, kGnnNodeIn)}, m->dZn, kGnnH, gr + GnnLayout::nin);
}

}  // namespace

namespace v3dba {

int gnn_precond_blocks(v3dba_precond_model m, const GnnGraph& g, const float* cinv, const float* xe, const float* xn,
                       float* ehat, cudaStream_t st) {
  int rc;
  if ((rc = gnn_forward(m, g, xe, xn, false, st))) return rc;
  if (g.ne > 0) {
    k_gnn_pcg_blocks<<<cdiv(g.ne, 128), 128, 0, st>>>(g, xe, m->coef, cinv, ehat);
    V3DBA_LAUNCH_CHECK();
  }
  return V3DBA_OK;
}

}  // namespace v3dba

// ---------------------------------------------------------------------------------------------
// system sets
// ---------------------------------------------------------------------------------------------

namespace {

struct PrecondSystem {
  int N = 0, nb = 0;
  GnnGraph g;
  PcgState ps;      // pattern, FP64 blocks, vectors
  float* cinv = nullptr;
  float* xe = nullptr;
  float* xn = nullptr;
  float* ehat = nullptr;
  double* frames = nullptr;   // camera frames of the gauge space
  double* rhs = nullptr;      // the LM's reduced right-hand side (captured systems only)
  double* x = nullptr;
  int* fail = nullptr;
};

void system_free(PrecondSystem& s) {
  gnn_graph_free(s.g);
  pcg_free(s.ps);
  cudaFree(s.cinv); cudaFree(s.xe); cudaFree(s.xn); cudaFree(s.ehat); cudaFree(s.frames); cudaFree(s.rhs);
  cudaFree(s.x);
  cudaFree(s.fail);
  s = PrecondSystem();
}

}  // namespace

struct v3dba_precond_set_s {
  std::vector<PrecondSystem> sys;
  cudaStream_t st = nullptr;
};

namespace v3dba {
// accessors into the opaque handle (solver.cu)
DevState& handle_state(v3dba_handle h);
cudaStream_t handle_stream(v3dba_handle h);
const std::vector<int>& handle_blk_i(v3dba_handle h);
const std::vector<int>& handle_blk_l(v3dba_handle h);
int handle_use_pcg(v3dba_handle h);
PcgState& handle_pcg(v3dba_handle h);
const double* handle_cur_R(v3dba_handle h);
const double* handle_cur_T(v3dba_handle h);
}  // namespace v3dba

namespace {

// Allocates a system over the block pattern and fills its FP64 blocks with `fill`.  The set
// keeps FP64 blocks: at the small damping of a converged LM run FP32 rounding of S exceeds the
// gauge eigenvalues (the LM itself then runs FP64 blocks), so FP32 copies would not be the
// systems the solver meets there.
template <typename Fill>
int system_create(v3dba_precond_set s, int N, const std::vector<int>& b_i, const std::vector<int>& b_l, Fill fill) {
  PrecondSystem ps;
  ps.N = N;
  ps.nb = (int)b_i.size();
  int rc;
  if ((rc = pcg_plan(ps.ps, b_i, b_l, N)) || (rc = pcg_alloc(ps.ps, ps.nb, N, 6)) ||
      (rc = gnn_graph_build(ps.g, N, b_i, b_l))) {
    system_free(ps);
    return rc;
  }
  auto al = [&](auto** p, size_t n) -> int {
    using T = typename std::remove_reference<decltype(**p)>::type;
    V3DBA_CUDA_TRY(cudaMalloc(p, sizeof(T) * std::max<size_t>(n, 1)));
    return V3DBA_OK;
  };
  if ((rc = al(&ps.cinv, (size_t)N * 36)) || (rc = al(&ps.xe, (size_t)ps.g.ne * kGnnEdgeIn)) ||
      (rc = al(&ps.xn, (size_t)N * kGnnNodeIn)) || (rc = al(&ps.ehat, (size_t)ps.nb * 36)) ||
      (rc = al(&ps.x, (size_t)N * 6)) || (rc = al(&ps.fail, 1))) {
    system_free(ps);
    return rc;
  }
  if ((rc = fill(ps))) { system_free(ps); return rc; }
  V3DBA_CUDA_TRY(cudaMemsetAsync(ps.fail, 0, sizeof(int), s->st));
  if ((rc = gnn_features(ps.g, ps.ps.Sb, true, ps.ps.diag_blk, ps.cinv, ps.xe, ps.xn, ps.fail, s->st))) {
    system_free(ps);
    return rc;
  }
  int hfail = 0;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(&hfail, ps.fail, sizeof(int), cudaMemcpyDeviceToHost, s->st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(s->st));
  if (hfail) { system_free(ps); return V3DBA_ERR_INVALID_INPUT; }
  s->sys.push_back(ps);
  return V3DBA_OK;
}

bool valid_index(v3dba_precond_set s, int index) { return s && index >= 0 && index < (int)s->sys.size(); }

}  // namespace

extern "C" {

int v3dba_precond_model_size(void) { return GnnLayout::total; }

int v3dba_precond_model_create(const float* weights, uint32_t seed, v3dba_precond_model* out) {
  if (!out) return V3DBA_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const int n = GnnLayout::total;
  std::vector<float> h(n, 0.f);
  if (weights) {
    std::memcpy(h.data(), weights, sizeof(float) * n);
  } else {
    // uniform(-1/sqrt(K), 1/sqrt(K)) for every [W; b] block; the output layer starts at zero
    std::mt19937 rng(seed);
    auto init = [&](int off, int K, int Nout) {
      std::uniform_real_distribution<float> u(-1.f / std::sqrt((float)K), 1.f / std::sqrt((float)K));
      for (int t = 0; t < (K + 1) * Nout; ++t) h[off + t] = u(rng);
    };
    init(GnnLayout::ein, kGnnEdgeIn, kGnnH);
    init(GnnLayout::nin, kGnnNodeIn, kGnnH);
    for (int l = 0; l < 3; ++l) init(GnnLayout::m0 + l * GnnLayout::msz, 3 * kGnnH, kGnnH);
    for (int l = 0; l < 2; ++l) init(GnnLayout::h0 + l * GnnLayout::hsz, 2 * kGnnH, kGnnH);
  }
  for (float v : h)
    if (!std::isfinite(v)) return V3DBA_ERR_INVALID_INPUT;
  auto* m = new v3dba_precond_model_s();
  auto fail = [&](cudaError_t e) {
    if (e != cudaSuccess) { cudaGetLastError(); return true; }
    return false;
  };
  const size_t packed = pack_offset(6);
  if (fail(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking)) || fail(cudaMalloc(&m->w, sizeof(float) * n)) ||
      fail(cudaMalloc(&m->grad, sizeof(float) * n)) || fail(cudaMalloc(&m->adam_m, sizeof(float) * n)) ||
      fail(cudaMalloc(&m->adam_v, sizeof(float) * n)) || fail(cudaMalloc(&m->wt, sizeof(__nv_bfloat16) * packed)) ||
      fail(cudaMalloc(&m->d_loss, sizeof(double) * 2)) ||
      fail(cudaMemcpy(m->w, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice)) ||
      fail(cudaMemset(m->adam_m, 0, sizeof(float) * n)) || fail(cudaMemset(m->adam_v, 0, sizeof(float) * n))) {
    v3dba_precond_model_destroy(m);
    return V3DBA_ERR_CUDA;
  }
  *out = m;
  return V3DBA_OK;
}

int v3dba_precond_model_destroy(v3dba_precond_model m) {
  if (!m) return V3DBA_ERR_INVALID_ARGUMENT;
  if (m->st) cudaStreamSynchronize(m->st);
  float** bufs[] = {&m->w, &m->grad, &m->adam_m, &m->adam_v, &m->coef, &m->dcoef, &m->Em, &m->dE, &m->dZ, &m->dX,
                    &m->dH, &m->dZn, &m->dXn, &m->vz, &m->vy, &m->vw, &m->vp, &m->vdp, &m->vdw, &m->vdy, &m->part};
  for (float** b : bufs) cudaFree(*b);
  for (auto* p : m->E) cudaFree(p);
  for (auto* p : m->A) cudaFree(p);
  for (auto* p : m->H) cudaFree(p);
  for (auto* p : m->Gm) cudaFree(p);
  for (auto* p : m->Cn) cudaFree(p);
  cudaFree(m->wt);
  cudaFree(m->dpart);
  cudaFree(m->d_loss);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
  return V3DBA_OK;
}

int v3dba_precond_model_get_weights(v3dba_precond_model m, float* weights) {
  if (!m || !weights) return V3DBA_ERR_INVALID_ARGUMENT;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(m->st));
  V3DBA_CUDA_TRY(cudaMemcpy(weights, m->w, sizeof(float) * GnnLayout::total, cudaMemcpyDeviceToHost));
  return V3DBA_OK;
}

int v3dba_precond_set_create(v3dba_precond_set* out) {
  if (!out) return V3DBA_ERR_INVALID_ARGUMENT;
  auto* s = new v3dba_precond_set_s();
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete s;
    return V3DBA_ERR_CUDA;
  }
  *out = s;
  return V3DBA_OK;
}

int v3dba_precond_set_destroy(v3dba_precond_set s) {
  if (!s) return V3DBA_ERR_INVALID_ARGUMENT;
  cudaStreamSynchronize(s->st);
  for (auto& p : s->sys) system_free(p);
  cudaStreamDestroy(s->st);
  delete s;
  return V3DBA_OK;
}

int v3dba_precond_set_count(v3dba_precond_set s) { return s ? (int)s->sys.size() : 0; }

int v3dba_precond_set_add_blocks(v3dba_precond_set s, int n_cameras, int n_blocks, const int32_t* blk_i,
                                 const int32_t* blk_l, const double* blocks, const double* R, const double* T) {
  if ((R == nullptr) != (T == nullptr)) return V3DBA_ERR_INVALID_ARGUMENT;
  if (!s || n_cameras <= 0 || n_blocks <= 0 || !blk_i || !blk_l || !blocks) return V3DBA_ERR_INVALID_ARGUMENT;
  std::vector<int> bi(n_blocks), bl(n_blocks);
  std::vector<uint8_t> seen_diag(n_cameras, 0);
  for (int b = 0; b < n_blocks; ++b) {
    bi[b] = blk_i[b];
    bl[b] = blk_l[b];
    if (bi[b] < 0 || bl[b] >= n_cameras || bi[b] > bl[b]) return V3DBA_ERR_INVALID_INPUT;
    if (bi[b] == bl[b]) {
      if (seen_diag[bi[b]]) return V3DBA_ERR_INVALID_INPUT;
      seen_diag[bi[b]] = 1;
    }
  }
  for (int i = 0; i < n_cameras; ++i)
    if (!seen_diag[i]) return V3DBA_ERR_INVALID_INPUT;
  for (size_t t = 0; t < (size_t)n_blocks * 36; ++t)
    if (!std::isfinite(blocks[t])) return V3DBA_ERR_INVALID_INPUT;
  return system_create(s, n_cameras, bi, bl, [&](PrecondSystem& ps) -> int {
    V3DBA_CUDA_TRY(cudaMemcpy(ps.ps.Sb, blocks, sizeof(double) * (size_t)n_blocks * 36, cudaMemcpyHostToDevice));
    if (R) {
      std::vector<double> f((size_t)n_cameras * 12);
      for (int i = 0; i < n_cameras; ++i) {
        for (int q = 0; q < 9; ++q) f[(size_t)i * 12 + q] = R[(size_t)i * 9 + q];
        for (int q = 0; q < 3; ++q) f[(size_t)i * 12 + 9 + q] = T[(size_t)i * 3 + q];
      }
      V3DBA_CUDA_TRY(cudaMalloc(&ps.frames, sizeof(double) * f.size()));
      V3DBA_CUDA_TRY(cudaMemcpy(ps.frames, f.data(), sizeof(double) * f.size(), cudaMemcpyHostToDevice));
    }
    return V3DBA_OK;
  });
}

int v3dba_precond_set_capture(v3dba_precond_set s, v3dba_handle h, double lambda) {
  if (!s || !h || !(lambda >= 0.0)) return V3DBA_ERR_INVALID_ARGUMENT;
  DevState& ds = handle_state(h);
  if (ds.d.DA != 6 || ds.d.DC != 0) return V3DBA_ERR_UNSUPPORTED;
  int rc;
  if ((rc = handle_use_pcg(h))) return rc;
  const LmOps* ops = lm_ops(ds.d.model, ds.d.DA, ds.d.DC, true);
  if (!ops) return V3DBA_ERR_UNSUPPORTED;
  cudaStream_t hst = handle_stream(h);
  if ((rc = ops->relinearize(ds, false, 0.0, hst))) return rc;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(ds.d_lambda, &lambda, sizeof(double), cudaMemcpyHostToDevice, hst));
  V3DBA_CUDA_TRY(cudaMemsetAsync(ds.d_fail, 0, sizeof(int), hst));
  if ((rc = ops->build_reduced(ds, hst))) return rc;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(hst));
  const void* src = handle_pcg(h).Sb;
  const double* src_rhs = handle_pcg(h).b;
  const size_t bytes = sizeof(double) * (size_t)ds.nb * 36;
  const int N = ds.d.N, n_fixed = ds.d.nnA;
  const double* R = handle_cur_R(h);
  const double* T = handle_cur_T(h);
  return system_create(s, N, handle_blk_i(h), handle_blk_l(h), [&](PrecondSystem& ps) -> int {
    V3DBA_CUDA_TRY(cudaMemcpy(ps.ps.Sb, src, bytes, cudaMemcpyDeviceToDevice));
    V3DBA_CUDA_TRY(cudaMalloc(&ps.rhs, sizeof(double) * 6 * (size_t)std::max(N, 1)));
    V3DBA_CUDA_TRY(cudaMemcpy(ps.rhs, src_rhs, sizeof(double) * 6 * (size_t)N, cudaMemcpyDeviceToDevice));
    V3DBA_CUDA_TRY(cudaMalloc(&ps.frames, sizeof(double) * 12 * (size_t)std::max(N, 1)));
    int rc2 = gauge_frames(R, T, N, n_fixed, ps.frames, s->st);
    if (rc2) return rc2;
    V3DBA_CUDA_TRY(cudaStreamSynchronize(s->st));
    return V3DBA_OK;
  });
}

int v3dba_precond_set_info(v3dba_precond_set s, int index, int* n_cameras, int* n_edges) {
  if (!valid_index(s, index)) return V3DBA_ERR_INVALID_ARGUMENT;
  if (n_cameras) *n_cameras = s->sys[index].N;
  if (n_edges) *n_edges = s->sys[index].g.ne;
  return V3DBA_OK;
}

int v3dba_precond_set_features(v3dba_precond_set s, int index, int32_t* edge_a, int32_t* edge_b, float* edge_feat,
                               float* node_feat, float* cinv) {
  if (!valid_index(s, index)) return V3DBA_ERR_INVALID_ARGUMENT;
  const PrecondSystem& p = s->sys[index];
  V3DBA_CUDA_TRY(cudaStreamSynchronize(s->st));
  const size_t ne = p.g.ne, N = p.N;
  if (edge_a && ne) V3DBA_CUDA_TRY(cudaMemcpy(edge_a, p.g.ea, sizeof(int) * ne, cudaMemcpyDeviceToHost));
  if (edge_b && ne) V3DBA_CUDA_TRY(cudaMemcpy(edge_b, p.g.eb, sizeof(int) * ne, cudaMemcpyDeviceToHost));
  if (edge_feat && ne) V3DBA_CUDA_TRY(cudaMemcpy(edge_feat, p.xe, sizeof(float) * ne * kGnnEdgeIn, cudaMemcpyDeviceToHost));
  if (node_feat) V3DBA_CUDA_TRY(cudaMemcpy(node_feat, p.xn, sizeof(float) * N * kGnnNodeIn, cudaMemcpyDeviceToHost));
  if (cinv) V3DBA_CUDA_TRY(cudaMemcpy(cinv, p.cinv, sizeof(float) * N * 36, cudaMemcpyDeviceToHost));
  return V3DBA_OK;
}

int v3dba_precond_loss_grad(v3dba_precond_model m, v3dba_precond_set s, int index, uint32_t probe_seed, double* loss,
                            float* grad) {
  if (!m || !valid_index(s, index)) return V3DBA_ERR_INVALID_ARGUMENT;
  const PrecondSystem& p = s->sys[index];
  V3DBA_CUDA_TRY(cudaStreamSynchronize(s->st));
  int rc;
  if ((rc = gnn_forward(m, p.g, p.xe, p.xn, true, m->st)) ||
      (rc = probe_loss(m, p.g, p.xe, probe_seed, m->d_loss, false, m->st)) ||
      (rc = gnn_backward(m, p.g, p.xe, p.xn, m->st)))
    return rc;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(m->st));
  if (loss) V3DBA_CUDA_TRY(cudaMemcpy(loss, m->d_loss, sizeof(double), cudaMemcpyDeviceToHost));
  if (grad) V3DBA_CUDA_TRY(cudaMemcpy(grad, m->grad, sizeof(float) * GnnLayout::total, cudaMemcpyDeviceToHost));
  return V3DBA_OK;
}

int v3dba_precond_coefficients(v3dba_precond_model m, v3dba_precond_set s, int index, int bf16, float* coeffs) {
  if (!m || !valid_index(s, index) || !coeffs) return V3DBA_ERR_INVALID_ARGUMENT;
  const PrecondSystem& p = s->sys[index];
  V3DBA_CUDA_TRY(cudaStreamSynchronize(s->st));
  int rc;
  if ((rc = gnn_forward(m, p.g, p.xe, p.xn, bf16 == 0, m->st))) return rc;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(m->st));
  if (p.g.ne) V3DBA_CUDA_TRY(cudaMemcpy(coeffs, m->coef, sizeof(float) * 3 * p.g.ne, cudaMemcpyDeviceToHost));
  return V3DBA_OK;
}

int v3dba_precond_train(v3dba_precond_model m, v3dba_precond_set s, int epochs, double learning_rate, uint32_t seed,
                        double* loss_per_epoch) {
  if (!m || !s || epochs < 0 || !(learning_rate > 0.0) || s->sys.empty()) return V3DBA_ERR_INVALID_ARGUMENT;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(s->st));
  std::mt19937 rng(seed);
  std::vector<int> order(s->sys.size());
  std::iota(order.begin(), order.end(), 0);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int n = GnnLayout::total;
  m->packed = false;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(order.begin(), order.end(), rng);
    V3DBA_CUDA_TRY(cudaMemsetAsync(m->d_loss + 1, 0, sizeof(double), m->st));
    for (int idx : order) {
      const PrecondSystem& p = s->sys[idx];
      int rc;
      if ((rc = gnn_forward(m, p.g, p.xe, p.xn, true, m->st)) ||
          (rc = probe_loss(m, p.g, p.xe, (uint32_t)rng(), m->d_loss + 1, true, m->st)) ||
          (rc = gnn_backward(m, p.g, p.xe, p.xn, m->st)))
        return rc;
      ++m->adam_t;
      const float c1 = 1.f - std::pow(b1, (float)m->adam_t), c2 = 1.f - std::pow(b2, (float)m->adam_t);
      k_adam<<<cdiv(n, 256), 256, 0, m->st>>>(m->w, m->grad, m->adam_m, m->adam_v, n, (float)learning_rate, b1, b2, c1,
                                              c2, eps);
      V3DBA_LAUNCH_CHECK();
    }
    double tot = 0.0;
    V3DBA_CUDA_TRY(cudaMemcpyAsync(&tot, m->d_loss + 1, sizeof(double), cudaMemcpyDeviceToHost, m->st));
    V3DBA_CUDA_TRY(cudaStreamSynchronize(m->st));
    if (loss_per_epoch) loss_per_epoch[ep] = tot / (double)s->sys.size();
    if (!std::isfinite(tot)) return V3DBA_ERR_NUMERICAL;
  }
  return V3DBA_OK;
}

int v3dba_precond_pcg_iterations(v3dba_precond_model m, v3dba_precond_set s, int index, double tol, int max_iter,
                                 uint32_t rhs_seed, int* iters, double* ms) {
  if (!valid_index(s, index) || !(tol > 0.0) || max_iter <= 0 || !iters) return V3DBA_ERR_INVALID_ARGUMENT;
  PrecondSystem& p = s->sys[index];
  const int n = p.N * 6;
  cudaStream_t st = s->st;
  std::vector<double> b(n);
  if (rhs_seed == 0 && p.rhs) {
    V3DBA_CUDA_TRY(cudaMemcpyAsync(p.ps.b, p.rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  } else {
    std::mt19937_64 rng(rhs_seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (double& v : b) v = nd(rng);
    V3DBA_CUDA_TRY(cudaMemcpyAsync(p.ps.b, b.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st));
  }
  int rc;
  cudaEvent_t e0, e1;
  V3DBA_CUDA_TRY(cudaEventCreate(&e0));
  V3DBA_CUDA_TRY(cudaEventCreate(&e1));
  auto elapsed = [&](double* out) -> int {
    float t = 0.f;
    V3DBA_CUDA_TRY(cudaEventSynchronize(e1));
    V3DBA_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
    if (out) *out = t;
    return V3DBA_OK;
  };
  if (ms)
    for (int v = 0; v < 5; ++v) ms[v] = -1.0;
  if (m) {
    V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
    V3DBA_CUDA_TRY(cudaEventRecord(e0, m->st));
    if ((rc = gnn_precond_blocks(m, p.g, p.cinv, p.xe, p.xn, p.ehat, m->st))) return rc;
    V3DBA_CUDA_TRY(cudaEventRecord(e1, m->st));
    if ((rc = elapsed(ms ? ms + 4 : nullptr))) return rc;
  }
  for (int v = 0; v < 4; ++v) {
    iters[v] = -1;
    const bool learned = v >= 2, gauge = (v & 1) != 0;
    if ((learned && !m) || (gauge && !p.frames)) continue;
    PcgPrecond P;
    if (learned) { P.cinv = p.cinv; P.ehat = p.ehat; }
    if (gauge) P.frames = p.frames;
    V3DBA_CUDA_TRY(cudaMemsetAsync(p.fail, 0, sizeof(int), st));
    V3DBA_CUDA_TRY(cudaEventRecord(e0, st));
    if ((rc = pcg_solve_precond(p.ps, p.N, 6, true, tol, max_iter, p.x, p.fail, st, P))) return rc;
    V3DBA_CUDA_TRY(cudaEventRecord(e1, st));
    if ((rc = elapsed(ms ? ms + v : nullptr))) return rc;
    int its = 0, fl = 0;
    V3DBA_CUDA_TRY(cudaMemcpyAsync(&its, p.ps.iters, sizeof(int), cudaMemcpyDeviceToHost, st));
    V3DBA_CUDA_TRY(cudaMemcpyAsync(&fl, p.fail, sizeof(int), cudaMemcpyDeviceToHost, st));
    V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
    iters[v] = fl ? max_iter : its;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return V3DBA_OK;
}

}  // extern "C"
