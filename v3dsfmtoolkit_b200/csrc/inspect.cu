// Inspection entry points of the C-ABI: per-observation linearisation in the caller's order,
// the damped reduced camera system, and a standalone tile-sparse Cholesky solve.  They expose
// each stage of the GPU path so that it can be checked against the CPU oracle stage by stage.
#include <algorithm>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "lm.cuh"
#include "model.cuh"

struct v3dba_handle_s;

namespace v3dba {

// Raw (unweighted) residual, Huber weight and Jacobian blocks, written in the caller's order.
template <int MODEL, int DA, int DC>
__global__ void __launch_bounds__(128) k_raw_linearize(DevState s, double* e, double* w, double* A, double* B, double* C) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const Dims& D = s.d;
  if (k >= D.K) return;
  constexpr int DCc = DC > 0 ? DC : 1;
  const int i = s.o_cam[k], j = s.o_pt[k], o = s.o_orig[k];
  Cam cam;
  load_cam<MODEL>(cam, s.cur.R, s.cur.T, s.cur.K, s.cur.dist, i);
  if (MODEL == kModelStereo) load_rig(cam, s.rig, s.o_sub[k]);
  const double X[3] = {s.cur.X[3 * j], s.cur.X[3 * j + 1], s.cur.X[3 * j + 2]};
  double ee[2], a[2][DA], b[2][3], c[2][DCc];
  linearize_obs<MODEL, DA, DC>(cam, X, s.o_meas[2 * k], s.o_meas[2 * k + 1], D.mode, D.cached_ar, ee, a, b, c);
  if (e) { e[2 * o] = ee[0]; e[2 * o + 1] = ee[1]; }
  if (w) w[o] = huber_weight(D.thr, ee);
  for (int r = 0; r < 2; ++r) {
    if (A) for (int q = 0; q < DA; ++q) A[((size_t)o * 2 + r) * DA + q] = a[r][q];
    if (B) for (int q = 0; q < 3; ++q) B[((size_t)o * 2 + r) * 3 + q] = b[r][q];
    if (C && DC > 0) for (int q = 0; q < DC; ++q) C[((size_t)o * 2 + r) * DC + q] = c[r][q];
  }
}

int launch_raw_linearize(DevState& s, double* e, double* w, double* A, double* B, double* C, cudaStream_t st) {
  const int g = (std::max(s.d.K, 1) + 127) / 128;
  const Dims& D = s.d;
#define RL(M_, A_, C_) k_raw_linearize<M_, A_, C_><<<g, 128, 0, st>>>(s, e, w, A, B, C)
  if (D.model == kModelStd) RL(kModelStd, 6, 0);
  else if (D.model == kModelStereo) RL(kModelStereo, 6, 0);
  else if (D.model == kModelCommon) {
    switch (D.DC) {
      case 0: RL(kModelCommon, 6, 0); break;
      case 1: RL(kModelCommon, 6, 1); break;
      case 3: RL(kModelCommon, 6, 3); break;
      case 5: RL(kModelCommon, 6, 5); break;
      case 7: RL(kModelCommon, 6, 7); break;
      default: return V3DBA_ERR_UNSUPPORTED;
    }
  } else {
    switch (D.DA) {
      case 6: RL(kModelVarying, 6, 0); break;
      case 7: RL(kModelVarying, 7, 0); break;
      case 9: RL(kModelVarying, 9, 0); break;
      case 11: RL(kModelVarying, 11, 0); break;
      case 13: RL(kModelVarying, 13, 0); break;
      default: return V3DBA_ERR_UNSUPPORTED;
    }
  }
#undef RL
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

}  // namespace v3dba

using namespace v3dba;

// accessors into the opaque handle (defined in solver.cu)
namespace v3dba {
int handle_use_dense(v3dba_handle h);
DevState& handle_state(v3dba_handle h);
TileChol& handle_chol(v3dba_handle h);
cudaStream_t handle_stream(v3dba_handle h);
}  // namespace v3dba

namespace {

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  template <typename T>
  int alloc(size_t n) {
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) { cudaGetLastError(); p = nullptr; return V3DBA_ERR_OUT_OF_MEMORY; }
    return V3DBA_OK;
  }
  template <typename T> T* as() { return static_cast<T*>(p); }
};

}  // namespace

extern "C" int v3dba_linearize(v3dba_handle h, int precision, double* e, double* w, double* A, double* B,
                               double* C, double* ga, double* gb, double* gc) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  DevState& s = handle_state(h);
  cudaStream_t st = handle_stream(h);
  const Dims& D = s.d;
  const int K = D.K;
  DevBuf de, dw, dA, dB, dC;
  int rc;
  if (e && (rc = de.alloc<double>(2 * (size_t)K))) return rc;
  if (w && (rc = dw.alloc<double>(K))) return rc;
  if (A && (rc = dA.alloc<double>(2 * (size_t)K * D.DA))) return rc;
  if (B && (rc = dB.alloc<double>(6 * (size_t)K))) return rc;
  if (C && D.DC && (rc = dC.alloc<double>(2 * (size_t)K * D.DC))) return rc;
  if ((rc = launch_raw_linearize(s, de.as<double>(), dw.as<double>(), dA.as<double>(), dB.as<double>(),
                                 dC.as<double>(), st)))
    return rc;
  if (ga || gb || gc) {
    const LmOps* ops = lm_ops(D.model, D.DA, D.DC, precision == V3DBA_PRECISION_FP64);
    if (!ops) return V3DBA_ERR_UNSUPPORTED;
    if ((rc = ops->relinearize(s, false, 0.0, st))) return rc;
  }
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  if (e) V3DBA_CUDA_TRY(cudaMemcpy(e, de.p, sizeof(double) * 2 * K, cudaMemcpyDeviceToHost));
  if (w) V3DBA_CUDA_TRY(cudaMemcpy(w, dw.p, sizeof(double) * K, cudaMemcpyDeviceToHost));
  if (A) V3DBA_CUDA_TRY(cudaMemcpy(A, dA.p, sizeof(double) * 2 * K * D.DA, cudaMemcpyDeviceToHost));
  if (B) V3DBA_CUDA_TRY(cudaMemcpy(B, dB.p, sizeof(double) * 6 * K, cudaMemcpyDeviceToHost));
  if (C && D.DC) V3DBA_CUDA_TRY(cudaMemcpy(C, dC.p, sizeof(double) * 2 * K * D.DC, cudaMemcpyDeviceToHost));
  const int SG = (D.DA + 1) & ~1;
  if (ga) {
    std::vector<double> t((size_t)std::max(D.N, 1) * SG);
    V3DBA_CUDA_TRY(cudaMemcpy(t.data(), s.c_ga, sizeof(double) * D.N * SG, cudaMemcpyDeviceToHost));
    for (int i = 0; i < D.N; ++i)
      for (int a = 0; a < D.DA; ++a) ga[(size_t)i * D.DA + a] = t[(size_t)i * SG + a];
  }
  if (gb) {
    std::vector<double> t((size_t)std::max(D.M, 1) * 4);
    V3DBA_CUDA_TRY(cudaMemcpy(t.data(), s.p_gb, sizeof(double) * D.M * 4, cudaMemcpyDeviceToHost));
    for (int j = 0; j < D.M; ++j)
      for (int b = 0; b < 3; ++b) gb[(size_t)j * 3 + b] = t[(size_t)j * 4 + b];
  }
  if (gc && D.DC) V3DBA_CUDA_TRY(cudaMemcpy(gc, s.g_gc, sizeof(double) * D.DC, cudaMemcpyDeviceToHost));
  return V3DBA_OK;
}

extern "C" int v3dba_reduced_system(v3dba_handle h, int precision, double lambda, double* S, double* rhs) {
  if (!h || !S || !rhs) return V3DBA_ERR_INVALID_ARGUMENT;
  int rc0 = handle_use_dense(h);
  if (rc0) return rc0;
  DevState& s = handle_state(h);
  TileChol& tc = handle_chol(h);
  cudaStream_t st = handle_stream(h);
  const Dims& D = s.d;
  const LmOps* ops = lm_ops(D.model, D.DA, D.DC, precision == V3DBA_PRECISION_FP64);
  if (!ops) return V3DBA_ERR_UNSUPPORTED;
  int rc;
  if ((rc = ops->relinearize(s, false, 0.0, st))) return rc;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(s.d_lambda, &lambda, sizeof(double), cudaMemcpyHostToDevice, st));
  V3DBA_CUDA_TRY(cudaMemsetAsync(s.d_fail, 0, sizeof(int), st));
  if ((rc = tile_chol_zero(tc, s.S, s.rhs, st))) return rc;
  if ((rc = ops->build_reduced(s, st))) return rc;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  const int n = s.n;
  std::vector<double> full((size_t)s.ld * s.n_pad);
  V3DBA_CUDA_TRY(cudaMemcpy(full.data(), s.S, sizeof(double) * full.size(), cudaMemcpyDeviceToHost));
  for (int r = 0; r < n; ++r)
    for (int c = 0; c <= r; ++c) {
      const double v = full[(size_t)c * s.ld + r];
      S[(size_t)r * n + c] = v;
      S[(size_t)c * n + r] = v;
    }
  for (int c = 0; c < n; ++c) rhs[c] = full[(size_t)c * s.ld + s.n_pad];
  return V3DBA_OK;
}

extern "C" int v3dba_dense_cholesky_solve(int n, const double* S, const double* rhs, double* x, int* fail) {
  if (n <= 0 || !S || !rhs || !x || !fail) return V3DBA_ERR_INVALID_ARGUMENT;
  TileChol tc;
  const int nt = (n + TileChol::TB - 1) / TileChol::TB;
  std::vector<uint8_t> nz((size_t)nt * nt, 0);
  // tile pattern of the lower triangle of S
  for (int r = 0; r < n; ++r)
    for (int c = 0; c <= r; ++c)
      if (S[(size_t)r * n + c] != 0.0) nz[(size_t)(r / 64) * nt + c / 64] = 1;
  int rc = tile_chol_plan(tc, n, nz);
  if (rc) { tile_chol_free(tc); return rc; }
  std::vector<double> full((size_t)tc.ld * tc.n_pad, 0.0);
  for (int c = 0; c < n; ++c) {
    for (int r = c; r < n; ++r) full[(size_t)c * tc.ld + r] = S[(size_t)r * n + c];
    full[(size_t)c * tc.ld + tc.n_pad] = rhs[c];
  }
  for (int d = n; d < tc.n_pad; ++d) full[(size_t)d * tc.ld + d] = 1.0;
  DevBuf dS, dx, df;
  if ((rc = dS.alloc<double>(full.size())) || (rc = dx.alloc<double>(tc.n_pad)) || (rc = df.alloc<int>(1))) {
    tile_chol_free(tc);
    return rc;
  }
  cudaMemcpy(dS.p, full.data(), sizeof(double) * full.size(), cudaMemcpyHostToDevice);
  cudaMemset(df.p, 0, sizeof(int));
  rc = tile_chol_solve(tc, dS.as<double>(), dx.as<double>(), df.as<int>(), 0);
  if (rc == V3DBA_OK) {
    cudaError_t e1 = cudaDeviceSynchronize();
    if (e1 != cudaSuccess) rc = V3DBA_ERR_CUDA;
  }
  if (rc == V3DBA_OK) {
    cudaMemcpy(x, dx.p, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(fail, df.p, sizeof(int), cudaMemcpyDeviceToHost);
  }
  tile_chol_free(tc);
  return rc;
}

// Benchmark support: the tile Cholesky factor + solve of one dense SPD system (row-major, host),
// timed alone.  The system is uploaded once; every repetition restores the factorised matrix
// from that copy (not timed) and times one solve with CUDA events on the launching stream.
// trace (host, may be NULL): the phase timestamps (globaltimer, ns) of the last repetition of
// the level kernel, (2 * n_levels + 2) slots per cluster rank, slot-major; *trace_len receives
// the number written (0 when the column kernel ran).
extern "C" int v3dba_dense_cholesky_profile(int n, const double* S, const double* rhs, int reps, double* ms,
                                            double* x, int* fail, unsigned long long* trace, int trace_cap,
                                            int* trace_len, int* ranks) {
  if (n <= 0 || !S || !rhs || reps <= 0 || !ms || !x || !fail) return V3DBA_ERR_INVALID_ARGUMENT;
  TileChol tc;
  const int nt = (n + TileChol::TB - 1) / TileChol::TB;
  std::vector<uint8_t> nz((size_t)nt * nt, 0);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c <= r; ++c)
      if (S[(size_t)r * n + c] != 0.0) nz[(size_t)(r / 64) * nt + c / 64] = 1;
  int rc = tile_chol_plan(tc, n, nz);
  if (rc) { tile_chol_free(tc); return rc; }
  std::vector<double> full((size_t)tc.ld * tc.n_pad, 0.0);
  for (int c = 0; c < n; ++c) {
    for (int r = c; r < n; ++r) full[(size_t)c * tc.ld + r] = S[(size_t)r * n + c];
    full[(size_t)c * tc.ld + tc.n_pad] = rhs[c];
  }
  for (int d = n; d < tc.n_pad; ++d) full[(size_t)d * tc.ld + d] = 1.0;
  const size_t slots = tc.levels ? (size_t)(2 * tc.n_levels + 2) * tc.lv_ranks : 0;
  DevBuf d0, dS, dx, df, dt;
  if ((rc = d0.alloc<double>(full.size())) || (rc = dS.alloc<double>(full.size())) ||
      (rc = dx.alloc<double>(tc.n_pad)) || (rc = df.alloc<int>(1)) ||
      (rc = dt.alloc<unsigned long long>(std::max<size_t>(slots, 1)))) {
    tile_chol_free(tc);
    return rc;
  }
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    tile_chol_free(tc);
    return V3DBA_ERR_CUDA;
  }
  cudaMemcpy(d0.p, full.data(), sizeof(double) * full.size(), cudaMemcpyHostToDevice);
  double total = 0.0;
  for (int r = 0; r < reps && rc == V3DBA_OK; ++r) {
    cudaMemcpyAsync(dS.p, d0.p, sizeof(double) * full.size(), cudaMemcpyDeviceToDevice, st);
    cudaMemsetAsync(df.p, 0, sizeof(int), st);
    cudaEventRecord(e0, st);
    rc = tc.levels ? chol_levels_solve(tc, dS.as<double>(), dx.as<double>(), df.as<int>(), st,
                                       r == reps - 1 ? dt.as<unsigned long long>() : nullptr)
                   : tile_chol_solve(tc, dS.as<double>(), dx.as<double>(), df.as<int>(), st);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = V3DBA_ERR_CUDA;
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    total += t;
  }
  if (rc == V3DBA_OK) {
    *ms = total / reps;
    cudaMemcpy(x, dx.p, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(fail, df.p, sizeof(int), cudaMemcpyDeviceToHost);
    const size_t w = trace ? std::min<size_t>(slots, (size_t)std::max(trace_cap, 0)) : 0;
    if (w) cudaMemcpy(trace, dt.p, sizeof(unsigned long long) * w, cudaMemcpyDeviceToHost);
    if (trace_len) *trace_len = (int)w;
    if (ranks) *ranks = tc.levels ? tc.lv_ranks : 0;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  tile_chol_free(tc);
  return rc;
}

// The structure built by v3dba_create: sizes always; every array pointer that is not NULL
// receives its array (o_orig, c_ptr, c_obs [K], [N+1], [K]; b_i, b_l [nb], b_ptr [nb+1];
// pr_k, pr_m [P]).
extern "C" int v3dba_structure(v3dba_handle h, int64_t* n_pairs, int* n_blocks, int* o_orig, int* c_ptr, int* c_obs,
                               int* b_i, int* b_l, int* b_ptr, int* pr_k, int* pr_m) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  DevState& s = handle_state(h);
  V3DBA_CUDA_TRY(cudaStreamSynchronize(handle_stream(h)));
  const size_t K = s.d.K, N = s.d.N, nb = s.nb, P = (size_t)s.P;
  if (n_pairs) *n_pairs = s.P;
  if (n_blocks) *n_blocks = s.nb;
  auto get = [](int* dst, const int* src, size_t n) -> int {
    if (dst && n) V3DBA_CUDA_TRY(cudaMemcpy(dst, src, sizeof(int) * n, cudaMemcpyDeviceToHost));
    return V3DBA_OK;
  };
  int rc;
  if ((rc = get(o_orig, s.o_orig, K)) || (rc = get(c_ptr, s.c_ptr, N + 1)) || (rc = get(c_obs, s.c_obs, K)) ||
      (rc = get(b_i, s.b_i, nb)) || (rc = get(b_l, s.b_l, nb)) || (rc = get(b_ptr, s.b_ptr, nb + 1)) ||
      (rc = get(pr_k, s.pr_k, P)) || (rc = get(pr_m, s.pr_m, P)))
    return rc;
  return V3DBA_OK;
}
