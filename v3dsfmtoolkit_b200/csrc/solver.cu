// Host side of the C-ABI: problem validation, device layout, structure analysis and the LM
// driver.  The driver restates SparseLevenbergOptimizer::minimize
// (V3D/src/Math/v3d_optimization.cpp:719-1250) and the lambda schedule of
// LevenbergOptimizerCommon (V3D/include/Math/v3d_optimization.h:38-59); every numeric step runs
// on the GPU, the host only reads back three or four FP64 scalars per LM iteration to take the
// accept / reject decision with the reference's exact tests.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "common.cuh"
#include "lm.cuh"
#include "model.cuh"
#include "precond.cuh"
#include "structure.cuh"

namespace v3dba {

static std::atomic<uint64_t> g_launches{0};
void note_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

size_t partial_doubles(const DevState& s);

}  // namespace v3dba

using namespace v3dba;

struct v3dba_handle_s {
  DevState s;
  TileChol chol;
  PcgState pcg;
  std::vector<int> blk_i, blk_l;   // camera-pair blocks (host copy)
  std::vector<uint8_t> tile_nz;    // tile pattern of the dense reduced system
  bool dense_ready = false;
  double* S_dense = nullptr;
  double* x_dense = nullptr;
  double* x_pcg = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double param_length = 0.0;
  double lambda = 1e-3;   // LevenbergOptimizerCommon ctor default (v3d_optimization.h:29)
  double nu = 2.0;        // _nu (v3d_optimization.h:31)
  double* h_scalars = nullptr;   // pinned readback area
  std::vector<void*> allocs;
  size_t nK = 0, nD = 0;
  // learned preconditioner and gauge space (PCG solver): attached model, camera graph, inputs
  v3dba_precond_model precond = nullptr;
  bool gnn_ready = false;
  GnnGraph gnn;
  float* gnn_cinv = nullptr;
  float* gnn_xe = nullptr;
  float* gnn_xn = nullptr;
  float* gnn_ehat = nullptr;
  int* gnn_fail = nullptr;
  double* gauge_frames = nullptr;   // [N x 12] camera frames of the gauge coarse space
};

namespace {

int dims_of(int model, int mode, int* dA, int* dC) {
  if (model < V3DBA_MODEL_STD || model > V3DBA_MODEL_STEREO) return V3DBA_ERR_INVALID_ARGUMENT;
  if (model == V3DBA_MODEL_STEREO) {   // rig pose (T, omega); intrinsics fixed on the rig cameras
    *dA = 6;
    *dC = 0;
    return V3DBA_OK;
  }
  if (model != V3DBA_MODEL_STD &&
      (mode < V3DBA_FULL_BUNDLE_NO_ROTATIONS || mode > V3DBA_FULL_BUNDLE_RADIAL_TANGENTIAL))
    return V3DBA_ERR_INVALID_ARGUMENT;
  const int ni = (model == V3DBA_MODEL_STD) ? 0 : intrinsic_dim(mode);
  *dA = 6 + (model == V3DBA_MODEL_VARYING ? ni : 0);
  *dC = (model == V3DBA_MODEL_COMMON ? ni : 0);
  return V3DBA_OK;
}


template <typename T>
int dalloc(v3dba_handle h, T** p, size_t count) {
  void* q = nullptr;
  const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
  int rc0 = ensure_pool();
  if (rc0) return rc0;
  if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
  cudaError_t e = cudaMallocAsync(&q, bytes, h->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? V3DBA_ERR_OUT_OF_MEMORY : V3DBA_ERR_CUDA;
  }
  h->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return V3DBA_OK;
}

int alloc_params(v3dba_handle h, ParamSet& P, int N, int M) {
  int rc;
  if ((rc = dalloc(h, &P.K, h->nK))) return rc;
  if ((rc = dalloc(h, &P.R, (size_t)N * 9))) return rc;
  if ((rc = dalloc(h, &P.T, (size_t)N * 3))) return rc;
  if ((rc = dalloc(h, &P.dist, std::max<size_t>(h->nD, 4)))) return rc;
  if ((rc = dalloc(h, &P.X, (size_t)M * 3))) return rc;
  return V3DBA_OK;
}

int copy_params(const ParamSet& dst, const ParamSet& src, const v3dba_handle h, cudaStream_t st) {
  const Dims& D = h->s.d;
  if (h->nK) V3DBA_CUDA_TRY(cudaMemcpyAsync(dst.K, src.K, sizeof(double) * h->nK, cudaMemcpyDeviceToDevice, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(dst.R, src.R, sizeof(double) * 9 * D.N, cudaMemcpyDeviceToDevice, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(dst.T, src.T, sizeof(double) * 3 * D.N, cudaMemcpyDeviceToDevice, st));
  if (h->nD) V3DBA_CUDA_TRY(cudaMemcpyAsync(dst.dist, src.dist, sizeof(double) * h->nD, cudaMemcpyDeviceToDevice, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(dst.X, src.X, sizeof(double) * 3 * D.M, cudaMemcpyDeviceToDevice, st));
  return V3DBA_OK;
}

int upload_params(v3dba_handle h, const ParamSet& P, const double* K, const double* R, const double* T,
                  const double* dist, const double* X) {
  const Dims& D = h->s.d;
  cudaStream_t st = h->stream;
  if (h->nK) V3DBA_CUDA_TRY(cudaMemcpyAsync(P.K, K, sizeof(double) * h->nK, cudaMemcpyHostToDevice, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(P.R, R, sizeof(double) * 9 * D.N, cudaMemcpyHostToDevice, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(P.T, T, sizeof(double) * 3 * D.N, cudaMemcpyHostToDevice, st));
  if (h->nD) V3DBA_CUDA_TRY(cudaMemcpyAsync(P.dist, dist, sizeof(double) * h->nD, cudaMemcpyHostToDevice, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(P.X, X, sizeof(double) * 3 * D.M, cudaMemcpyHostToDevice, st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  return V3DBA_OK;
}

template <typename T>
int upload(v3dba_handle h, T** d, const std::vector<T>& v) {
  int rc = dalloc(h, d, v.size());
  if (rc) return rc;
  if (!v.empty())
    V3DBA_CUDA_TRY(cudaMemcpyAsync(*d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, h->stream));
  return V3DBA_OK;
}

void free_handle(v3dba_handle h) {
  if (!h) return;
  if (h->stream) {
    for (void* p : h->allocs) cudaFreeAsync(p, h->stream);
    cudaStreamSynchronize(h->stream);
  }
  tile_chol_free(h->chol);
  pcg_free(h->pcg);
  gnn_graph_free(h->gnn);
  if (h->h_scalars) cudaFreeHost(h->h_scalars);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

// Dense reduced system (tile Cholesky): allocated on first use.
int use_dense(v3dba_handle h) {
  DevState& s = h->s;
  if (!h->dense_ready) {
    std::vector<uint8_t> nz = h->tile_nz;
    int rc = tile_chol_plan(h->chol, std::max(s.n, 1), nz);
    if (rc) return rc;
    if (!h->S_dense && (rc = dalloc(h, &h->S_dense, (size_t)h->chol.ld * h->chol.n_pad))) return rc;
    if (!h->x_dense && (rc = dalloc(h, &h->x_dense, (size_t)h->chol.n_pad))) return rc;
    h->dense_ready = true;
  }
  s.n_pad = h->chol.n_pad;
  s.ld = h->chol.ld;
  s.S = h->S_dense;
  s.rhs = h->S_dense + s.n_pad;
  s.rhs_stride = s.ld;
  s.x = h->x_dense;
  s.Sb = nullptr;
  s.diag_blk = nullptr;
  return V3DBA_OK;
}

// Block-sparse reduced system (PCG): allocated on first use.
int use_pcg(v3dba_handle h) {
  DevState& s = h->s;
  if (!h->pcg.ready) {
    pcg_free(h->pcg);   // a retry after a failed attempt (out of memory) starts clean
    int rc = pcg_plan(h->pcg, h->blk_i, h->blk_l, s.d.N);
    if (!rc) rc = pcg_alloc(h->pcg, s.nb, s.d.N, s.d.DA);
    if (rc) {
      pcg_free(h->pcg);
      return rc;
    }
  }
  if (!h->x_pcg) {
    const int rc = dalloc(h, &h->x_pcg, (size_t)std::max(s.n, 1));
    if (rc) return rc;
  }
  s.n_pad = s.n;
  s.ld = 1;
  s.S = nullptr;
  s.rhs = h->pcg.b;
  s.rhs_stride = 1;
  s.x = h->x_pcg;
  s.Sb = h->pcg.Sb;
  s.diag_blk = h->pcg.diag_blk;
  return V3DBA_OK;
}

// Gauge frames, and for the learned preconditioner its camera graph and input buffers: built
// on first use.
int use_gnn(v3dba_handle h, bool learned) {
  if (!h->gauge_frames) {
    int rc0 = dalloc(h, &h->gauge_frames, (size_t)std::max(h->s.d.N, 1) * 12);
    if (rc0 || (rc0 = dalloc(h, &h->gnn_fail, 1))) return rc0;
  }
  if (h->gnn_ready || !learned) return V3DBA_OK;
  const int N = h->s.d.N;
  int rc;
  if ((rc = gnn_graph_build(h->gnn, N, h->blk_i, h->blk_l))) return rc;
  const size_t ne = (size_t)std::max(h->gnn.ne, 1);
  if ((rc = dalloc(h, &h->gnn_cinv, (size_t)N * 36)) || (rc = dalloc(h, &h->gnn_xe, ne * kGnnEdgeIn)) ||
      (rc = dalloc(h, &h->gnn_xn, (size_t)N * kGnnNodeIn)) || (rc = dalloc(h, &h->gnn_ehat, (size_t)h->s.nb * 36)))
    return rc;
  h->gnn_ready = true;
  return V3DBA_OK;
}

// Start of a trial: the damping and a cleared failure flag, set on the device in stream order
// (no host-to-device copy on the critical path).
__global__ void k_trial_setup(double lambda, double* __restrict__ d_lambda, int* __restrict__ d_fail) {
  pdl_wait();
  pdl_trigger();
  *d_lambda = lambda;
  *d_fail = 0;
}

// o_sub[k] = subcamera of the caller's observation o_orig[k] (point-major order)
// Sort key of point j for the track-length order: longer tracks first (lengths of at least
// kTrackBuckets - 1 share the first bucket).  Up to kOrderMaxObs observations the linearisation
// takes the points in that order: a warp's tracks are equally long and the last wave holds the
// short ones (sequence200, 375k observations: 70 -> 54 us).  Beyond it the per-observation block
// writes, scattered by the order, go to DRAM instead of L2, and the stored order is faster
// (2,000 cameras / 5.8M observations: 4% per LM step).
constexpr int kTrackBuckets = 64;
constexpr long kOrderMaxObs = 2000000;
__global__ void k_track_keys(const int* __restrict__ p_ptr, int M, int* __restrict__ keys) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < M) keys[j] = kTrackBuckets - 1 - min(p_ptr[j + 1] - p_ptr[j], kTrackBuckets - 1);
}

__global__ void k_gather_sub(const int* __restrict__ sub, const int* __restrict__ orig, int K, int* __restrict__ out) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < K) out[k] = sub[orig[k]];
}

// Work chunks over the camera observation lists and the camera-pair blocks: long lists are cut
// into chunks of 64 observations / 128 pairs, one warp per chunk.
struct Chunks {
  std::vector<int> cc_beg, cc_end, cam_cc_ptr, bc_beg, bc_end, blk_bc_ptr;
};

constexpr int kCamChunk = 64;     // observations per camera work chunk
constexpr int kPairChunk = 128;   // observation pairs per camera-pair work chunk

void build_chunks(const std::vector<int>& c_ptr, const std::vector<int>& b_ptr, int N, Chunks& S) {
  S.cam_cc_ptr.assign(1, 0);
  for (int i = 0; i < N; ++i) {
    for (int b = c_ptr[i]; b < c_ptr[i + 1]; b += kCamChunk) {
      S.cc_beg.push_back(b);
      S.cc_end.push_back(std::min(b + kCamChunk, c_ptr[i + 1]));
    }
    S.cam_cc_ptr.push_back((int)S.cc_beg.size());
  }
  const int nb = (int)b_ptr.size() - 1;
  S.blk_bc_ptr.assign(1, 0);
  for (int b = 0; b < nb; ++b) {
    for (int p = b_ptr[b]; p < b_ptr[b + 1]; p += kPairChunk) {
      S.bc_beg.push_back(p);
      S.bc_end.push_back(std::min(p + kPairChunk, b_ptr[b + 1]));
    }
    S.blk_bc_ptr.push_back((int)S.bc_beg.size());
  }
}

}  // namespace

extern "C" {

void v3dba_default_options(v3dba_options* o) {
  if (!o) return;
  o->tau = 1e-3;
  o->max_iterations = 50;
  o->gradient_threshold = 1e-10;
  o->update_threshold = 1e-10;
  o->verbosity = 0;
  o->precision = V3DBA_PRECISION_MIXED;
  o->solver = V3DBA_SOLVER_AUTO;
  o->pcg_tolerance = 1e-6;
  o->pcg_max_iterations = 500;
  o->stop_cost = 0.0;
  o->mixed_escalation = 1;
  o->preconditioner = V3DBA_PRECOND_BLOCK_JACOBI;
}

int v3dba_dims(int model, int mode, int* dA, int* dC) {
  if (!dA || !dC) return V3DBA_ERR_INVALID_ARGUMENT;
  return dims_of(model, mode, dA, dC);
}

const char* v3dba_error_string(int code) {
  switch (code) {
    case V3DBA_OK: return "ok";
    case V3DBA_ERR_INVALID_ARGUMENT: return "invalid argument";
    case V3DBA_ERR_INVALID_INPUT: return "invalid input (index out of range or non-finite value)";
    case V3DBA_ERR_CUDA: return "CUDA error";
    case V3DBA_ERR_OUT_OF_MEMORY: return "out of device memory";
    case V3DBA_ERR_NO_DEVICE: return "no CUDA device";
    case V3DBA_ERR_UNSUPPORTED: return "unsupported configuration";
    case V3DBA_ERR_TIMEOUT: return "device-side wait timed out";
    case V3DBA_ERR_NUMERICAL: return "training diverged";
  }
  return "unknown error";
}

uint64_t v3dba_launch_count(void) { return g_launches.load(); }

int v3dba_create(const v3dba_problem* p, v3dba_handle* out) {
  if (!p || !out) return V3DBA_ERR_INVALID_ARGUMENT;
  NvtxRange nvtx("v3dba_create");
  PhaseTrace trace("V3DBA_TRACE_CREATE", "v3dba_create");
  *out = nullptr;
  int dA, dC;
  int rc = dims_of(p->model, p->mode, &dA, &dC);
  if (rc) return rc;
  const int N = p->n_cameras, M = p->n_points, K = p->n_measurements;
  const bool stereo = p->model == V3DBA_MODEL_STEREO;
  if (N < 0 || M < 0 || K < 0) return V3DBA_ERR_INVALID_ARGUMENT;
  if ((N > 0 && (!p->R || !p->T || (!stereo && !p->K))) || (M > 0 && !p->X) ||
      (K > 0 && (!p->measurements || !p->view || !p->point)))
    return V3DBA_ERR_INVALID_ARGUMENT;
  if (p->model == V3DBA_MODEL_COMMON && !p->K) return V3DBA_ERR_INVALID_ARGUMENT;
  if ((p->model == V3DBA_MODEL_COMMON || p->model == V3DBA_MODEL_VARYING) && !p->dist)
    return V3DBA_ERR_INVALID_ARGUMENT;
  const int nrig = stereo ? p->n_rig_cameras : 0;
  if (stereo) {
    if (nrig < 0 || (K > 0 && (nrig == 0 || !p->subcamera)) ||
        (nrig > 0 && (!p->rig_K || !p->rig_R || !p->rig_T)))
      return V3DBA_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < K; ++k)
      if (p->subcamera[k] < 0 || p->subcamera[k] >= nrig) return V3DBA_ERR_INVALID_INPUT;
    if (!all_finite(p->rig_K, (size_t)9 * nrig) || !all_finite(p->rig_R, (size_t)9 * nrig) ||
        !all_finite(p->rig_T, (size_t)3 * nrig))
      return V3DBA_ERR_INVALID_INPUT;
    for (int l = 0; l < nrig; ++l)
      if (p->rig_K[9 * l] == 0.0) return V3DBA_ERR_INVALID_INPUT;   // f divides the aspect ratio
  }
  if (!(p->inlier_threshold > 0.0) || !std::isfinite(p->inlier_threshold)) return V3DBA_ERR_INVALID_INPUT;
  for (int k = 0; k < K; ++k)
    if (p->view[k] < 0 || p->view[k] >= N || p->point[k] < 0 || p->point[k] >= M) return V3DBA_ERR_INVALID_INPUT;
  const size_t nK = stereo ? 0 : (p->model == V3DBA_MODEL_COMMON) ? 9 : (size_t)9 * N;
  const size_t nD = (p->model == V3DBA_MODEL_COMMON) ? 4 : (p->model == V3DBA_MODEL_VARYING ? (size_t)4 * N : 0);
  if (!all_finite(p->K, nK) || !all_finite(p->R, (size_t)9 * N) || !all_finite(p->T, (size_t)3 * N) ||
      !all_finite(p->X, (size_t)3 * M) || !all_finite(p->measurements, (size_t)2 * K) ||
      (nD && !all_finite(p->dist, nD)))
    return V3DBA_ERR_INVALID_INPUT;
  if (p->model == V3DBA_MODEL_COMMON && p->K[0] == 0.0) return V3DBA_ERR_INVALID_INPUT;

  trace.mark("validate");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return V3DBA_ERR_NO_DEVICE;
  }

  v3dba_handle h = new (std::nothrow) v3dba_handle_s();
  if (!h) return V3DBA_ERR_OUT_OF_MEMORY;
  h->nK = nK;
  h->nD = nD;
  DevState& s = h->s;
  Dims& D = s.d;
  D.N = N; D.M = M; D.K = K; D.DA = dA; D.DC = dC;
  D.model = p->model; D.mode = (p->model == V3DBA_MODEL_STD || stereo) ? 0 : p->mode;
  D.thr = p->inlier_threshold;
  D.cached_ar = (p->model == V3DBA_MODEL_COMMON) ? p->K[4] / p->K[0] : 1.0;

  // |p| cached at construction over every camera and point (v3d_metricbundle.h:37-45)
  double pl = 0.0;
  for (int i = 0; i < N; ++i)
    pl += p->T[3 * i] * p->T[3 * i] + p->T[3 * i + 1] * p->T[3 * i + 1] + p->T[3 * i + 2] * p->T[3 * i + 2] + 3.0;
  for (int j = 0; j < M; ++j)
    pl += p->X[3 * j] * p->X[3 * j] + p->X[3 * j + 1] * p->X[3 * j + 1] + p->X[3 * j + 2] * p->X[3 * j + 2];
  h->param_length = std::sqrt(pl);

#define TRY(x) do { if ((rc = (x)) != V3DBA_OK) { free_handle(h); return rc; } } while (0)
#define CTRY(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { cudaGetLastError(); free_handle(h); \
    return _e == cudaErrorMemoryAllocation ? V3DBA_ERR_OUT_OF_MEMORY : V3DBA_ERR_CUDA; } } while (0)

  CTRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  CTRY(cudaEventCreate(&h->ev0));
  CTRY(cudaEventCreate(&h->ev1));
  CTRY(cudaMallocHost(&h->h_scalars, 24 * sizeof(double)));

  trace.mark("stream");
  DeviceStructure ds;
  const DevAlloc alloc = [h](void** q, size_t bytes) { return dalloc(h, reinterpret_cast<char**>(q), bytes); };
  TRY(build_structure_device(p, alloc, h->stream, ds));
  s.o_cam = ds.o_cam;
  s.o_pt = ds.o_pt;
  s.o_orig = ds.o_orig;
  s.o_meas = ds.o_meas;
  s.p_ptr = ds.p_ptr;
  s.p_order = nullptr;
  if (M > 0 && (long)K <= kOrderMaxObs) {   // points by descending track length (stable sort)
    int *keys, *kptr;
    TRY(dalloc(h, &s.p_order, (size_t)M));
    TRY(dalloc(h, &keys, (size_t)M));
    TRY(dalloc(h, &kptr, (size_t)kTrackBuckets + 1));
    k_track_keys<<<(M + 255) / 256, 256, 0, h->stream>>>(s.p_ptr, M, keys);
    CTRY(cudaGetLastError());
    TRY(group_by_key_device(keys, M, kTrackBuckets, s.p_order, kptr, h->stream));
  }
  s.c_ptr = ds.c_ptr;
  s.c_obs = ds.c_obs;
  s.nb = (int)ds.h_b_i.size();
  s.P = ds.P;
  s.b_i = ds.b_i;
  s.b_l = ds.b_l;
  s.b_ptr = ds.b_ptr;
  s.pr_k = ds.pr_k;
  s.pr_m = ds.pr_m;
  if (stereo) {   // rig cameras, and the rig camera of every point-major observation
    std::vector<double> rig((size_t)std::max(nrig, 1) * kRigStride, 0.0);
    for (int l = 0; l < nrig; ++l) {
      std::memcpy(&rig[(size_t)l * kRigStride], p->rig_K + 9 * l, 9 * sizeof(double));
      std::memcpy(&rig[(size_t)l * kRigStride + 9], p->rig_R + 9 * l, 9 * sizeof(double));
      std::memcpy(&rig[(size_t)l * kRigStride + 18], p->rig_T + 3 * l, 3 * sizeof(double));
    }
    TRY(upload(h, &s.rig, rig));
    int* sub_in;
    TRY(dalloc(h, &sub_in, (size_t)std::max(K, 1)));
    TRY(dalloc(h, &s.o_sub, (size_t)std::max(K, 1)));
    if (K > 0) {
      CTRY(cudaMemcpyAsync(sub_in, p->subcamera, sizeof(int) * K, cudaMemcpyHostToDevice, h->stream));
      k_gather_sub<<<(K + 255) / 256, 256, 0, h->stream>>>(sub_in, s.o_orig, K, s.o_sub);
      note_launches(1);
      CTRY(cudaPeekAtLastError());
    }
    CTRY(cudaStreamSynchronize(h->stream));   // `rig` must outlive its copy
  }
  trace.mark("structure", h->stream);
  Chunks st;
  build_chunks(ds.h_c_ptr, ds.h_b_ptr, N, st);
  s.nch_cam = (int)st.cc_beg.size();
  s.nch_blk = (int)st.bc_beg.size();
  TRY(upload(h, &s.cc_beg, st.cc_beg));
  TRY(upload(h, &s.cc_end, st.cc_end));
  TRY(upload(h, &s.cam_cc_ptr, st.cam_cc_ptr));
  TRY(upload(h, &s.bc_beg, st.bc_beg));
  TRY(upload(h, &s.bc_end, st.bc_end));
  TRY(upload(h, &s.blk_bc_ptr, st.blk_bc_ptr));
  TRY(dalloc(h, &s.part_cc, (size_t)std::max(s.nch_cam, 1) * camera_chunk_values(dA, dC)));
  TRY(dalloc(h, &s.part_bc, (size_t)std::max(s.nch_blk, 1) * block_chunk_values(dA)));

  trace.mark("chunks", h->stream);
  TRY(alloc_params(h, s.cur, N, M));
  TRY(alloc_params(h, s.trial, N, M));
  TRY(alloc_params(h, s.init, N, M));
  const size_t Kz = std::max(K, 1), Mz = std::max(M, 1), Nz = std::max(N, 1);
  // 8-byte slots per block, sized for the larger (FP32, 4-float vectors) of the two strides that
  // lm_kernels.cu uses for each block
  const int SA = (2 * dA + 3) & ~3, SW = (3 * dA + 3) & ~3, SC = (2 * std::max(dC, 1) + 3) & ~3;
  const int SG = (dA + 1) & ~1, SY = (3 * std::max(dC, 1) + 3) & ~3, SU = (dA * dA + 3) & ~3;
  const int SX = (dA * std::max(dC, 1) + 3) & ~3;
  double* tmp;
  TRY(dalloc(h, &tmp, Kz * SA)); s.o_A = tmp;
  TRY(dalloc(h, &tmp, dC ? Kz * SC : 4)); s.o_C = tmp;
  TRY(dalloc(h, &s.o_W, Kz * SW));   // FP32 blocks
  TRY(dalloc(h, &s.o_T, Kz * SW));
  TRY(dalloc(h, &s.o_B, Kz * 8));    // FP64 blocks
  TRY(dalloc(h, &s.o_ga, Kz * SG));
  TRY(dalloc(h, &s.o_w, Kz));
  TRY(dalloc(h, &tmp, Mz * 8)); s.p_V = tmp;
  TRY(dalloc(h, &tmp, Mz * SY)); s.p_Y = tmp;
  TRY(dalloc(h, &tmp, Mz * 8)); s.p_Vinv = tmp;
  TRY(dalloc(h, &tmp, Mz * SY)); s.p_YV = tmp;
  TRY(dalloc(h, &s.p_gb, Mz * 4));
  TRY(dalloc(h, &s.p_q, Mz * 4));
  TRY(dalloc(h, &tmp, Nz * SU)); s.c_U = tmp;
  TRY(dalloc(h, &tmp, Nz * SX)); s.c_X = tmp;
  TRY(dalloc(h, &s.c_ga, Nz * SG));
  TRY(dalloc(h, &s.g_Z, 64));
  TRY(dalloc(h, &s.g_gc, 8));
  TRY(dalloc(h, &s.d_lambda, 1));
  TRY(dalloc(h, &s.d_relin, 8));   // relinearisation scalars, then the trial's: read back together
  s.d_trial = s.d_relin + 4;
  TRY(dalloc(h, &s.d_fail, 1));
  s.part_cap = partial_doubles(s);
  TRY(dalloc(h, &s.part, s.part_cap));
  CTRY(cudaMemsetAsync(s.g_Z, 0, 64 * sizeof(double), h->stream));
  CTRY(cudaMemsetAsync(s.g_gc, 0, 8 * sizeof(double), h->stream));

  trace.mark("buffers", h->stream);
  // reduced system: n = N*dA + dC.  The dense tiles (Cholesky) or the block arrays (PCG) are
  // allocated on first use; here only the tile pattern is derived from the blocks and border.
  s.n = N * dA + dC;
  {
    const int nt = std::max(1, (s.n + TileChol::TB - 1) / TileChol::TB);
    h->tile_nz.assign((size_t)nt * nt, 0);
    auto mark = [&](int r0, int r1, int c0, int c1) {  // scalar row range x col range, r >= c part
      for (int tr = r0 / 64; tr <= (r1 - 1) / 64; ++tr)
        for (int tcl = c0 / 64; tcl <= (c1 - 1) / 64; ++tcl)
          if (tr >= tcl) h->tile_nz[(size_t)tr * nt + tcl] = 1;
    };
    for (int b = 0; b < s.nb; ++b) mark(ds.h_b_l[b] * dA, ds.h_b_l[b] * dA + dA, ds.h_b_i[b] * dA, ds.h_b_i[b] * dA + dA);
    for (int i = 0; i < N; ++i) {
      mark(i * dA, i * dA + dA, i * dA, i * dA + dA);
      if (dC) mark(N * dA, N * dA + dC, i * dA, i * dA + dA);
    }
    if (dC) mark(N * dA, N * dA + dC, N * dA, N * dA + dC);
  }
  h->blk_i = ds.h_b_i;
  h->blk_l = ds.h_b_l;

  trace.mark("pattern");
  TRY(upload_params(h, s.cur, p->K, p->R, p->T, p->dist, p->X));
  TRY(copy_params(s.init, s.cur, h, h->stream));
  TRY(copy_params(s.trial, s.cur, h, h->stream));
  CTRY(cudaStreamSynchronize(h->stream));
  trace.mark("params");
#undef TRY
#undef CTRY
  *out = h;
  return V3DBA_OK;
}

int v3dba_destroy(v3dba_handle h) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  free_handle(h);
  return V3DBA_OK;
}

int v3dba_set_nonvarying(v3dba_handle h, int nA, int nB, int nC) {
  if (!h || nA < 0 || nB < 0 || nC < 0) return V3DBA_ERR_INVALID_ARGUMENT;
  h->s.d.nnA = std::min(nA, h->s.d.N);
  h->s.d.nnB = std::min(nB, h->s.d.M);
  h->s.d.nnC = std::min(nC, h->s.d.DC);
  return V3DBA_OK;
}

int v3dba_set_lambda(v3dba_handle h, double lambda) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  h->lambda = lambda;
  return V3DBA_OK;
}

int v3dba_set_params(v3dba_handle h, const double* K, const double* R, const double* T, const double* dist,
                     const double* X) {
  if (!h || (h->nK && !K) || !R || !T || !X || (h->nD && !dist)) return V3DBA_ERR_INVALID_ARGUMENT;
  return upload_params(h, h->s.cur, K, R, T, dist, X);
}

int v3dba_get_params(v3dba_handle h, double* K, double* R, double* T, double* dist, double* X) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  const Dims& D = h->s.d;
  const ParamSet& P = h->s.cur;
  cudaStream_t st = h->stream;
  if (K && h->nK) V3DBA_CUDA_TRY(cudaMemcpyAsync(K, P.K, sizeof(double) * h->nK, cudaMemcpyDeviceToHost, st));
  if (R) V3DBA_CUDA_TRY(cudaMemcpyAsync(R, P.R, sizeof(double) * 9 * D.N, cudaMemcpyDeviceToHost, st));
  if (T) V3DBA_CUDA_TRY(cudaMemcpyAsync(T, P.T, sizeof(double) * 3 * D.N, cudaMemcpyDeviceToHost, st));
  if (dist && h->nD) V3DBA_CUDA_TRY(cudaMemcpyAsync(dist, P.dist, sizeof(double) * h->nD, cudaMemcpyDeviceToHost, st));
  if (X) V3DBA_CUDA_TRY(cudaMemcpyAsync(X, P.X, sizeof(double) * 3 * D.M, cudaMemcpyDeviceToHost, st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  return V3DBA_OK;
}

int v3dba_reset_params(v3dba_handle h) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  int rc = copy_params(h->s.cur, h->s.init, h, h->stream);
  if (rc) return rc;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(h->stream));
  h->lambda = 1e-3;
  h->nu = 2.0;
  return V3DBA_OK;
}

int v3dba_cost(v3dba_handle h, double* cost) {
  if (!h || !cost) return V3DBA_ERR_INVALID_ARGUMENT;
  DevState& s = h->s;
  const LmOps* ops = lm_ops(s.d.model, s.d.DA, s.d.DC, true);
  if (!ops) return V3DBA_ERR_UNSUPPORTED;
  int rc = ops->cost(s, s.cur, s.d_trial, h->stream);
  if (rc) return rc;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(h->h_scalars, s.d_trial, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(h->stream));
  *cost = h->h_scalars[0];
  return V3DBA_OK;
}

}  // extern "C"

namespace {

// One damped trial: reduced system at *d_lambda, Cholesky or PCG, back-substitution, trial
// parameters and their cost.  Reads back {new_err, |delta|^2, delta . g, fail, pcg iterations}.
int run_trial(v3dba_handle h, const LmOps* ops, double lambda, bool pcg, int precond, bool fp64,
              const v3dba_options& o, double out[6]) {
  DevState& s = h->s;
  cudaStream_t st = h->stream;
  NvtxRange nvtx_trial("v3dba.trial");
  int rc;
  {
    NvtxRange nvtx("v3dba.reduced_system");
    if (!pcg && !h->chol.h_tiles.empty()) {
      // clearing the reduced system's tiles also sets the damping and the failure flag
      if ((rc = tile_chol_zero_setup(h->chol, s.S, lambda, s.d_lambda, s.d_fail, st))) return rc;
    } else {
      V3DBA_CUDA_TRY(launch_pdl(k_trial_setup, dim3(1), dim3(1), 0, st, lambda, s.d_lambda, s.d_fail));
      V3DBA_LAUNCH_CHECK();
    }
    if ((rc = ops->build_reduced(s, st))) return rc;
  }
  int fallback = 0;
  auto solve = [&]() -> int {
    if (pcg && precond != V3DBA_PRECOND_BLOCK_JACOBI) {
      // learned factor or block-Jacobi + gauge space; plain block-Jacobi re-solves the trial when
      // that breaks down
      const bool learned = precond == V3DBA_PRECOND_LEARNED;
      V3DBA_CUDA_TRY(cudaMemsetAsync(h->gnn_fail, 0, sizeof(int), st));
      if ((rc = gauge_frames(s.cur.R, s.cur.T, s.d.N, s.d.nnA, h->gauge_frames, st))) return rc;
      if (learned &&
          ((rc = gnn_features(h->gnn, s.Sb, fp64, s.diag_blk, h->gnn_cinv, h->gnn_xe, h->gnn_xn, h->gnn_fail, st)) ||
           (rc = gnn_precond_blocks(h->precond, h->gnn, h->gnn_cinv, h->gnn_xe, h->gnn_xn, h->gnn_ehat, st))))
        return rc;
      int ffail = 0;
      V3DBA_CUDA_TRY(cudaMemcpyAsync(&ffail, h->gnn_fail, sizeof(int), cudaMemcpyDeviceToHost, st));
      V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
      int its = 0;
      if (!ffail) {
        PcgPrecond P;
        if (learned) { P.cinv = h->gnn_cinv; P.ehat = h->gnn_ehat; }
        else P.frames = h->gauge_frames;
        if ((rc = pcg_solve_precond(h->pcg, s.d.N, s.d.DA, fp64, o.pcg_tolerance, o.pcg_max_iterations, s.x,
                                    h->gnn_fail, st, P)))
          return rc;
        V3DBA_CUDA_TRY(cudaMemcpyAsync(&its, h->pcg.iters, sizeof(int), cudaMemcpyDeviceToHost, st));
        V3DBA_CUDA_TRY(cudaMemcpyAsync(&ffail, h->gnn_fail, sizeof(int), cudaMemcpyDeviceToHost, st));
        V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
      }
      h->h_scalars[10] = its;
      // an iteration-capped solve is an inexact step, as with block-Jacobi; only a breakdown (a
      // diagonal block that is not positive definite, or p.Ap <= 0) falls back
      if (ffail) {
        fallback = 1;
        if ((rc = pcg_solve(h->pcg, s.d.N, s.d.DA, fp64, o.pcg_tolerance, o.pcg_max_iterations, s.x, s.d_fail, st)))
          return rc;
        V3DBA_CUDA_TRY(cudaMemcpyAsync(h->h_scalars + 9, h->pcg.iters, sizeof(int), cudaMemcpyDeviceToHost, st));
      } else {
        std::memcpy(h->h_scalars + 9, &its, sizeof(int));
      }
    } else if (pcg) {
      if ((rc = pcg_solve(h->pcg, s.d.N, s.d.DA, fp64, o.pcg_tolerance, o.pcg_max_iterations, s.x, s.d_fail, st)))
        return rc;
      V3DBA_CUDA_TRY(cudaMemcpyAsync(h->h_scalars + 9, h->pcg.iters, sizeof(int), cudaMemcpyDeviceToHost, st));
    } else if ((rc = tile_chol_solve(h->chol, s.S, s.x, s.d_fail, st))) {
      return rc;
    }
    return V3DBA_OK;
  };
  {
    NvtxRange nvtx("v3dba.reduced_solve");
    if ((rc = solve())) return rc;
  }
  NvtxRange nvtx_finish("v3dba.backsub_update_cost");
  if ((rc = ops->finish_trial(s, st))) return rc;
  // one copy: the relinearisation scalars (h_scalars[16..18]) and the trial's {new cost, |d|^2,
  // d.g, failure flag} (h_scalars[20..23], the flag stored by k_trial_finalize)
  V3DBA_CUDA_TRY(cudaMemcpyAsync(h->h_scalars + 16, s.d_relin, 8 * sizeof(double), cudaMemcpyDeviceToHost, st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  out[0] = h->h_scalars[20];
  out[1] = h->h_scalars[21];
  out[2] = h->h_scalars[22];
  const int fail = h->h_scalars[23] != 0.0 ? 1 : 0;
  int its = 0;
  if (pcg) std::memcpy(&its, h->h_scalars + 9, sizeof(int));
  out[3] = fail ? 1.0 : 0.0;
  out[4] = its + (fallback ? h->h_scalars[10] : 0.0);   // iterations of a failed attempt count too
  out[5] = fallback;
  return V3DBA_OK;
}

}  // namespace

extern "C" int v3dba_minimize(v3dba_handle h, const v3dba_options* opts, v3dba_result* res) {
  if (!h || !res) return V3DBA_ERR_INVALID_ARGUMENT;
  v3dba_options o;
  if (opts) o = *opts; else v3dba_default_options(&o);
  std::memset(res, 0, sizeof(*res));
  res->status = V3DBA_STATUS_TIMEOUT;
  res->fp64_from_iteration = -1;
  NvtxRange nvtx("v3dba_minimize");
  DevState& s = h->s;
  const Dims& D = s.d;
  bool fp64 = (o.precision == V3DBA_PRECISION_FP64);
  const LmOps* ops64 = lm_ops(D.model, D.DA, D.DC, true);
  const LmOps* ops = lm_ops(D.model, D.DA, D.DC, fp64);
  if (!ops || !ops64) return V3DBA_ERR_UNSUPPORTED;
  bool relinearize_again = false;   // blocks to be rebuilt in FP64 at unchanged parameters
  int solver = o.solver;
  if (solver == V3DBA_SOLVER_AUTO) solver = (s.n <= 4096 || D.DC > 0) ? V3DBA_SOLVER_CHOLESKY : V3DBA_SOLVER_PCG;
  if (solver == V3DBA_SOLVER_PCG && D.DC > 0) return V3DBA_ERR_UNSUPPORTED;
  const bool pcg = solver == V3DBA_SOLVER_PCG;
  const bool learned = pcg && o.preconditioner == V3DBA_PRECOND_LEARNED;
  const bool gauge = pcg && o.preconditioner != V3DBA_PRECOND_BLOCK_JACOBI;
  if (o.preconditioner < V3DBA_PRECOND_BLOCK_JACOBI || o.preconditioner > V3DBA_PRECOND_GAUGE)
    return V3DBA_ERR_INVALID_ARGUMENT;
  if (learned && !h->precond) return V3DBA_ERR_INVALID_ARGUMENT;
  if (gauge && D.DA != 6) return V3DBA_ERR_UNSUPPORTED;
  {
    const int rc0 = pcg ? use_pcg(h) : use_dense(h);
    if (rc0) return rc0;
    if (gauge) {
      const int rc1 = use_gnn(h, learned);
      if (rc1) return rc1;
    }
  }

  const int nvA = D.N - D.nnA, nvB = D.M - D.nnB, nvC = D.DC - D.nnC;
  if (nvA <= 0 && nvB <= 0 && nvC <= 0) {
    res->status = V3DBA_STATUS_CONVERGED;
    res->lambda = h->lambda;
    return V3DBA_OK;
  }
  cudaStream_t st = h->stream;
  V3DBA_CUDA_TRY(cudaEventRecord(h->ev0, st));
  bool compute_derivatives = true;
  double err = 0.0;
  double lambda = h->lambda;
  int it;
  int rc;
  for (it = 0; it < o.max_iterations; ++it) {
    if (o.verbosity >= 2) printf("SparseLevenbergOptimizer: currentIteration: %d\n", it);
    if (relinearize_again && !compute_derivatives) {
      // same parameters, same FP64 cost and gradient; only the block precision changes
      NvtxRange nvtx_relin("v3dba.relinearize");
      if ((rc = ops->relinearize(s, false, o.tau, st))) return rc;
    }
    relinearize_again = false;
    // The relinearisation's cost, gradient maximum and diagonal maximum are read back before the
    // trial: when they end the run (stop cost, gradient) no trial is spent.  (Reading them with
    // the trial's results instead saved no measurable time on the dense path and cost one
    // discarded trial per call, a whole PCG solve on large scenes.)
    bool stop = false;
    auto take_relin = [&]() {
      err = h->h_scalars[16];
      const double gmax = h->h_scalars[17], dmax = h->h_scalars[18];
      if (res->n_relinearizations == 0) res->initial_cost = err;
      res->n_relinearizations++;
      res->cost = err;
      if (o.verbosity >= 1) printf("SparseLevenbergOptimizer: |residual|^2 = %.17g\n", err);
      if (o.verbosity >= 2) printf("SparseLevenbergOptimizer: lambda = %.17g\n", lambda);
      if (o.stop_cost > 0.0 && err <= o.stop_cost) {
        res->reached_stop_cost = 1;
        stop = true;
        return;
      }
      if (gmax < o.gradient_threshold) {   // cpp:857-861
        res->status = V3DBA_STATUS_CONVERGED;
        stop = true;
        return;
      }
      if (it == 0) {
        lambda = o.tau * dmax;             // cpp:981-1052
        if (o.verbosity >= 2) printf("SparseLevenbergOptimizer: initial lambda = %.17g\n", lambda);
      }
    };
    if (compute_derivatives) {
      NvtxRange nvtx_relin("v3dba.relinearize");
      if ((rc = ops->relinearize(s, it == 0, o.tau, st))) return rc;
      V3DBA_CUDA_TRY(cudaMemcpyAsync(h->h_scalars + 16, s.d_relin, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
      V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
      take_relin();
      if (stop) break;
    }
    double t[6];
    if ((rc = run_trial(h, ops, lambda, pcg, pcg ? o.preconditioner : V3DBA_PRECOND_BLOCK_JACOBI, fp64, o, t)))
      return rc;
    res->pcg_iterations += (int)t[4];
    res->pcg_fallbacks += (int)t[5];
    const bool success = t[3] == 0.0;
    double rho = 0.0;
    if (success) {
      const double d2 = t[1];
      if (o.verbosity >= 2) printf("SparseLevenbergOptimizer: ||delta||^2 = %.17g\n", d2);
      if (std::sqrt(d2) < o.update_threshold * (h->param_length + o.update_threshold)) {  // cpp:1154-1159
        res->status = V3DBA_STATUS_SMALL_UPDATE;
        break;
      }
      const double new_err = t[0];
      rho = (err - new_err) / (lambda * d2 + t[2]);   // cpp:1188-1210
      if (o.verbosity >= 2)
        printf("SparseLevenbergOptimizer: |new residual|^2 = %.17g rho = %.17g\n", new_err, rho);
    } else if (o.verbosity >= 2) {
      printf("SparseLevenbergOptimizer: LDL decomposition failed. Increasing lambda.\n");
    }
    if (!fp64 && o.mixed_escalation && (!success || rho < 0.1)) {
      // the quadratic model is no longer trusted: stop adding FP32 rounding to it
      fp64 = true;
      ops = ops64;
      res->fp64_from_iteration = it;
      relinearize_again = true;
      if (o.verbosity >= 2) printf("v3dba: normal-equation blocks switched to FP64 at iteration %d\n", it);
    }
    if (success && rho > 0.0) {
      std::swap(s.cur, s.trial);           // accept
      const double r = 2.0 * rho - 1.0;
      lambda *= std::max(1.0 / 3.0, 1.0 - r * r * r);
      if (lambda < 1e-10) lambda = 1e-10;
      h->nu = 2.0;
      compute_derivatives = true;
    } else {
      res->n_rejected++;
      lambda *= h->nu;
      h->nu *= 2.0;
      compute_derivatives = false;
    }
  }
  V3DBA_CUDA_TRY(cudaEventRecord(h->ev1, st));
  V3DBA_CUDA_TRY(cudaEventSynchronize(h->ev1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  res->device_ms = ms;
  res->iterations = it;
  res->lambda = lambda;
  h->lambda = lambda;
  if (o.verbosity >= 2) printf("Leaving SparseLevenbergOptimizer::minimize().\n");
  return V3DBA_OK;
}

extern "C" int v3dba_profile_stages(v3dba_handle h, int precision, int reps, double* ms) {
  if (!h || !ms || reps <= 0) return V3DBA_ERR_INVALID_ARGUMENT;
  DevState& s = h->s;
  const Dims& D = s.d;
  const LmOps* ops = lm_ops(D.model, D.DA, D.DC, precision == V3DBA_PRECISION_FP64);
  if (!ops) return V3DBA_ERR_UNSUPPORTED;
  cudaStream_t st = h->stream;
  int rc;
  if ((rc = use_dense(h))) return rc;
  // a valid state for every stage: linearise, damp with tau * max diagonal, build and solve once
  if ((rc = ops->relinearize(s, true, 1e-3, st))) return rc;
  V3DBA_CUDA_TRY(cudaMemsetAsync(s.d_fail, 0, sizeof(int), st));
  if ((rc = tile_chol_zero(h->chol, s.S, s.rhs, st))) return rc;
  if ((rc = ops->build_reduced(s, st))) return rc;
  if ((rc = tile_chol_solve(h->chol, s.S, s.x, s.d_fail, st))) return rc;
  if ((rc = ops->finish_trial(s, st))) return rc;
  float t = 0.f;
  for (int id = 0; id < kNumLmStages; ++id) {
    V3DBA_CUDA_TRY(cudaEventRecord(h->ev0, st));
    for (int r = 0; r < reps; ++r)
      if ((rc = ops->stage(s, id, 0, 1e-3, st))) return rc;
    V3DBA_CUDA_TRY(cudaEventRecord(h->ev1, st));
    V3DBA_CUDA_TRY(cudaEventSynchronize(h->ev1));
    cudaEventElapsedTime(&t, h->ev0, h->ev1);
    ms[id] = t / reps;
  }
  // Cholesky factor + solve: rebuild the system before every timed factorisation
  double chol = 0.0, zero = 0.0;
  for (int r = 0; r < reps; ++r) {
    V3DBA_CUDA_TRY(cudaEventRecord(h->ev0, st));
    if ((rc = tile_chol_zero(h->chol, s.S, s.rhs, st))) return rc;
    V3DBA_CUDA_TRY(cudaEventRecord(h->ev1, st));
    V3DBA_CUDA_TRY(cudaEventSynchronize(h->ev1));
    cudaEventElapsedTime(&t, h->ev0, h->ev1);
    zero += t;
    if ((rc = ops->build_reduced(s, st))) return rc;
    V3DBA_CUDA_TRY(cudaEventRecord(h->ev0, st));
    if ((rc = tile_chol_solve(h->chol, s.S, s.x, s.d_fail, st))) return rc;
    V3DBA_CUDA_TRY(cudaEventRecord(h->ev1, st));
    V3DBA_CUDA_TRY(cudaEventSynchronize(h->ev1));
    cudaEventElapsedTime(&t, h->ev0, h->ev1);
    chol += t;
  }
  ms[kNumLmStages] = chol / reps;
  ms[kNumLmStages + 1] = zero / reps;
  return V3DBA_OK;
}

extern "C" int v3dba_cholesky_flops(v3dba_handle h, double* flops) {
  if (!h || !flops) return V3DBA_ERR_INVALID_ARGUMENT;
  const int rc = use_dense(h);
  if (rc) return rc;
  const TileChol& tc = h->chol;
  if (tc.levels) {
    *flops = tc.level_flops;
    return V3DBA_OK;
  }
  const double gemm = 2.0 * 64.0 * 64.0 * 64.0;
  // per tile column: the diagonal factor (L and L^-1, about 2/3 + 1/3 of 64^3) and one GEMM per
  // panel tile and per trailing tile
  double f = 0.0;
  for (int k = 0; k < tc.nt; ++k) {
    f += 64.0 * 64.0 * 64.0;
    f += gemm * (tc.h_panel_ptr[k + 1] - tc.h_panel_ptr[k]);
    f += gemm * (tc.h_upd_ptr[k + 1] - tc.h_upd_ptr[k]);
  }
  *flops = f;
  return V3DBA_OK;
}

extern "C" int v3dba_cholesky_schedule(v3dba_handle h, int* schedule, int* n_levels, int* nt) {
  if (!h || !schedule || !n_levels || !nt) return V3DBA_ERR_INVALID_ARGUMENT;
  const int rc = use_dense(h);
  if (rc) return rc;
  const TileChol& tc = h->chol;
  *schedule = tc.levels ? 1 : 0;
  *n_levels = tc.levels ? tc.n_levels : tc.nt;
  *nt = tc.nt;
  return V3DBA_OK;
}

namespace v3dba {
int handle_use_dense(v3dba_handle h) { return use_dense(h); }
DevState& handle_state(v3dba_handle h) { return h->s; }
TileChol& handle_chol(v3dba_handle h) { return h->chol; }
cudaStream_t handle_stream(v3dba_handle h) { return h->stream; }
const std::vector<int>& handle_blk_i(v3dba_handle h) { return h->blk_i; }
const std::vector<int>& handle_blk_l(v3dba_handle h) { return h->blk_l; }
int handle_use_pcg(v3dba_handle h) { return use_pcg(h); }
PcgState& handle_pcg(v3dba_handle h) { return h->pcg; }
const double* handle_cur_R(v3dba_handle h) { return h->s.cur.R; }
const double* handle_cur_T(v3dba_handle h) { return h->s.cur.T; }
}  // namespace v3dba

extern "C" int v3dba_set_precond_model(v3dba_handle h, v3dba_precond_model m) {
  if (!h) return V3DBA_ERR_INVALID_ARGUMENT;
  h->precond = m;
  return V3DBA_OK;
}
