// Shared device/host helpers of the B200 bundle adjuster.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "v3dba.h"

namespace v3dba {

// Counts every kernel launch issued by this library (reported by v3dba_launch_count()).
void note_launches(uint64_t n);

// True when no value is Inf or NaN (host; branch-free so the scan vectorises).
bool all_finite(const double* p, size_t n);
bool all_finite_f(const float* p, size_t n);

// NVTX range for the scope of the object (names the LM stages on an Nsight timeline).  NVTX is
// header-only: without a tool attached each push / pop is a branch on a null function pointer.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Host phase timings on stderr when the environment variable `env` is set (diagnostics).
struct PhaseTrace {
  explicit PhaseTrace(const char* env, const char* label);
  void mark(const char* phase, cudaStream_t st = nullptr);
  bool on;
  const char* label;
  double t;
};

// Many device buffers carved from one stream-ordered allocation (one cudaMallocAsync, one
// cudaFreeAsync): add() records the requests, commit() allocates and assigns the pointers.
struct Arena {
  template <typename T>
  void add(T** p, size_t n) {
    req_.push_back({reinterpret_cast<void**>(p), (std::max<size_t>(n, 1) * sizeof(T) + 255) & ~(size_t)255});
  }
  int commit(cudaStream_t st);
  void release(cudaStream_t st);
  char* base = nullptr;

 private:
  struct Req {
    void** p;
    size_t bytes;
  };
  std::vector<Req> req_;
};

// Allocation-failure injection for tests (v3dba_debug_fail_allocation): true when the device
// allocation about to be made is to report out-of-memory instead, as a failed cudaMalloc would.
// Every device allocation of the handle / batch / structure paths asks first.
bool injected_alloc_failure();

// Raises the release threshold of the current device's stream-ordered pool once, so memory
// freed by one handle is kept for the next (handles are created and destroyed in loops).
int ensure_pool();

#define V3DBA_CUDA_TRY(expr)                                                        \
  do {                                                                              \
    cudaError_t _e = (expr);                                                        \
    if (_e != cudaSuccess) {                                                        \
      fprintf(stderr, "v3dba: %s failed: %s (%s:%d)\n", #expr, cudaGetErrorString(_e), \
              __FILE__, __LINE__);                                                  \
      return _e == cudaErrorMemoryAllocation ? V3DBA_ERR_OUT_OF_MEMORY : V3DBA_ERR_CUDA; \
    }                                                                               \
  } while (0)

#define V3DBA_LAUNCH_CHECK()                                                        \
  do {                                                                              \
    ::v3dba::note_launches(1);                                                      \
    cudaError_t _e = cudaPeekAtLastError();                                         \
    if (_e != cudaSuccess) {                                                        \
      fprintf(stderr, "v3dba: launch failed: %s (%s:%d)\n", cudaGetErrorString(_e), \
              __FILE__, __LINE__);                                                  \
      return V3DBA_ERR_CUDA;                                                        \
    }                                                                               \
  } while (0)

constexpr int kWarp = 32;

// Programmatic dependent launch (sm_90 and later).  A kernel launched with launch_pdl may be
// scheduled while its predecessor in the stream is still running: it must call pdl_wait(), which
// returns once the predecessor grid has completed and its writes are visible, before it touches
// anything the predecessor writes.  pdl_trigger() lets the next kernel be scheduled once every
// block of this one has issued it (so all of this kernel's blocks are resident by then).  In a
// kernel launched the usual way both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T u = __shfl_xor_sync(0xffffffffu, v, o);
    v = u > v ? u : v;
  }
  return v;
}

// Deterministic block-wide reduction of NV values (first NS summed, the rest max-reduced),
// result valid in thread 0.  smem needs blockDim.x/32 * NV doubles.
template <int NV, int NS>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* smem) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int t = 0; t < NV; ++t) v[t] = (t < NS) ? warp_sum(v[t]) : warp_max(v[t]);
  if (lane == 0) {
#pragma unroll
    for (int t = 0; t < NV; ++t) smem[wid * NV + t] = v[t];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nw; ++w) {
#pragma unroll
      for (int t = 0; t < NV; ++t) {
        double u = smem[w * NV + t];
        v[t] = (t < NS) ? v[t] + u : (u > v[t] ? u : v[t]);
      }
    }
  }
  __syncthreads();
}

// Real-valued storage type of the normal-equation blocks.
template <typename Real>
__device__ __forceinline__ Real to_real(double x) { return static_cast<Real>(x); }

}  // namespace v3dba
