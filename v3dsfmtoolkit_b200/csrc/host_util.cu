// Host-side helpers shared by the entry points.
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>

#include "common.cuh"

namespace v3dba {

bool all_finite(const double* p, size_t n) {
  constexpr uint64_t kExp = 0x7ff0000000000000ull;   // exponent all ones: Inf or NaN
  uint64_t bad = 0;
  for (size_t i = 0; i < n; ++i) {
    uint64_t b;
    std::memcpy(&b, p + i, sizeof(b));
    bad |= (uint64_t)((b & kExp) == kExp);
  }
  return bad == 0;
}

bool all_finite_f(const float* p, size_t n) {
  constexpr uint32_t kExp = 0x7f800000u;
  uint32_t bad = 0;
  for (size_t i = 0; i < n; ++i) {
    uint32_t b;
    std::memcpy(&b, p + i, sizeof(b));
    bad |= (uint32_t)((b & kExp) == kExp);
  }
  return bad == 0;
}

static double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

PhaseTrace::PhaseTrace(const char* env, const char* lbl) : on(std::getenv(env) != nullptr), label(lbl), t(now_ms()) {}

void PhaseTrace::mark(const char* phase, cudaStream_t st) {
  if (!on) return;
  if (st) cudaStreamSynchronize(st);
  const double n = now_ms();
  std::fprintf(stderr, "%s %-12s %8.3f ms\n", label, phase, n - t);
  t = n;
}

// -1: off; k >= 0: the allocation k requests from now reports out-of-memory (then off again)
static std::atomic<long long> g_alloc_countdown{-1};

bool injected_alloc_failure() {
  if (g_alloc_countdown.load(std::memory_order_relaxed) < 0) return false;
  long long c = g_alloc_countdown.load(std::memory_order_relaxed);
  while (c >= 0 && !g_alloc_countdown.compare_exchange_weak(c, c - 1, std::memory_order_relaxed)) {
  }
  return c == 0;
}

int Arena::commit(cudaStream_t st) {
  size_t total = 0;
  for (const Req& r : req_) total += r.bytes;
  int rc = ensure_pool();
  if (rc) return rc;
  if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
  void* q = nullptr;
  V3DBA_CUDA_TRY(cudaMallocAsync(&q, std::max<size_t>(total, 256), st));
  base = static_cast<char*>(q);
  size_t off = 0;
  for (const Req& r : req_) {
    *r.p = base + off;
    off += r.bytes;
  }
  return V3DBA_OK;
}

void Arena::release(cudaStream_t st) {
  if (base) cudaFreeAsync(base, st);
  base = nullptr;
}

int ensure_pool() {
  static std::atomic<uint64_t> done_mask{0};
  int dev = 0;
  V3DBA_CUDA_TRY(cudaGetDevice(&dev));
  const uint64_t bit = 1ull << (dev & 63);
  if (done_mask.load() & bit) return V3DBA_OK;
  cudaMemPool_t pool;
  V3DBA_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t thr = UINT64_MAX;
  V3DBA_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  done_mask.fetch_or(bit);
  return V3DBA_OK;
}

}  // namespace v3dba

extern "C" int v3dba_debug_fail_allocation(long long k) {
  if (k < -1) return V3DBA_ERR_INVALID_ARGUMENT;
  v3dba::g_alloc_countdown.store(k);
  return V3DBA_OK;
}
