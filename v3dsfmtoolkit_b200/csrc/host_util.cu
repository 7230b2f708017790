// Host-side helpers shared by the entry points.
#include <atomic>
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
