// Device construction of a problem's structure: the point-major observation order, the camera
// observation lists and the camera-pair blocks of the reduced camera system with their
// observation pairs.
//
// The reference's callers hand the optimizer the flat arrays of a BundlePointStructure
// (V3D/include/Geometry/v3d_mviewutilities.h:132-163: measurements point after point, with
// correspondingView / correspondingPoint), and its SparseLevenbergOptimizer derives the
// Jacobian pattern from them on the host (setupSparseJtJ, V3D/src/Math/v3d_optimization.cpp:
// 301-554).  Here the raw arrays go to the device once and every ordering is made there by one
// stable LSD radix sort (8-bit digits; within a tile, ranks by warp match masks in item order,
// so equal keys keep their input order and the result is deterministic):
//   * observations sorted by point (stable: the caller's order inside a track);
//   * the observations of each camera, in point-major order;
//   * observation pairs (k, m) of a point with camera(m) >= camera(k), generated point after
//     point, then sorted by camera(m) and stably by camera(k): grouped by block (i, l), i <= l,
//     and inside a block by point.
// Only the per-camera and per-block pointers (a few KB) return to the host, for the work
// chunks and the factorisation plan.
#include <algorithm>
#include <cstring>
#include <functional>
#include <vector>

#include "common.cuh"
#include "lm.cuh"
#include "structure.cuh"

namespace v3dba {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 8;
constexpr int kSortTile = kSortThreads * kSortRounds;   // items per block and pass
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 2 * kScanThreads;            // items per block of the scan

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// Per-block digit counts of one pass: hist[d * nblk + b].
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint32_t* __restrict__ keys, int n, int shift,
                                                             int* __restrict__ hist) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * kSortTile;
  for (int r = 0; r < kSortRounds; ++r) {
    const int i = base + r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255], 1);
  }
  __syncthreads();
  hist[threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

// Stable scatter of one pass.  Items are taken in order (round by round, thread by thread); the
// rank of an item among the earlier items of its digit in the block is its rank inside its warp
// (match mask) plus the counts of the earlier warps of the round plus the earlier rounds.
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint32_t* __restrict__ kin,
                                                                const int* __restrict__ vin, int n, int shift,
                                                                const int* __restrict__ offs, uint32_t* kout,
                                                                int* vout) {
  __shared__ int run[256];
  __shared__ int wcnt[kSortThreads / 32][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  run[threadIdx.x] = offs[threadIdx.x * gridDim.x + blockIdx.x];
  const unsigned lt = (1u << lane) - 1u;
  const int base = blockIdx.x * kSortTile;
  for (int r = 0; r < kSortRounds; ++r) {
    for (int w = 0; w < kSortThreads / 32; ++w) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const int i = base + r * kSortThreads + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key = valid ? kin[i] : 0u;
    const int d = valid ? (int)((key >> shift) & 255) : 256;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int wrank = __popc(peers & lt);
    if (valid && wrank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      int pos = run[d] + wrank;
      for (int w = 0; w < warp; ++w) pos += wcnt[w][d];
      kout[pos] = key;
      vout[pos] = vin[i];
    }
    __syncthreads();
    int add = 0;
    for (int w = 0; w < kSortThreads / 32; ++w) add += wcnt[w][threadIdx.x];
    run[threadIdx.x] += add;
    __syncthreads();
  }
}

// Exclusive scan, in place, of one block's 2048 items; the block's total to sums[blockIdx].
__global__ void __launch_bounds__(kScanThreads) k_scan_block(int* __restrict__ a, int n, int* __restrict__ sums) {
  __shared__ int s[kScanItems];
  const int base = blockIdx.x * kScanItems;
  for (int t = threadIdx.x; t < kScanItems; t += kScanThreads) s[t] = (base + t < n) ? a[base + t] : 0;
  __syncthreads();
  // up-sweep / down-sweep (work-efficient exclusive scan)
  for (int d = 1; d < kScanItems; d <<= 1) {
    const int i = (threadIdx.x + 1) * 2 * d - 1;
    if (i < kScanItems) s[i] += s[i - d];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (sums) sums[blockIdx.x] = s[kScanItems - 1];
    s[kScanItems - 1] = 0;
  }
  __syncthreads();
  for (int d = kScanItems / 2; d >= 1; d >>= 1) {
    const int i = (threadIdx.x + 1) * 2 * d - 1;
    if (i < kScanItems) {
      const int t = s[i - d];
      s[i - d] = s[i];
      s[i] += t;
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < kScanItems; t += kScanThreads)
    if (base + t < n) a[base + t] = s[t];
}

__global__ void k_scan_add(int* __restrict__ a, int n, const int* __restrict__ sums) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) a[i] += sums[i / kScanItems];
}

__global__ void k_iota(int* v, int n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) v[i] = (int)i;
}

__global__ void k_int_to_key(const int* __restrict__ a, uint32_t* k, int n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) k[i] = (uint32_t)a[i];
}

// ptr[v] = first position of key v in the sorted keys (ptr[nv] = n), for every v in [0, nv].
__global__ void k_key_bounds(const uint32_t* __restrict__ keys, int n, int nv, int* __restrict__ ptr) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i > n) return;
  const int lo = i == 0 ? 0 : (int)keys[i - 1] + 1;   // keys in (keys[i-1], keys[i]] start at i
  const int hi = i == n ? nv : (int)keys[i];
  for (int v = lo; v <= hi; ++v) ptr[v] = (int)i;
}

__global__ void k_gather_obs(const int* __restrict__ orig, const int* __restrict__ view, const double* __restrict__ meas,
                             int K, int* o_cam, double* o_meas) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= K) return;
  const int o = orig[k];
  o_cam[k] = view[o];
  o_meas[2 * k] = meas[2 * (size_t)o];
  o_meas[2 * k + 1] = meas[2 * (size_t)o + 1];
}

// pairs of each point: sum over its observations k of #{m in the track : cam(m) >= cam(k)}
__global__ void k_pair_count(const int* __restrict__ p_ptr, const int* __restrict__ o_cam, int M, int* cnt,
                             unsigned long long* total) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  int c = 0;
  for (int k = p_ptr[j]; k < p_ptr[j + 1]; ++k)
    for (int m = p_ptr[j]; m < p_ptr[j + 1]; ++m) c += o_cam[m] >= o_cam[k];
  cnt[j] = c;
  atomicAdd(total, (unsigned long long)c);   // integer sum: order-independent
}

// the pairs of each point in (k, m) order, with their block's camera columns as sort keys
__global__ void k_pair_gen(const int* __restrict__ p_ptr, const int* __restrict__ o_cam, int M,
                           const int* __restrict__ off, int* pk, int* pm, uint32_t* key_l) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= M) return;
  int o = off[j];
  for (int k = p_ptr[j]; k < p_ptr[j + 1]; ++k)
    for (int m = p_ptr[j]; m < p_ptr[j + 1]; ++m)
      if (o_cam[m] >= o_cam[k]) {
        pk[o] = k;
        pm[o] = m;
        key_l[o] = (uint32_t)o_cam[m];
        ++o;
      }
}

__global__ void k_pair_key_i(const int* __restrict__ perm, const int* __restrict__ pk, const int* __restrict__ o_cam,
                             int P, uint32_t* key_i) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t < P) key_i[t] = (uint32_t)o_cam[pk[perm[t]]];
}

__global__ void k_pair_finish(const int* __restrict__ perm, const int* __restrict__ pk, const int* __restrict__ pm,
                              int P, int* pr_k, int* pr_m) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= P) return;
  const int q = perm[t];
  pr_k[t] = pk[q];
  pr_m[t] = pm[q];
}

// heads of runs of equal block keys: flag[t] = 1 where a new block starts
__global__ void k_run_heads(const int* __restrict__ perm, const int* __restrict__ pk, const int* __restrict__ pm,
                            const int* __restrict__ o_cam, int P, int* flag) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= P) return;
  if (t == 0) { flag[0] = 1; return; }
  const int q = perm[t], q0 = perm[t - 1];
  flag[t] = (o_cam[pk[q]] != o_cam[pk[q0]] || o_cam[pm[q]] != o_cam[pm[q0]]) ? 1 : 0;
}

__global__ void k_run_starts(const int* __restrict__ flag_scan, const int* __restrict__ flag, const int* __restrict__ perm,
                             const int* __restrict__ pk, const int* __restrict__ pm, const int* __restrict__ o_cam,
                             int P, int* b_start, int* b_i, int* b_l) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= P || !flag[t]) return;
  const int b = flag_scan[t];
  const int q = perm[t];
  b_start[b] = (int)t;
  b_i[b] = o_cam[pk[q]];
  b_l[b] = o_cam[pm[q]];
}

struct Scratch {
  std::vector<void*> bufs;
  cudaStream_t st;
  ~Scratch() { for (void* p : bufs) cudaFreeAsync(p, st); }
  template <typename T>
  int get(T** p, size_t n) {
    void* q = nullptr;
    if (injected_alloc_failure()) return V3DBA_ERR_OUT_OF_MEMORY;
    cudaError_t e = cudaMallocAsync(&q, sizeof(T) * std::max<size_t>(n, 1), st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return e == cudaErrorMemoryAllocation ? V3DBA_ERR_OUT_OF_MEMORY : V3DBA_ERR_CUDA;
    }
    bufs.push_back(q);
    *p = static_cast<T*>(q);
    return V3DBA_OK;
  }
};

// In-place exclusive scan of n ints (recursive over block totals).
int scan_exclusive(Scratch& sc, int* a, int n, cudaStream_t st) {
  if (n <= 0) return V3DBA_OK;
  const int nb = cdiv(n, kScanItems);
  int* sums = nullptr;
  int rc;
  if (nb > 1 && (rc = sc.get(&sums, nb))) return rc;
  k_scan_block<<<nb, kScanThreads, 0, st>>>(a, n, sums);
  V3DBA_LAUNCH_CHECK();
  if (nb > 1) {
    if ((rc = scan_exclusive(sc, sums, nb, st))) return rc;
    k_scan_add<<<cdiv(n, 256), 256, 0, st>>>(a, n, sums);
    V3DBA_LAUNCH_CHECK();
  }
  return V3DBA_OK;
}

int bits_for(uint64_t max_value) {
  int b = 0;
  while (b < 32 && (max_value >> b) != 0) ++b;
  return std::max(b, 1);
}

// Stable sort of (key, value) pairs by the low `bits` bits of the keys.  The result ends in
// (*keys, *vals) (the pointers may be swapped with the ping-pong buffers).
int radix_sort(Scratch& sc, uint32_t** keys, int** vals, uint32_t* ktmp, int* vtmp, int n, int bits, cudaStream_t st) {
  if (n <= 1) return V3DBA_OK;
  const int nblk = cdiv(n, kSortTile);
  int* hist;
  int rc;
  if ((rc = sc.get(&hist, (size_t)256 * nblk))) return rc;
  uint32_t *kin = *keys, *kout = ktmp;
  int *vin = *vals, *vout = vtmp;
  for (int shift = 0; shift < bits; shift += 8) {
    k_radix_hist<<<nblk, kSortThreads, 0, st>>>(kin, n, shift, hist);
    V3DBA_LAUNCH_CHECK();
    if ((rc = scan_exclusive(sc, hist, 256 * nblk, st))) return rc;
    k_radix_scatter<<<nblk, kSortThreads, 0, st>>>(kin, vin, n, shift, hist, kout, vout);
    V3DBA_LAUNCH_CHECK();
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  *keys = kin;
  *vals = vin;
  return V3DBA_OK;
}

// ---- BundlePointStructure (V3D/include/Geometry/v3d_mviewutilities.h:132-205) ----------------

// keep[j] = 1 when track j has at least n_required measurements (the reference compares the
// size_t track length with the int threshold, so a negative threshold keeps nothing); cnt[j] =
// its measurement count when kept.  Entry n of both is 0 (the scans then end in the totals).
__global__ void k_bps_flags(const int* __restrict__ ptr, int n, int n_required, int* __restrict__ keep,
                            int* __restrict__ cnt) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > n) return;
  if (j == n) {
    keep[n] = 0;
    cnt[n] = 0;
    return;
  }
  const int len = ptr[j + 1] - ptr[j];
  const bool k = n_required >= 0 && len >= n_required;
  keep[j] = k ? 1 : 0;
  cnt[j] = k ? len : 0;
}

// One thread per kept track: its point, its index, and its measurements (float positions widened
// to double, as makeVector2<double> does) at the scanned offsets.
__global__ void k_bps_scatter(const int* __restrict__ ptr, const double* __restrict__ pos, const int* __restrict__ view,
                              const int* __restrict__ id, const float* __restrict__ mpos, int n,
                              const int* __restrict__ pidx, const int* __restrict__ midx, double* __restrict__ points3d,
                              double* __restrict__ meas, int* __restrict__ ids, int* __restrict__ cview,
                              int* __restrict__ cpoint, int* __restrict__ xs) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || pidx[j + 1] == pidx[j]) return;
  const int i = pidx[j], o = midx[j], b = ptr[j], len = ptr[j + 1] - b;
  points3d[3 * (size_t)i] = pos[3 * (size_t)j];
  points3d[3 * (size_t)i + 1] = pos[3 * (size_t)j + 1];
  points3d[3 * (size_t)i + 2] = pos[3 * (size_t)j + 2];
  xs[i] = j;
  for (int k = 0; k < len; ++k) {
    meas[2 * (size_t)(o + k)] = (double)mpos[2 * (size_t)(b + k)];
    meas[2 * (size_t)(o + k) + 1] = (double)mpos[2 * (size_t)(b + k) + 1];
    ids[o + k] = id[b + k];
    cview[o + k] = view[b + k];
    cpoint[o + k] = i;
  }
}

// createPointStructure from scratch: measurement t of the new tracks is the caller's src = perm[t]
// (grouped by point, the caller's order inside a point); positions narrowed to float.
__global__ void k_cps_gather(const int* __restrict__ perm, const double* __restrict__ meas, const int* __restrict__ ids,
                             const int* __restrict__ cview, int K, int* __restrict__ view, int* __restrict__ id,
                             float* __restrict__ mpos) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= K) return;
  const int src = perm[t];
  view[t] = cview[src];
  id[t] = ids[src];
  mpos[2 * (size_t)t] = (float)meas[2 * (size_t)src];
  mpos[2 * (size_t)t + 1] = (float)meas[2 * (size_t)src + 1];
}

__global__ void k_cps_lengths(const int* __restrict__ ptr, const int* __restrict__ xs, int M, int* __restrict__ len) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < M) len[i] = ptr[xs[i] + 1] - ptr[xs[i]];
  else if (i == M) len[M] = 0;
}

// createPointStructure in place: kept track xs[i] gets point i and, in order, the next len_i
// measurements (from offset off[i]) as its measurement positions.
__global__ void k_cps_inplace(const int* __restrict__ ptr, const int* __restrict__ xs, const int* __restrict__ off,
                              int M, const double* __restrict__ points3d, const double* __restrict__ meas,
                              double* __restrict__ pos, float* __restrict__ mpos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M) return;
  const int j = xs[i], b = ptr[j], len = ptr[j + 1] - b, o = off[i];
  pos[3 * (size_t)j] = points3d[3 * (size_t)i];
  pos[3 * (size_t)j + 1] = points3d[3 * (size_t)i + 1];
  pos[3 * (size_t)j + 2] = points3d[3 * (size_t)i + 2];
  for (int k = 0; k < len; ++k) {
    mpos[2 * (size_t)(b + k)] = (float)meas[2 * (size_t)(o + k)];
    mpos[2 * (size_t)(b + k) + 1] = (float)meas[2 * (size_t)(o + k) + 1];
  }
}

}  // namespace

int build_structure_device(const v3dba_problem* p, const DevAlloc& alloc, cudaStream_t st, DeviceStructure& S) {
  const int N = p->n_cameras, M = p->n_points, K = p->n_measurements;
  Scratch sc;
  sc.st = st;
  int rc;
  auto dal = [&](auto** q, size_t n) -> int {
    using T = typename std::remove_reference<decltype(**q)>::type;
    return alloc(reinterpret_cast<void**>(q), sizeof(T) * std::max<size_t>(n, 1));
  };
  // raw inputs
  int *d_view, *d_point;
  double* d_meas;
  if ((rc = sc.get(&d_view, K)) || (rc = sc.get(&d_point, K)) || (rc = sc.get(&d_meas, 2 * (size_t)K))) return rc;
  if (K > 0) {
    V3DBA_CUDA_TRY(cudaMemcpyAsync(d_view, p->view, sizeof(int) * K, cudaMemcpyHostToDevice, st));
    V3DBA_CUDA_TRY(cudaMemcpyAsync(d_point, p->point, sizeof(int) * K, cudaMemcpyHostToDevice, st));
    V3DBA_CUDA_TRY(cudaMemcpyAsync(d_meas, p->measurements, sizeof(double) * 2 * K, cudaMemcpyHostToDevice, st));
  }
  const int gK = cdiv(std::max(K, 1), 256);
  // 1. point-major permutation
  uint32_t *ka, *kb;
  int *va, *vb;
  if ((rc = sc.get(&ka, K)) || (rc = sc.get(&kb, K)) || (rc = sc.get(&va, K)) || (rc = sc.get(&vb, K))) return rc;
  if ((rc = dal(&S.o_orig, K)) || (rc = dal(&S.o_pt, K)) || (rc = dal(&S.o_cam, K)) || (rc = dal(&S.o_meas, 2 * (size_t)K)) ||
      (rc = dal(&S.p_ptr, (size_t)M + 1)) || (rc = dal(&S.c_ptr, (size_t)N + 1)) || (rc = dal(&S.c_obs, K)))
    return rc;
  if (K > 0) {
    k_int_to_key<<<gK, 256, 0, st>>>(d_point, ka, K);
    V3DBA_LAUNCH_CHECK();
    k_iota<<<gK, 256, 0, st>>>(va, K);
    V3DBA_LAUNCH_CHECK();
  }
  uint32_t* keys = ka;
  int* vals = va;
  if ((rc = radix_sort(sc, &keys, &vals, kb, vb, K, bits_for((uint64_t)std::max(M - 1, 0)), st))) return rc;
  if (K > 0) {
    V3DBA_CUDA_TRY(cudaMemcpyAsync(S.o_orig, vals, sizeof(int) * K, cudaMemcpyDeviceToDevice, st));
    V3DBA_CUDA_TRY(cudaMemcpyAsync(S.o_pt, keys, sizeof(int) * K, cudaMemcpyDeviceToDevice, st));
  }
  k_key_bounds<<<cdiv((long)K + 1, 256), 256, 0, st>>>(keys, K, M, S.p_ptr);
  V3DBA_LAUNCH_CHECK();
  if (K > 0) {
    k_gather_obs<<<gK, 256, 0, st>>>(S.o_orig, d_view, d_meas, K, S.o_cam, S.o_meas);
    V3DBA_LAUNCH_CHECK();
  }
  // 2. observation lists of every camera (stable: point-major order)
  if (K > 0) {
    k_int_to_key<<<gK, 256, 0, st>>>(S.o_cam, ka, K);
    V3DBA_LAUNCH_CHECK();
    k_iota<<<gK, 256, 0, st>>>(va, K);
    V3DBA_LAUNCH_CHECK();
  }
  keys = ka;
  vals = va;
  if ((rc = radix_sort(sc, &keys, &vals, kb, vb, K, bits_for((uint64_t)std::max(N - 1, 0)), st))) return rc;
  if (K > 0) V3DBA_CUDA_TRY(cudaMemcpyAsync(S.c_obs, vals, sizeof(int) * K, cudaMemcpyDeviceToDevice, st));
  k_key_bounds<<<cdiv((long)K + 1, 256), 256, 0, st>>>(keys, K, N, S.c_ptr);
  V3DBA_LAUNCH_CHECK();
  // 3. observation pairs, grouped by camera-pair block
  int* off;
  unsigned long long* d_total;
  if ((rc = sc.get(&off, (size_t)M + 1)) || (rc = sc.get(&d_total, 1))) return rc;
  const int gM = cdiv(std::max(M, 1), 128);
  V3DBA_CUDA_TRY(cudaMemsetAsync(d_total, 0, sizeof(unsigned long long), st));
  if (M > 0) {
    k_pair_count<<<gM, 128, 0, st>>>(S.p_ptr, S.o_cam, M, off, d_total);
    V3DBA_LAUNCH_CHECK();
  }
  unsigned long long total = 0;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(&total, d_total, sizeof(total), cudaMemcpyDeviceToHost, st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  if (total > 0x7fffffffull) return V3DBA_ERR_UNSUPPORTED;   // pair indices are 32-bit
  const int P = (int)total;
  S.P = P;
  V3DBA_CUDA_TRY(cudaMemsetAsync(off + M, 0, sizeof(int), st));
  if ((rc = scan_exclusive(sc, off, M + 1, st))) return rc;
  int *pk, *pm, *perm, *permt, *flag;
  uint32_t *kl, *klt;
  if ((rc = sc.get(&pk, P)) || (rc = sc.get(&pm, P)) || (rc = sc.get(&perm, P)) || (rc = sc.get(&permt, P)) ||
      (rc = sc.get(&kl, P)) || (rc = sc.get(&klt, P)) || (rc = sc.get(&flag, (size_t)P + 1)))
    return rc;
  if ((rc = dal(&S.pr_k, P)) || (rc = dal(&S.pr_m, P))) return rc;
  const int gP = cdiv(std::max(P, 1), 256);
  if (M > 0 && P > 0) {
    k_pair_gen<<<gM, 128, 0, st>>>(S.p_ptr, S.o_cam, M, off, pk, pm, kl);
    V3DBA_LAUNCH_CHECK();
    k_iota<<<gP, 256, 0, st>>>(perm, P);
    V3DBA_LAUNCH_CHECK();
  }
  const int cam_bits = bits_for((uint64_t)std::max(N - 1, 0));
  keys = kl;
  vals = perm;
  if ((rc = radix_sort(sc, &keys, &vals, klt, permt, P, cam_bits, st))) return rc;   // by camera l
  int* perm_l = vals;
  uint32_t* ki = (keys == kl) ? klt : kl;
  int* permt2 = (perm_l == perm) ? permt : perm;
  if (P > 0) {
    k_pair_key_i<<<gP, 256, 0, st>>>(perm_l, pk, S.o_cam, P, ki);
    V3DBA_LAUNCH_CHECK();
  }
  // stable by camera i on top: (i, l) order, generation order inside a block
  uint32_t* kspare = (ki == kl) ? klt : kl;
  keys = ki;
  vals = perm_l;
  if ((rc = radix_sort(sc, &keys, &vals, kspare, permt2, P, cam_bits, st))) return rc;
  int* order = vals;
  int nb_run = 0;
  std::vector<int> run_start, run_i, run_l;
  if (P > 0) {
    k_pair_finish<<<gP, 256, 0, st>>>(order, pk, pm, P, S.pr_k, S.pr_m);
    V3DBA_LAUNCH_CHECK();
    k_run_heads<<<gP, 256, 0, st>>>(order, pk, pm, S.o_cam, P, flag);
    V3DBA_LAUNCH_CHECK();
    int* fscan;
    if ((rc = sc.get(&fscan, P))) return rc;
    V3DBA_CUDA_TRY(cudaMemcpyAsync(fscan, flag, sizeof(int) * P, cudaMemcpyDeviceToDevice, st));
    if ((rc = scan_exclusive(sc, fscan, P, st))) return rc;
    int last_scan = 0, last_flag = 0;
    V3DBA_CUDA_TRY(cudaMemcpyAsync(&last_scan, fscan + P - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    V3DBA_CUDA_TRY(cudaMemcpyAsync(&last_flag, flag + P - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
    nb_run = last_scan + last_flag;
    int *rs, *ri, *rl;
    if ((rc = sc.get(&rs, nb_run)) || (rc = sc.get(&ri, nb_run)) || (rc = sc.get(&rl, nb_run))) return rc;
    k_run_starts<<<gP, 256, 0, st>>>(fscan, flag, order, pk, pm, S.o_cam, P, rs, ri, rl);
    V3DBA_LAUNCH_CHECK();
    run_start.resize(nb_run);
    run_i.resize(nb_run);
    run_l.resize(nb_run);
    V3DBA_CUDA_TRY(cudaMemcpyAsync(run_start.data(), rs, sizeof(int) * nb_run, cudaMemcpyDeviceToHost, st));
    V3DBA_CUDA_TRY(cudaMemcpyAsync(run_i.data(), ri, sizeof(int) * nb_run, cudaMemcpyDeviceToHost, st));
    V3DBA_CUDA_TRY(cudaMemcpyAsync(run_l.data(), rl, sizeof(int) * nb_run, cudaMemcpyDeviceToHost, st));
  }
  S.h_c_ptr.resize((size_t)N + 1);
  V3DBA_CUDA_TRY(cudaMemcpyAsync(S.h_c_ptr.data(), S.c_ptr, sizeof(int) * ((size_t)N + 1), cudaMemcpyDeviceToHost, st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  // blocks in (i, l) order; every camera gets its diagonal block, even without observations
  S.h_b_i.clear();
  S.h_b_l.clear();
  S.h_b_ptr.assign(1, 0);
  int r = 0;
  for (int i = 0; i < N; ++i) {
    bool diag = false;
    auto emit = [&](int l, int end) {
      S.h_b_i.push_back(i);
      S.h_b_l.push_back(l);
      S.h_b_ptr.push_back(end);
    };
    while (r < nb_run && run_i[r] == i) {
      const int end = (r + 1 < nb_run) ? run_start[r + 1] : P;
      if (run_l[r] == i) diag = true;
      if (!diag && run_l[r] > i) {   // no pair of camera i with itself: empty diagonal block first
        emit(i, S.h_b_ptr.back());
        diag = true;
      }
      emit(run_l[r], end);
      ++r;
    }
    if (!diag) emit(i, S.h_b_ptr.back());
  }
  if ((rc = dal(&S.b_i, S.h_b_i.size())) || (rc = dal(&S.b_l, S.h_b_l.size())) || (rc = dal(&S.b_ptr, S.h_b_ptr.size())))
    return rc;
  V3DBA_CUDA_TRY(cudaMemcpyAsync(S.b_i, S.h_b_i.data(), sizeof(int) * S.h_b_i.size(), cudaMemcpyHostToDevice, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(S.b_l, S.h_b_l.data(), sizeof(int) * S.h_b_l.size(), cudaMemcpyHostToDevice, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(S.b_ptr, S.h_b_ptr.data(), sizeof(int) * S.h_b_ptr.size(), cudaMemcpyHostToDevice, st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));   // the host vectors above must outlive their copies
  return V3DBA_OK;
}

int group_by_key_device(const int* keys, int n, int nv, int* perm, int* ptr, cudaStream_t st) {
  if (n < 0 || nv < 0) return V3DBA_ERR_INVALID_ARGUMENT;
  Scratch sc;
  sc.st = st;
  int rc;
  uint32_t *ka, *kb;
  int *va, *vb;
  if ((rc = sc.get(&ka, n)) || (rc = sc.get(&kb, n)) || (rc = sc.get(&va, n)) || (rc = sc.get(&vb, n))) return rc;
  const int g = cdiv(std::max(n, 1), 256);
  if (n > 0) {
    k_int_to_key<<<g, 256, 0, st>>>(keys, ka, n);
    V3DBA_LAUNCH_CHECK();
    k_iota<<<g, 256, 0, st>>>(va, n);
    V3DBA_LAUNCH_CHECK();
  }
  uint32_t* k = ka;
  int* v = va;
  if ((rc = radix_sort(sc, &k, &v, kb, vb, n, bits_for((uint64_t)std::max(nv - 1, 0)), st))) return rc;
  if (n > 0) V3DBA_CUDA_TRY(cudaMemcpyAsync(perm, v, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
  k_key_bounds<<<cdiv((long)n + 1, 256), 256, 0, st>>>(k, n, nv, ptr);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}

}  // namespace v3dba

using namespace v3dba;

namespace {

// A stream and a scratch list for one standalone call; the stream is synchronised and destroyed
// at the end.
struct CallScope {
  cudaStream_t st = nullptr;
  Scratch* sc = nullptr;
  ~CallScope() {
    if (sc) delete sc;   // frees the buffers on the stream
    if (st) {
      cudaStreamSynchronize(st);
      cudaStreamDestroy(st);
    }
  }
};

template <typename T>
int up_copy(Scratch& sc, T** d, const T* h, size_t n, cudaStream_t st) {
  int rc = sc.get(d, n);
  if (rc) return rc;
  if (n && h) V3DBA_CUDA_TRY(cudaMemcpyAsync(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice, st));
  return V3DBA_OK;
}

template <typename T>
int down_copy(T* h, const T* d, size_t n, cudaStream_t st) {
  if (n && h) V3DBA_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(T) * n, cudaMemcpyDeviceToHost, st));
  return V3DBA_OK;
}

bool valid_track_ptr(const int* ptr, int n) {
  if (ptr[0] != 0) return false;
  for (int j = 0; j < n; ++j)
    if (ptr[j + 1] < ptr[j]) return false;
  return true;
}

}  // namespace

extern "C" int v3dba_bundle_point_structure(int n_tracks, const int* track_ptr, const double* track_pos,
                                            const int* meas_view, const int* meas_id, const float* meas_pos,
                                            int n_required, int* n_points, int* n_measurements, double* points3d,
                                            double* measurements, int* measurement_ids, int* corresponding_view,
                                            int* corresponding_point, int* xs_indices) {
  if (n_tracks < 0 || !track_ptr || !n_points || !n_measurements) return V3DBA_ERR_INVALID_ARGUMENT;
  if (!valid_track_ptr(track_ptr, n_tracks)) return V3DBA_ERR_INVALID_INPUT;
  const int K = track_ptr[n_tracks];
  if ((n_tracks && !track_pos) || (K && (!meas_view || !meas_id || !meas_pos))) return V3DBA_ERR_INVALID_ARGUMENT;
  NvtxRange nvtx("v3dba_bundle_point_structure");
  CallScope cs;
  V3DBA_CUDA_TRY(cudaStreamCreateWithFlags(&cs.st, cudaStreamNonBlocking));
  cs.sc = new Scratch();
  cs.sc->st = cs.st;
  Scratch& sc = *cs.sc;
  const cudaStream_t st = cs.st;
  int *d_ptr, *d_view, *d_id, *d_keep, *d_cnt, *o_ids, *o_view, *o_point, *o_xs;
  double *d_pos, *o_pts, *o_meas;
  float* d_mpos;
  int rc;
  if ((rc = up_copy(sc, &d_ptr, track_ptr, (size_t)n_tracks + 1, st)) ||
      (rc = up_copy(sc, &d_pos, track_pos, 3 * (size_t)n_tracks, st)) ||
      (rc = up_copy(sc, &d_view, meas_view, (size_t)K, st)) || (rc = up_copy(sc, &d_id, meas_id, (size_t)K, st)) ||
      (rc = up_copy(sc, &d_mpos, meas_pos, 2 * (size_t)K, st)) || (rc = sc.get(&d_keep, (size_t)n_tracks + 1)) ||
      (rc = sc.get(&d_cnt, (size_t)n_tracks + 1)) || (rc = sc.get(&o_pts, 3 * (size_t)n_tracks)) ||
      (rc = sc.get(&o_meas, 2 * (size_t)K)) || (rc = sc.get(&o_ids, (size_t)K)) || (rc = sc.get(&o_view, (size_t)K)) ||
      (rc = sc.get(&o_point, (size_t)K)) || (rc = sc.get(&o_xs, (size_t)n_tracks)))
    return rc;
  k_bps_flags<<<cdiv(n_tracks + 1, 256), 256, 0, st>>>(d_ptr, n_tracks, n_required, d_keep, d_cnt);
  V3DBA_LAUNCH_CHECK();
  if ((rc = scan_exclusive(sc, d_keep, n_tracks + 1, st)) || (rc = scan_exclusive(sc, d_cnt, n_tracks + 1, st))) return rc;
  if (n_tracks > 0) {
    k_bps_scatter<<<cdiv(n_tracks, 128), 128, 0, st>>>(d_ptr, d_pos, d_view, d_id, d_mpos, n_tracks, d_keep, d_cnt,
                                                       o_pts, o_meas, o_ids, o_view, o_point, o_xs);
    V3DBA_LAUNCH_CHECK();
  }
  int tot[2] = {0, 0};
  V3DBA_CUDA_TRY(cudaMemcpyAsync(&tot[0], d_keep + n_tracks, sizeof(int), cudaMemcpyDeviceToHost, st));
  V3DBA_CUDA_TRY(cudaMemcpyAsync(&tot[1], d_cnt + n_tracks, sizeof(int), cudaMemcpyDeviceToHost, st));
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  const int M = tot[0], Kk = tot[1];
  if ((rc = down_copy(points3d, o_pts, 3 * (size_t)M, st)) || (rc = down_copy(measurements, o_meas, 2 * (size_t)Kk, st)) ||
      (rc = down_copy(measurement_ids, o_ids, (size_t)Kk, st)) || (rc = down_copy(corresponding_view, o_view, (size_t)Kk, st)) ||
      (rc = down_copy(corresponding_point, o_point, (size_t)Kk, st)) || (rc = down_copy(xs_indices, o_xs, (size_t)M, st)))
    return rc;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  *n_points = M;
  *n_measurements = Kk;
  return V3DBA_OK;
}

extern "C" int v3dba_create_point_structure(int from_scratch, int n_points, int n_measurements, const double* points3d,
                                            const double* measurements, const int* measurement_ids,
                                            const int* corresponding_view, const int* corresponding_point,
                                            const int* xs_indices, int n_tracks, int* track_ptr, double* track_pos,
                                            int* meas_view, int* meas_id, float* meas_pos) {
  if (n_points < 0 || n_measurements < 0 || !track_ptr) return V3DBA_ERR_INVALID_ARGUMENT;
  if ((n_points && !points3d) || (n_measurements && !measurements)) return V3DBA_ERR_INVALID_ARGUMENT;
  // track_pos is written for the n_points new tracks (from scratch) or the n_tracks existing ones
  // (in place); with none it may be NULL, as data() of an empty vector is
  if (!track_pos && (from_scratch ? n_points > 0 : n_tracks > 0)) return V3DBA_ERR_INVALID_ARGUMENT;
  NvtxRange nvtx("v3dba_create_point_structure");
  CallScope cs;
  V3DBA_CUDA_TRY(cudaStreamCreateWithFlags(&cs.st, cudaStreamNonBlocking));
  cs.sc = new Scratch();
  cs.sc->st = cs.st;
  Scratch& sc = *cs.sc;
  const cudaStream_t st = cs.st;
  int rc;
  if (from_scratch) {
    const int K = n_measurements, M = n_points;
    if (K && (!measurement_ids || !corresponding_view || !corresponding_point || !meas_view || !meas_id || !meas_pos))
      return V3DBA_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < K; ++k)
      if (corresponding_point[k] < 0 || corresponding_point[k] >= M) return V3DBA_ERR_INVALID_INPUT;
    int *d_cp, *d_ids, *d_cv, *d_perm, *d_ptr, *o_view, *o_id;
    double* d_meas;
    float* o_mpos;
    if ((rc = up_copy(sc, &d_cp, corresponding_point, (size_t)K, st)) ||
        (rc = up_copy(sc, &d_ids, measurement_ids, (size_t)K, st)) ||
        (rc = up_copy(sc, &d_cv, corresponding_view, (size_t)K, st)) ||
        (rc = up_copy(sc, &d_meas, measurements, 2 * (size_t)K, st)) || (rc = sc.get(&d_perm, (size_t)K)) ||
        (rc = sc.get(&d_ptr, (size_t)M + 1)) || (rc = sc.get(&o_view, (size_t)K)) || (rc = sc.get(&o_id, (size_t)K)) ||
        (rc = sc.get(&o_mpos, 2 * (size_t)K)))
      return rc;
    if ((rc = group_by_key_device(d_cp, K, M, d_perm, d_ptr, st))) return rc;
    if (K > 0) {
      k_cps_gather<<<cdiv(K, 256), 256, 0, st>>>(d_perm, d_meas, d_ids, d_cv, K, o_view, o_id, o_mpos);
      V3DBA_LAUNCH_CHECK();
    }
    if ((rc = down_copy(track_ptr, d_ptr, (size_t)M + 1, st)) || (rc = down_copy(meas_view, o_view, (size_t)K, st)) ||
        (rc = down_copy(meas_id, o_id, (size_t)K, st)) || (rc = down_copy(meas_pos, o_mpos, 2 * (size_t)K, st)))
      return rc;
    V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
    if (M) std::memcpy(track_pos, points3d, sizeof(double) * 3 * (size_t)M);
    return V3DBA_OK;
  }
  // in place: the tracks keep their measurement lists; kept track xs[i] is updated
  const int M = n_points;
  if (n_tracks < 0 || (M && !xs_indices) || !valid_track_ptr(track_ptr, n_tracks)) return V3DBA_ERR_INVALID_INPUT;
  const int KT = track_ptr[n_tracks];
  if (KT && !meas_pos) return V3DBA_ERR_INVALID_ARGUMENT;
  long need = 0;
  for (int i = 0; i < M; ++i) {
    if (xs_indices[i] < 0 || xs_indices[i] >= n_tracks) return V3DBA_ERR_INVALID_INPUT;
    need += track_ptr[xs_indices[i] + 1] - track_ptr[xs_indices[i]];
  }
  if (need > n_measurements) return V3DBA_ERR_INVALID_INPUT;
  int *d_ptr, *d_xs, *d_off;
  double *d_pts, *d_meas, *d_pos;
  float* d_mpos;
  if ((rc = up_copy(sc, &d_ptr, (const int*)track_ptr, (size_t)n_tracks + 1, st)) ||
      (rc = up_copy(sc, &d_xs, xs_indices, (size_t)M, st)) || (rc = sc.get(&d_off, (size_t)M + 1)) ||
      (rc = up_copy(sc, &d_pts, points3d, 3 * (size_t)M, st)) ||
      (rc = up_copy(sc, &d_meas, measurements, 2 * (size_t)n_measurements, st)) ||
      (rc = up_copy(sc, &d_pos, (const double*)track_pos, 3 * (size_t)n_tracks, st)) ||
      (rc = up_copy(sc, &d_mpos, (const float*)meas_pos, 2 * (size_t)KT, st)))
    return rc;
  k_cps_lengths<<<cdiv(M + 1, 256), 256, 0, st>>>(d_ptr, d_xs, M, d_off);
  V3DBA_LAUNCH_CHECK();
  if ((rc = scan_exclusive(sc, d_off, M + 1, st))) return rc;
  if (M > 0) {
    k_cps_inplace<<<cdiv(M, 128), 128, 0, st>>>(d_ptr, d_xs, d_off, M, d_pts, d_meas, d_pos, d_mpos);
    V3DBA_LAUNCH_CHECK();
  }
  if ((rc = down_copy(track_pos, d_pos, 3 * (size_t)n_tracks, st)) || (rc = down_copy(meas_pos, d_mpos, 2 * (size_t)KT, st)))
    return rc;
  V3DBA_CUDA_TRY(cudaStreamSynchronize(st));
  return V3DBA_OK;
}
