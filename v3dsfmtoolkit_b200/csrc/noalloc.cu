// Dense SPD solve that allocates nothing: v3dba_dense_cholesky_solve_noalloc.
//
// Some callers cannot allocate device memory where they need a solve: a tracking or
// reconstruction loop that reserved all of its GPU memory up front (cudaMalloc can stall and
// synchronise the device, which a per-frame loop cannot afford), or a host framework that owns
// every device allocation and hands libraries only the buffers it manages.  This entry point
// serves them: the caller passes its own device buffers for the inputs and outputs, and every
// piece of working memory (the padded tiled matrix, the inverted diagonal tiles, the solution
// tiles and the tile schedule) lives in one fixed array compiled into the library
// (g_noalloc_scratch below).  Every GPU that loads the library holds that array, about
// 0.8 MB, until the process exits.
//
// Limits and sharing: n <= V3DBA_NOALLOC_MAX_N (256); larger systems are rejected.  All calls
// share the one array and it keeps the previous call's contents, so each call rewrites every
// entry it reads; two calls whose work overlaps on the GPU (different streams, or threads that
// do not serialise their calls) race on the array and must not be issued.  The first call on a
// device looks up the array's device address (cudaGetSymbolAddress) with that device current;
// make that first call before any stream capture.  The work is enqueued on the caller's stream
// and the call returns without waiting; synchronise the stream before reading x or fail.
#include <atomic>
#include <cstdio>

#include "common.cuh"
#include "lm.cuh"

namespace v3dba {
namespace {

constexpr int kNaMaxN = V3DBA_NOALLOC_MAX_N;
constexpr int kNaTB = 64;
constexpr int kNaMaxNt = kNaMaxN / kNaTB;                       // 4 tile columns
constexpr int kNaPad = kNaMaxNt * kNaTB;                        // 256
constexpr int kNaLd = kNaPad + kNaTB;                           // 320 (rhs tile row below)
constexpr size_t kNaMatrix = (size_t)kNaLd * kNaPad;            // working matrix
constexpr size_t kNaDiag = (size_t)kNaMaxNt * kNaTB * kNaTB;    // inverted diagonal tiles
constexpr size_t kNaX = kNaPad;                                 // solution tiles
constexpr size_t kNaInts = 256;                                 // tile schedule (as ints)
constexpr size_t kNaDoubles = kNaMatrix + kNaDiag + kNaX + kNaInts / 2;

// The fixed working memory of the entry point (device side; host code must not use its name as
// an address -- see scratch_address()).
static __device__ __align__(256) double g_noalloc_scratch[kNaDoubles];

// Copies the caller's row-major S (lower triangle used) and rhs into the padded column-major
// tiled layout: padding diagonal 1, every other unused entry 0, rhs as the first row of the
// tile row below the matrix.  Also clears the caller's failure flag.
__global__ void k_na_pack(const double* __restrict__ S, const double* __restrict__ rhs, int n, int n_pad, int ld,
                          int* __restrict__ fail) {
  double* W = g_noalloc_scratch;
  const size_t total = (size_t)ld * n_pad;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(e / ld), r = (int)(e % ld);
    double v = 0.0;
    if (r < n && c < n) v = (r >= c) ? S[(size_t)r * n + c] : 0.0;
    else if (r == c && r < n_pad) v = 1.0;
    else if (r == n_pad && c < n) v = rhs[c];
    W[e] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *fail = 0;
}

// The dense tile schedule for nt tile columns: at step k the panel rows are k+1..nt-1 and the
// rhs row nt; the trailing tiles are all pairs of them except (nt, nt).
__global__ void k_na_plan(int nt, int* __restrict__ ints) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int* pptr = ints;                 // nt + 1
  int* uptr = pptr + (kNaMaxNt + 1);  // nt + 1
  int* prows = uptr + (kNaMaxNt + 1);
  int* ur = prows + kNaMaxNt * (kNaMaxNt + 1);
  int* uc = ur + 64;
  int np = 0, nu = 0;
  pptr[0] = 0;
  uptr[0] = 0;
  for (int k = 0; k < nt; ++k) {
    const int first = np;
    for (int r = k + 1; r <= nt; ++r) prows[np++] = r;
    for (int a = first; a < np; ++a)
      for (int b = first; b <= a; ++b) {
        if (prows[a] == nt && prows[b] == nt) continue;
        ur[nu] = prows[a];
        uc[nu] = prows[b];
        ++nu;
      }
    pptr[k + 1] = np;
    uptr[k + 1] = nu;
  }
}

__global__ void k_na_unpack(const double* __restrict__ xs, int n, double* __restrict__ x) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = xs[i];
}

// Device address of g_noalloc_scratch for each device, looked up once per process with that
// device current and cached.  The cache entries are atomics: two host threads making their first
// call on one device at once both look the address up (the same value) and store it, with no data
// race.  The cached address belongs to the device's primary context; after a cudaDeviceReset the
// next call must come from a fresh process.
double* scratch_address(int dev) {
  constexpr int kMaxDevices = 64;
  static std::atomic<double*> addr[kMaxDevices];
  if (dev < 0 || dev >= kMaxDevices) return nullptr;
  double* a = addr[dev].load(std::memory_order_acquire);
  if (a == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      fprintf(stderr, "v3dba: cudaGetSymbolAddress of the no-allocation scratch failed: %s\n", cudaGetErrorString(e));
      return nullptr;
    }
    a = static_cast<double*>(p);
    addr[dev].store(a, std::memory_order_release);
  }
  return a;
}

}  // namespace
}  // namespace v3dba

using namespace v3dba;

extern "C" int v3dba_dense_cholesky_solve_noalloc(int n, const double* S, const double* rhs, double* x, int* fail,
                                                  void* stream) {
  if (n <= 0 || !S || !rhs || !x || !fail) return V3DBA_ERR_INVALID_ARGUMENT;
  if (n > kNaMaxN) {
    fprintf(stderr, "v3dba_dense_cholesky_solve_noalloc: n = %d exceeds the fixed scratch limit of %d\n", n, kNaMaxN);
    return V3DBA_ERR_INVALID_ARGUMENT;
  }
  int dev = 0;
  V3DBA_CUDA_TRY(cudaGetDevice(&dev));
  double* base = scratch_address(dev);
  if (!base) return V3DBA_ERR_CUDA;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nt = (n + kNaTB - 1) / kNaTB;
  TileChol tc;  // views into the fixed scratch; no memory of its own
  tc.n = n;
  tc.nt = nt;
  tc.n_pad = nt * kNaTB;
  tc.ld = tc.n_pad + kNaTB;
  double* W = base;
  tc.d_ldiag = base + kNaMatrix;
  double* xs = base + kNaMatrix + kNaDiag;
  int* ints = reinterpret_cast<int*>(base + kNaMatrix + kNaDiag + kNaX);
  tc.d_panel_ptr = ints;
  tc.d_upd_ptr = ints + (kNaMaxNt + 1);
  tc.d_panel_rows = ints + 2 * (kNaMaxNt + 1);
  tc.d_upd_r = tc.d_panel_rows + kNaMaxNt * (kNaMaxNt + 1);
  tc.d_upd_c = tc.d_upd_r + 64;
  k_na_pack<<<64, 256, 0, st>>>(S, rhs, n, tc.n_pad, tc.ld, fail);
  V3DBA_LAUNCH_CHECK();
  k_na_plan<<<1, 1, 0, st>>>(nt, ints);
  V3DBA_LAUNCH_CHECK();
  const int rc = chol_cluster_solve(tc, W, xs, fail, st);
  if (rc) return rc;
  k_na_unpack<<<1, 256, 0, st>>>(xs, n, x);
  V3DBA_LAUNCH_CHECK();
  return V3DBA_OK;
}
