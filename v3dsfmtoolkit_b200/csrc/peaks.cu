// Benchmark support: the FP64 tensor-core (DMMA) throughput of this GPU and the executed work of
// a reduced-system factorisation, the denominators / numerators of the Cholesky roofline.
#include <cstdio>

#include "common.cuh"
#include "lm.cuh"

namespace v3dba {
namespace {

// Every warp issues long chains of independent mma.sync.m8n8k4.f64 on register operands.
__global__ void __launch_bounds__(256) k_dmma_peak(int iters, double* sink) {
  const int lane = threadIdx.x & 31;
  double a = 1.0 + 1e-3 * lane, b = 1.0 - 1e-3 * lane;
  double c[8][2];
#pragma unroll
  for (int t = 0; t < 8; ++t) c[t][0] = c[t][1] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int t = 0; t < 8; ++t)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(c[t][0]), "+d"(c[t][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < 8; ++t) s += c[t][0] + c[t][1];
  if (s == 1234.5) sink[blockIdx.x] = s;   // keeps the work alive
}

// Every thread runs 8 independent chains of FP64 FMAs on registers.
__global__ void __launch_bounds__(256) k_dfma_peak(int iters, double* sink) {
  double v[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) v[t] = 1.0 + 1e-3 * (threadIdx.x + t);
  const double a = 0.999999, b = 1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int t = 0; t < 8; ++t) v[t] = fma(v[t], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < 8; ++t) s += v[t];
  if (s == 1234.5) sink[blockIdx.x] = s;   // keeps the work alive
}

}  // namespace
}  // namespace v3dba

using namespace v3dba;

extern "C" int v3dba_measure_fp64_mma_peak(double* tflops) {
  if (!tflops) return V3DBA_ERR_INVALID_ARGUMENT;
  int dev = 0, sms = 148;
  V3DBA_CUDA_TRY(cudaGetDevice(&dev));
  V3DBA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double* sink = nullptr;
  V3DBA_CUDA_TRY(cudaMalloc(&sink, sizeof(double) * sms * 8));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 4, iters = 4096;
  k_dmma_peak<<<blocks, 256>>>(16, sink);   // warm-up
  note_launches(1);
  cudaEventRecord(e0);
  k_dmma_peak<<<blocks, 256>>>(iters, sink);
  note_launches(1);
  cudaEventRecord(e1);
  const cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) return V3DBA_ERR_CUDA;
  const double flops = 2.0 * 256.0 * 8.0 * iters * (blocks * 8.0);   // 8x8x4 FMA per mma, 8 warps per block
  *tflops = flops / (ms * 1e-3) / 1e12;
  return V3DBA_OK;
}

// The FP64 FMA-pipe throughput of this GPU (TFLOP/s, 2 flops per FMA): the roofline denominator of
// the batched triplet adjuster, whose per-point work is scalar FP64.
extern "C" int v3dba_measure_fp64_fma_peak(double* tflops) {
  if (!tflops) return V3DBA_ERR_INVALID_ARGUMENT;
  int dev = 0, sms = 148;
  V3DBA_CUDA_TRY(cudaGetDevice(&dev));
  V3DBA_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double* sink = nullptr;
  V3DBA_CUDA_TRY(cudaMalloc(&sink, sizeof(double) * sms * 8));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 8, iters = 16384;
  k_dfma_peak<<<blocks, 256>>>(64, sink);   // warm-up
  note_launches(1);
  cudaEventRecord(e0);
  k_dfma_peak<<<blocks, 256>>>(iters, sink);
  note_launches(1);
  cudaEventRecord(e1);
  const cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) return V3DBA_ERR_CUDA;
  const double flops = 2.0 * 8.0 * iters * (double)blocks * 256.0;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return V3DBA_OK;
}
