// peak.cu -- FP64 throughput microkernels (DFMA and mma.sync m8n8k4 f64).
//
// They give the measured FP64 roofline denominators: every thread runs
// independent dependency chains long enough to hide pipeline latency, on a
// grid of 4 CTAs per SM.  2 flops per FMA; an m8n8k4 f64 MMA is 256 FMAs.
#include <algorithm>

#include "bgw_internal.cuh"

namespace bgw {
namespace {

constexpr int kPeakThreads = 256;

__global__ void __launch_bounds__(kPeakThreads) peak_dfma_kernel(double *out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = threadIdx.x * 1e-9 + j * 1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int j = 0; j < 8; ++j) x[j] = fma(x[j], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += x[j];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void __launch_bounds__(kPeakThreads) peak_dmma_kernel(double *out, int iters, double a, double b) {
  double c[8][2];
#pragma unroll
  for (int j = 0; j < 8; ++j) c[j][0] = c[j][1] = 0.0;
  const double av = a + threadIdx.x * 1e-12;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(c[j][0]), "+d"(c[j][1])
                   : "d"(av), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += c[j][0] + c[j][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace
}  // namespace bgw

using namespace bgw;

extern "C" int bgw_measure_fp64_peak(int32_t device, double *dfma_tflops, double *dmma_tflops) {
  if (!dfma_tflops || !dmma_tflops) return BGW_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    (void)cudaGetLastError();
    return BGW_ERR_NO_DEVICE;
  }
  int dev = device;
  if (dev < 0) BGW_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= ndev) return BGW_ERR_INVALID_ARG;
  BGW_CUDA_TRY(cudaSetDevice(dev));
  int sms = 0;
  BGW_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 4;
  double *out = nullptr;
  BGW_CUDA_TRY(cudaMalloc(&out, sizeof(double) * blocks * kPeakThreads));
  cudaEvent_t e0, e1;
  BGW_CUDA_TRY(cudaEventCreate(&e0));
  BGW_CUDA_TRY(cudaEventCreate(&e1));
  float ms = 0.f;
  double best_fma = 0.0, best_mma = 0.0;
  for (int rep = 0; rep < 3; ++rep) {
    const int it_f = 4000, it_m = 4000;
    BGW_CUDA_TRY(cudaEventRecord(e0));
    peak_dfma_kernel<<<blocks, kPeakThreads>>>(out, it_f, 0.999999, 1e-7);
    BGW_CUDA_TRY(cudaEventRecord(e1));
    BGW_CUDA_TRY(cudaEventSynchronize(e1));
    BGW_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    const double fma_flops = 2.0 * blocks * kPeakThreads * (double)it_f * 16 * 8;
    best_fma = std::max(best_fma, fma_flops / (ms * 1e-3) / 1e12);
    BGW_CUDA_TRY(cudaEventRecord(e0));
    peak_dmma_kernel<<<blocks, kPeakThreads>>>(out, it_m, 1.0, 1e-3);
    BGW_CUDA_TRY(cudaEventRecord(e1));
    BGW_CUDA_TRY(cudaEventSynchronize(e1));
    BGW_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    const double mma_flops = 512.0 * blocks * (kPeakThreads / 32) * (double)it_m * 8;
    best_mma = std::max(best_mma, mma_flops / (ms * 1e-3) / 1e12);
  }
  count_launch(6);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  BGW_CUDA_TRY(cudaFree(out));
  *dfma_tflops = best_fma;
  *dmma_tflops = best_mma;
  return BGW_OK;
}
