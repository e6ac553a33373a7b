// peak.cu -- FP64 throughput microkernels (DFMA and mma.sync m8n8k4 f64) and
// the reciprocal probe.
//
// The microkernels give the measured FP64 roofline denominators: every
// thread runs independent dependency chains long enough to hide pipeline
// latency, on a grid of 4 CTAs per SM.  2 flops per FMA; an m8n8k4 f64 MMA is
// 256 FMAs.  The probe evaluates the kernels' own reciprocals on given
// values, so their accuracy can be checked against the IEEE reciprocal.
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

// refined[i] = rcp_refined(in[i]) (the FP64 kernels' reciprocal), seed[i] =
// rcp.approx.ftz.f64(in[i]) (its starting value), f32[i] =
// rcp.approx.ftz.f32((float)in[i]) (the mixed remainder's reciprocal).
__global__ void rcp_probe_kernel(const double *__restrict__ in, long long n, double *__restrict__ refined,
                                 double *__restrict__ seed, float *__restrict__ f32) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = in[i];
    double y0;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(d));
    float yf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"((float)d));
    refined[i] = rcp_refined(d);
    seed[i] = y0;
    f32[i] = yf;
  }
}

}  // namespace
}  // namespace bgw

using namespace bgw;

extern "C" int bgw_debug_rcp_probe(const double *in, int64_t n, double *refined, double *seed, float *f32,
                                   int32_t device) {
  if (n < 0 || (n > 0 && (!in || !refined || !seed || !f32))) return BGW_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    (void)cudaGetLastError();
    return BGW_ERR_NO_DEVICE;
  }
  int dev = device;
  if (dev < 0) BGW_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= ndev) return BGW_ERR_INVALID_ARG;
  BGW_CUDA_TRY(cudaSetDevice(dev));
  if (n == 0) return BGW_OK;
  void *buf = nullptr;
  const size_t b8 = sizeof(double) * (size_t)n;
  BGW_CUDA_TRY(cudaMalloc(&buf, 3 * b8 + sizeof(float) * (size_t)n));
  double *d_in = static_cast<double *>(buf), *d_ref = d_in + n, *d_seed = d_ref + n;
  float *d_f = reinterpret_cast<float *>(d_seed + n);
  int rc = BGW_OK;
  if (cudaMemcpy(d_in, in, b8, cudaMemcpyHostToDevice) != cudaSuccess) rc = BGW_ERR_CUDA;
  if (rc == BGW_OK) {
    const int grid = (int)std::min<long long>((n + 255) / 256, 4096);
    rcp_probe_kernel<<<grid, 256>>>(d_in, n, d_ref, d_seed, d_f);
    count_launch();
    if (cudaGetLastError() != cudaSuccess || cudaMemcpy(refined, d_ref, b8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(seed, d_seed, b8, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(f32, d_f, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = BGW_ERR_CUDA;
  }
  (void)cudaGetLastError();
  BGW_CUDA_TRY(cudaFree(buf));
  return rc;
}

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
