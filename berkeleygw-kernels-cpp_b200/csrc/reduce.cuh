// reduce.cuh -- deterministic (fixed-order, atomic-free) reductions.
#pragma once

#include "bgw_internal.cuh"

namespace bgw {

// Butterfly sum over a warp; every lane ends with the same value and the
// combination order is fixed, so the result is reproducible bit for bit.
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums W doubles per thread over a block of NT threads.  `red` is shared
// scratch of (NT / 32) * W doubles.  Thread 0 returns the block totals in
// v[] (other threads' v[] are unspecified).  Order: warp butterfly, then the
// warp partials in warp order.
template <int W, int NT>
__device__ __forceinline__ void block_sum(double (&v)[W], double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < W; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < W; ++k) red[warp * W + k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < W; ++k) {
      double s = red[k];
      for (int w = 1; w < NT / 32; ++w) s += red[w * W + k];
      v[k] = s;
    }
  }
  __syncthreads();
}

// out[k] = sum_{i < n} partials[i * W + k] for k < W, in a fixed order
// (thread-strided sums, then block_sum).  One block of 256 threads.
template <int W>
__global__ void __launch_bounds__(256) reduce_partials_kernel(const double *__restrict__ partials, int n,
                                                              double *__restrict__ out) {
  __shared__ double red[8 * W];
  double v[W];
#pragma unroll
  for (int k = 0; k < W; ++k) v[k] = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) {
#pragma unroll
    for (int k = 0; k < W; ++k) v[k] += partials[(size_t)i * W + k];
  }
  block_sum<W, 256>(v, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < W; ++k) out[k] = v[k];
  }
}

}  // namespace bgw
