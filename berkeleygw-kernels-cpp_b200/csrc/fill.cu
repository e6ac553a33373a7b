// fill.cu -- seeded input generation on the GPU (bgw_fill_uniform).
//
// The reference drivers fill their ArrayMD inputs on the host, one thread,
// before every run (GPP/gpp.cpp:246-275, FF/ff.cpp:585-633).  Here the large
// arrays are generated where they are used: a counter-based generator gives
// every element its own random word, so any sub-block of an array (a rank's
// G' rows, a chunk) is produced without generating the rest, and the values
// are independent of the grid, the device and the order of generation.
//
// Generator: Philox4x64-10 (J. K. Salmon, M. A. Moraes, R. O. Dror and
// D. E. Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11): a block
// of four 64-bit words is 10 rounds of two 64 x 64 -> 128-bit products over
// the counter, with the 128-bit key bumped by two Weyl constants between
// rounds.  Word w of stream (seed, stream) is word w % 4 of the block with
// counter (w / 4 + 1, 0, 0, 0) and key (seed, stream) -- the sequence of
// numpy's Philox bit generator with key seed + stream * 2^64, which is
// therefore the host twin of this kernel.  Word -> double: u = (word >> 11)
// * 2^-53 in [0, 1) (exact), then lo + (hi - lo) * u with two separately
// rounded operations (no contraction), as numpy's Generator.random followed
// by `a *= hi - lo; a += lo`.
#include <algorithm>

#include "bgw_internal.cuh"

namespace bgw {
namespace {

struct Words4 {
  unsigned long long v[4];
};

__device__ __forceinline__ Words4 philox4x64_10(unsigned long long ctr, unsigned long long k0, unsigned long long k1) {
  constexpr unsigned long long kM0 = 0xD2E7470EE14C6C93ULL, kM1 = 0xCA5A826395121157ULL;  // round multipliers
  constexpr unsigned long long kW0 = 0x9E3779B97F4A7C15ULL, kW1 = 0xBB67AE8584CAA73BULL;  // key Weyl increments
  unsigned long long x0 = ctr, x1 = 0, x2 = 0, x3 = 0;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += kW0;
      k1 += kW1;
    }
    const unsigned long long lo0 = kM0 * x0, hi0 = __umul64hi(kM0, x0);
    const unsigned long long lo1 = kM1 * x2, hi1 = __umul64hi(kM1, x2);
    x0 = hi1 ^ x1 ^ k0;
    x1 = lo1;
    x2 = hi0 ^ x3 ^ k1;
    x3 = lo0;
  }
  return {{x0, x1, x2, x3}};
}

__device__ __forceinline__ double to_range(unsigned long long w, double lo, double scale) {
  const double u = (double)(w >> 11) * 0x1.0p-53;
  return __dadd_rn(__dmul_rn(u, scale), lo);
}

// out[i] (i < n) = value of word off + i; even words use (lo0, sc0), odd
// words (lo1, sc1): the real and imaginary parts of an interleaved complex
// array.  One thread per Philox block; consecutive threads write
// consecutive 32-byte runs (two 16-byte stores when aligned).
__global__ void __launch_bounds__(256) fill_uniform_kernel(double *__restrict__ out, long long n,
                                                           unsigned long long seed, unsigned long long stream,
                                                           long long off, double lo0, double sc0, double lo1,
                                                           double sc1) {
  const long long b0 = off >> 2, b1 = (off + n + 3) >> 2;
  const bool vec = (off & 3) == 0 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
  for (long long b = b0 + blockIdx.x * (long long)blockDim.x + threadIdx.x; b < b1;
       b += (long long)gridDim.x * blockDim.x) {
    const Words4 r = philox4x64_10((unsigned long long)b + 1ULL, seed, stream);
    const long long i0 = 4 * b - off;
    const double v0 = to_range(r.v[0], lo0, sc0), v1 = to_range(r.v[1], lo1, sc1);
    const double v2 = to_range(r.v[2], lo0, sc0), v3 = to_range(r.v[3], lo1, sc1);
    if (vec && i0 + 4 <= n) {
      reinterpret_cast<double2 *>(out + i0)[0] = make_double2(v0, v1);
      reinterpret_cast<double2 *>(out + i0)[1] = make_double2(v2, v3);
    } else {
      const double v[4] = {v0, v1, v2, v3};
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        const long long i = i0 + l;
        if (i >= 0 && i < n) out[i] = v[l];
      }
    }
  }
}

}  // namespace

// Enqueues the fill of `n` doubles at device pointer `out` (words off ..
// off + n - 1 of stream (seed, stream)) on env->stream.
int fill_uniform_enqueue(CallEnv *env, double *out, int64_t n, uint64_t seed, uint64_t stream, int64_t off,
                         double lo_even, double hi_even, double lo_odd, double hi_odd) {
  if (n <= 0) return BGW_OK;
  const long long blocks = ((off + n + 3) >> 2) - (off >> 2);
  const int grid = (int)std::min<long long>((blocks + 255) / 256, (long long)env->ws->sm_count * 8);
  fill_uniform_kernel<<<std::max(grid, 1), 256, 0, env->stream>>>(out, n, seed, stream, off, lo_even,
                                                                   hi_even - lo_even, lo_odd, hi_odd - lo_odd);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

}  // namespace bgw
