// bgw_internal.cuh -- shared host/device helpers of libbgwsigma (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <functional>
#include <cstddef>
#include <mutex>

#include "bgw_sigma.h"

namespace bgw {

// ------------------------------------------------------------ host status --

// Launch counter exported through bgw_launch_count().
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t n = 1) { g_launches.fetch_add(n, std::memory_order_relaxed); }

#define BGW_CUDA_TRY(expr)                                   \
  do {                                                       \
    cudaError_t bgw_e_ = (expr);                             \
    if (bgw_e_ != cudaSuccess) {                             \
      ::bgw::note_cuda_error(bgw_e_, #expr, __FILE__, __LINE__); \
      return BGW_ERR_CUDA;                                   \
    }                                                        \
  } while (0)

#define BGW_TRY(expr)              \
  do {                             \
    int bgw_s_ = (expr);           \
    if (bgw_s_ != BGW_OK) return bgw_s_; \
  } while (0)

void note_cuda_error(cudaError_t e, const char *what, const char *file, int line);

// Device-side status word layout (int32[4] in the workspace):
//   [0] first error code raised by a kernel (BGW_ERR_INDEX, BGW_ERR_TIMEOUT)
//   [1] detail (e.g. the offending index position)
enum { STATUS_WORDS = 4 };

__device__ __forceinline__ void raise_status(int *status, int code, int detail) {
  if (atomicCAS(status, 0, code) == 0) status[1] = detail;
}

// Debug build (-DBGW_CHECK, lib/libbgwsigma_check.so): BGW_CHECKED(cond,
// status, site) is `cond`; when it is false the kernel raises BGW_ERR_CHECK
// with the site code as the status detail, and the caller skips the access
// the check guards.  In the product build it is `true` and compiles away.
#ifdef BGW_CHECK
#define BGW_CHECKED(cond, status, site) \
  ((cond) ? true : (::bgw::raise_status((status), BGW_ERR_CHECK, (site)), false))
#else
#define BGW_CHECKED(cond, status, site) true
#endif

// ------------------------------------------------------------- workspace --
//
// One grow-only set of device buffers per device, reused across calls.  A
// call holds the device's mutex while it enqueues work; `last_use` orders a
// later call on another stream after the previous call's kernels.
enum Slot {
  SLOT_STATUS = 0,
  SLOT_PARTIALS,
  SLOT_TABLE0,
  SLOT_TABLE1,
  SLOT_TABLE2,
  SLOT_PLAN,
  SLOT_IN0,  // host-memory staging of inputs
  SLOT_IN1,
  SLOT_IN2,
  SLOT_IN3,
  SLOT_IN4,
  SLOT_IN5,
  SLOT_IN6,
  SLOT_IN7,
  SLOT_IN8,
  SLOT_IN9,
  SLOT_IN10,
  SLOT_IN11,
  SLOT_OUT,
  SLOT_COUNT
};

struct Workspace {
  std::mutex mu;
  void *buf[SLOT_COUNT] = {};
  size_t cap[SLOT_COUNT] = {};
  cudaEvent_t last_use = nullptr;
  cudaEvent_t prof[4] = {};  // call start, main start, main stop, call stop
  cudaStream_t copy_stream = nullptr;  // host-input staging (non-blocking)
  cudaEvent_t copy_start = nullptr;
  cudaEvent_t chunk_ready[16] = {};
  cudaEvent_t stage_free[2] = {};  // page-locked staging slot reusable
  int sm_count = 0;
  int device = -1;
  void *pinned = nullptr;  // page-locked host staging (grow-only)
  size_t pinned_cap = 0;
  void *stage_slots = nullptr;  // two page-locked slots for stage_input
};

// Returns the workspace of `device` (created on first use).
Workspace *workspace_for(int device);
// Ensures slot `s` holds at least `bytes` (256-byte aligned); grow-only.
int ws_reserve(Workspace *ws, int s, size_t bytes, void **out);
// Ensures the page-locked host staging buffer holds `bytes`; grow-only.  The
// caller must not overwrite it while an earlier copy from it is in flight.
int ws_reserve_pinned(Workspace *ws, size_t bytes, void **out);
// Makes `stream` wait for the previous user of the workspace, and records
// this call as the new last user (call after enqueuing).
int ws_acquire(Workspace *ws, cudaStream_t stream);
// The workspace's copy stream and its events (created on first use).
int ws_copy_stream(Workspace *ws, cudaStream_t *out);
int ws_release(Workspace *ws, cudaStream_t stream);

// ------------------------------------------------------ call environment --
struct CallEnv {
  bgw_options opt;
  int device = 0;
  cudaStream_t stream = nullptr;
  Workspace *ws = nullptr;
  bool host = true;
  bool profile = false;
  int *d_status = nullptr;  // device status words
  uint64_t launches0 = 0;   // g_launches at the start of the call
  bgw_profile prof = {};    // filled by the enqueue functions / finish_call
};

// Profiling marks (no-ops unless BGW_FLAG_PROFILE).
int prof_mark(CallEnv *env, int which);
// Stores `p` as this thread's last profile (bgw_last_profile).
void set_last_profile(const bgw_profile &p);

// Validates options, selects the device, fetches the workspace.
int begin_call(const bgw_options *user, CallEnv *env);
// Copies `bytes` from a host or device input into a device pointer usable
// by kernels (host memory: staged into slot `s`; large pageable inputs go
// through two page-locked slots filled by several host threads, so the host
// copy of one piece overlaps the DMA of the previous one).
int stage_input(CallEnv *env, int s, const void *src, size_t bytes, const void **dev_out);

// Runs fn(i0, i1) over [0, n) in `parts` contiguous ranges, one host thread
// each (the calling thread takes the first).
void parallel_ranges(int64_t n, int parts, const std::function<void(int64_t, int64_t)> &fn);
// Host threads for `work_items` items of which each thread should get at
// least `per_thread` (at most 16 and the hardware concurrency).
int host_threads(int64_t work_items, int64_t per_thread);
// True when `p` is host memory that CUDA has not page-locked.
bool is_pageable(const void *p);
// memcpy of `bytes` by several host threads (1 MiB pieces).
void parallel_memcpy(void *dst, const void *src, size_t bytes);
// Synchronous completion: waits for the stream, reads the device status.
int finish_call(CallEnv *env);

// ---------------------------------------------------------- device math --

// Reciprocal of a positive, normal double without a divide instruction.
// y0 = rcp.approx.ftz.f64 (the PTX ISA's documented approximate reciprocal),
// refined by one third-order Newton-Raphson / Householder step for f(y) =
// 1/y - d: with e = 1 - d*y0, y = y0 (1 + e + e^2) = (1 - e^3) / d, so the
// relative error drops from |e| to |e|^3 (A. S. Householder, "The Numerical
// Treatment of a Single Nonlinear Equation", 1970, ch. 4; the same series
// is used for division by P. Markstein, "IA-64 and Elementary Functions",
// 2000, ch. 8).  Checked against the IEEE reciprocal on the GPU
// (bgw_debug_rcp_probe): at most 1 ulp from 1/d whenever 1/d is a normal
// double.  Flush to zero of the approximation: a zero or subnormal d gives a
// non-finite result, a d whose reciprocal is subnormal gives 0.
__device__ __forceinline__ double rcp_refined(double d) {
  double y0;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(d));
  double e = fma(-d, y0, 1.0);
  double s = fma(e, e, e);
  return fma(y0, s, y0);
}

// Bounded mbarrier / bulk-copy helpers (sm_90+ PTX).
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> shared (no multicast); bytes % 16 == 0, both
// addresses 16-byte aligned.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of `bar`; gives up after `max_cycles` SM clocks
// and returns false (the caller records BGW_ERR_TIMEOUT).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, long long max_cycles) {
  if (mbar_try_wait(bar, parity)) return true;
  long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > max_cycles) return false;
  }
  return true;
}

// About 2 s at the B200's 1.965 GHz boost clock.
constexpr long long kWaitCycles = 4000000000LL;

// Stall injection (bgw_debug_inject_stall; tests of the timeout path).
// Kernels that stage step j into buffer j & 1 of a double buffer take the
// CTA-local step index at which to stall (-1: never).  At that step the
// main-loop wait is made on `never`, an mbarrier no thread or copy ever
// arrives on, with a short budget: it runs out, and the kernel takes the
// same path as a real timeout (BGW_ERR_TIMEOUT, drain, exit).
constexpr long long kStallCycles = 200000;  // ~0.1 ms

// The main-loop wait of a double-buffered kernel for step j: phase
// (j >> 1) & 1 of `bar` (the buffer's barrier), or the injected stall.
__device__ __forceinline__ bool staged_wait(uint64_t *bar, long long j, long long stall, uint64_t *never) {
  if (j == stall) return mbar_wait_bounded(never, 0, kStallCycles);
  return mbar_wait_bounded(bar, (uint32_t)((j >> 1) & 1), kWaitCycles);
}

// After the wait for step j ran out: the copies still in flight are step
// j's, on bar[j & 1] with phase parity (j >> 1) & 1, and, if it was issued,
// step j + 1's, on bar[(j + 1) & 1] with parity ((j + 1) >> 1) & 1.  Both
// are waited for with the full budget, so no bulk copy writes into the
// CTA's shared memory after the CTA has exited.  (A wait for parity 0 on
// both barriers would be wrong: when a barrier's outstanding phase is odd,
// its completed parity-0 phase satisfies the wait at once.)
__device__ __forceinline__ void drain_staged(uint64_t *bar0, uint64_t *bar1, long long j, bool next_issued) {
  (void)mbar_wait_bounded((j & 1) ? bar1 : bar0, (uint32_t)((j >> 1) & 1), kWaitCycles);
  if (next_issued) (void)mbar_wait_bounded((j & 1) ? bar0 : bar1, (uint32_t)(((j + 1) >> 1) & 1), kWaitCycles);
}

// Host side: the stall step for kernels launched from now on (-1: off).
long long stall_step();

}  // namespace bgw
