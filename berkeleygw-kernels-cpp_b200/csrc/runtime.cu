// runtime.cu -- options, per-device workspace cache, host<->device staging
// and status handling shared by every libbgwsigma entry point.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

#include <thread>
#include <vector>

#include "bgw_internal.cuh"

namespace bgw {

std::atomic<uint64_t> g_launches{0};

namespace {
std::atomic<long long> g_stall_step{-1};  // bgw_debug_inject_stall
}  // namespace
long long stall_step() { return g_stall_step.load(std::memory_order_relaxed); }

void note_cuda_error(cudaError_t e, const char *what, const char *file, int line) {
  if (std::getenv("BGW_SIGMA_QUIET") == nullptr)
    std::fprintf(stderr, "libbgwsigma: %s failed: %s (%s:%d)\n", what, cudaGetErrorString(e), file, line);
}

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_ws_mu;
std::unique_ptr<Workspace> g_ws[kMaxDevices];
}  // namespace

Workspace *workspace_for(int device) {
  if (device < 0 || device >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lk(g_ws_mu);
  if (!g_ws[device]) {
    g_ws[device].reset(new Workspace());
    g_ws[device]->device = device;
  }
  return g_ws[device].get();
}

int ws_reserve_pinned(Workspace *ws, size_t bytes, void **out) {
  if (bytes == 0) bytes = 256;
  if (ws->pinned_cap < bytes) {
    if (ws->pinned) {
      BGW_CUDA_TRY(cudaDeviceSynchronize());
      BGW_CUDA_TRY(cudaFreeHost(ws->pinned));
      ws->pinned = nullptr;
      ws->pinned_cap = 0;
    }
    cudaError_t e = cudaHostAlloc(&ws->pinned, bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      ws->pinned = nullptr;
      return BGW_ERR_ALLOC;
    }
    ws->pinned_cap = bytes;
  }
  *out = ws->pinned;
  return BGW_OK;
}

int ws_reserve(Workspace *ws, int s, size_t bytes, void **out) {
  if (bytes == 0) bytes = 256;
  if (ws->cap[s] < bytes) {
    if (ws->buf[s]) {
      // The old buffer may still be read by an earlier call's kernels.
      BGW_CUDA_TRY(cudaDeviceSynchronize());
      BGW_CUDA_TRY(cudaFree(ws->buf[s]));
      ws->buf[s] = nullptr;
      ws->cap[s] = 0;
    }
    size_t rounded = (bytes + 255) & ~size_t(255);
    cudaError_t e = cudaMalloc(&ws->buf[s], rounded);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      ws->buf[s] = nullptr;
      return BGW_ERR_ALLOC;
    }
    ws->cap[s] = rounded;
  }
  *out = ws->buf[s];
  return BGW_OK;
}

int ws_acquire(Workspace *ws, cudaStream_t stream) {
  if (!ws->last_use) {
    BGW_CUDA_TRY(cudaEventCreateWithFlags(&ws->last_use, cudaEventDisableTiming));
    for (auto &e : ws->prof) BGW_CUDA_TRY(cudaEventCreate(&e));
    BGW_CUDA_TRY(cudaDeviceGetAttribute(&ws->sm_count, cudaDevAttrMultiProcessorCount, ws->device));
    return BGW_OK;
  }
  BGW_CUDA_TRY(cudaStreamWaitEvent(stream, ws->last_use, 0));
  return BGW_OK;
}

int ws_copy_stream(Workspace *ws, cudaStream_t *out) {
  if (!ws->copy_stream) {
    BGW_CUDA_TRY(cudaStreamCreateWithFlags(&ws->copy_stream, cudaStreamNonBlocking));
    BGW_CUDA_TRY(cudaEventCreateWithFlags(&ws->copy_start, cudaEventDisableTiming));
    for (auto &e : ws->chunk_ready) BGW_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : ws->stage_free) BGW_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  *out = ws->copy_stream;
  return BGW_OK;
}

int ws_release(Workspace *ws, cudaStream_t stream) {
  BGW_CUDA_TRY(cudaEventRecord(ws->last_use, stream));
  return BGW_OK;
}

namespace {
thread_local bgw_profile t_last_profile = {};
}

void set_last_profile(const bgw_profile &p) { t_last_profile = p; }

int prof_mark(CallEnv *env, int which) {
  if (!env->profile) return BGW_OK;
  BGW_CUDA_TRY(cudaEventRecord(env->ws->prof[which], env->stream));
  return BGW_OK;
}

int begin_call(const bgw_options *user, CallEnv *env) {
  bgw_options_init(&env->opt);
  if (user) {
    if (user->struct_size < (int32_t)offsetof(bgw_options, device_status) + (int32_t)sizeof(int32_t *))
      return BGW_ERR_INVALID_ARG;
    // A caller built against a shorter bgw_options keeps the defaults of
    // the fields it does not have.
    std::memcpy(&env->opt, user, std::min<size_t>((size_t)user->struct_size, sizeof(bgw_options)));
    env->opt.struct_size = (int32_t)sizeof(bgw_options);
  }
  const bgw_options &o = env->opt;
  if (o.memory != BGW_MEMORY_HOST && o.memory != BGW_MEMORY_DEVICE) return BGW_ERR_INVALID_ARG;
  if (o.precision != BGW_PRECISION_FP64 && o.precision != BGW_PRECISION_MIXED) return BGW_ERR_INVALID_ARG;
  if (o.gpp_algorithm != BGW_GPP_BANDLOOP && o.gpp_algorithm != BGW_GPP_FACTORED && o.gpp_algorithm != BGW_GPP_AUTO)
    return BGW_ERR_INVALID_ARG;
  if (o.wx_band_stride < 0) return BGW_ERR_INVALID_ARG;
  if (!(o.pole_guard >= 0.0) || !std::isfinite(o.pole_guard)) return BGW_ERR_INVALID_ARG;
  if (o.mixed_order < 0 || o.mixed_order > 3) return BGW_ERR_INVALID_ARG;
  if ((o.flags & BGW_FLAG_ASYNC) && (o.memory != BGW_MEMORY_DEVICE || o.device_status == nullptr))
    return BGW_ERR_INVALID_ARG;
  if ((o.flags & BGW_FLAG_PROFILE) && (o.flags & BGW_FLAG_ASYNC)) return BGW_ERR_INVALID_ARG;
  env->profile = (o.flags & BGW_FLAG_PROFILE) != 0;
  env->launches0 = g_launches.load();
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    (void)cudaGetLastError();
    return BGW_ERR_NO_DEVICE;
  }
  int dev = o.device;
  if (dev < 0) BGW_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= ndev) return BGW_ERR_INVALID_ARG;
  BGW_CUDA_TRY(cudaSetDevice(dev));
  env->device = dev;
  env->stream = static_cast<cudaStream_t>(o.stream);
  env->host = (o.memory == BGW_MEMORY_HOST);
  env->ws = workspace_for(dev);
  if (!env->ws) return BGW_ERR_INVALID_ARG;
  return BGW_OK;
}

void parallel_ranges(int64_t n, int parts, const std::function<void(int64_t, int64_t)> &fn) {
  parts = (int)std::max<int64_t>(1, std::min<int64_t>(parts, n));
  std::vector<std::thread> pool;
  for (int t = 1; t < parts; ++t) pool.emplace_back(fn, n * t / parts, n * (t + 1) / parts);
  fn(0, n / parts);
  for (auto &th : pool) th.join();
}

int host_threads(int64_t work_items, int64_t per_thread) {
  return (int)std::max<int64_t>(
      1, std::min<int64_t>({16, (int64_t)std::thread::hardware_concurrency(), work_items / per_thread}));
}

bool is_pageable(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return true;
  }
  return at.type == cudaMemoryTypeUnregistered;
}

void parallel_memcpy(void *dst, const void *src, size_t bytes) {
  const int64_t pieces = (int64_t)((bytes + (1 << 20) - 1) >> 20);
  parallel_ranges(pieces, host_threads(pieces, 4), [&](int64_t b0, int64_t b1) {
    const size_t lo = (size_t)b0 << 20, hi = std::min(bytes, (size_t)b1 << 20);
    if (hi > lo) std::memcpy(static_cast<char *>(dst) + lo, static_cast<const char *>(src) + lo, hi - lo);
  });
}

namespace {
constexpr size_t kStageSlot = size_t(32) << 20;        // bytes per page-locked slot
constexpr size_t kStageMin = size_t(8) << 20;          // smaller inputs: one plain copy
}  // namespace

int stage_input(CallEnv *env, int s, const void *src, size_t bytes, const void **dev_out) {
  if (!env->host) {
    if ((reinterpret_cast<uintptr_t>(src) & 15u) != 0) return BGW_ERR_INVALID_ARG;
    *dev_out = src;
    return BGW_OK;
  }
  void *d = nullptr;
  Workspace *ws = env->ws;
  BGW_TRY(ws_reserve(ws, s, bytes, &d));
  *dev_out = d;
  if (!bytes) return BGW_OK;
  if (bytes < kStageMin || !is_pageable(src)) {
    BGW_CUDA_TRY(cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, env->stream));
    return BGW_OK;
  }
  // Pageable: pieces of kStageSlot bytes, alternating between two slots; a
  // slot is refilled only after the DMA that read it has completed.
  cudaStream_t cs = nullptr;
  BGW_TRY(ws_copy_stream(ws, &cs));  // creates the slot events
  if (!ws->stage_slots) {
    cudaError_t e = cudaHostAlloc(&ws->stage_slots, 2 * kStageSlot, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      ws->stage_slots = nullptr;
      return BGW_ERR_ALLOC;
    }
  }
  for (size_t off = 0, k = 0; off < bytes; off += kStageSlot, ++k) {
    const size_t n = std::min(kStageSlot, bytes - off);
    const int slot = (int)(k & 1);
    BGW_CUDA_TRY(cudaEventSynchronize(ws->stage_free[slot]));
    char *buf = static_cast<char *>(ws->stage_slots) + (size_t)slot * kStageSlot;
    parallel_memcpy(buf, static_cast<const char *>(src) + off, n);
    BGW_CUDA_TRY(cudaMemcpyAsync(static_cast<char *>(d) + off, buf, n, cudaMemcpyHostToDevice, env->stream));
    BGW_CUDA_TRY(cudaEventRecord(ws->stage_free[slot], env->stream));
  }
  return BGW_OK;
}

int finish_call(CallEnv *env) {
  BGW_TRY(ws_release(env->ws, env->stream));
  if (env->opt.flags & BGW_FLAG_ASYNC) {
    BGW_CUDA_TRY(cudaMemcpyAsync(env->opt.device_status, env->d_status, sizeof(int32_t),
                                 cudaMemcpyDeviceToDevice, env->stream));
    BGW_CUDA_TRY(cudaGetLastError());
    return BGW_OK;
  }
  int32_t st[STATUS_WORDS] = {0, 0, 0, 0};
  BGW_TRY(prof_mark(env, 3));
  BGW_CUDA_TRY(cudaMemcpyAsync(st, env->d_status, sizeof(st), cudaMemcpyDeviceToHost, env->stream));
  BGW_CUDA_TRY(cudaStreamSynchronize(env->stream));
  BGW_CUDA_TRY(cudaGetLastError());
  if (env->profile) {
    float a = 0.f, b = 0.f;
    BGW_CUDA_TRY(cudaEventElapsedTime(&a, env->ws->prof[1], env->ws->prof[2]));
    BGW_CUDA_TRY(cudaEventElapsedTime(&b, env->ws->prof[0], env->ws->prof[3]));
    env->prof.main_kernel_ms = a;
    env->prof.device_ms = b;
    env->prof.total_launches = (int32_t)(g_launches.load() - env->launches0);
    t_last_profile = env->prof;
  }
  return st[0];
}

}  // namespace bgw

extern "C" {

void bgw_options_init(bgw_options *opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->struct_size = (int32_t)sizeof(bgw_options);
  opt->memory = BGW_MEMORY_HOST;
  opt->precision = BGW_PRECISION_FP64;
  opt->gpp_algorithm = BGW_GPP_AUTO;
  opt->wx_band_stride = 0;
  opt->device = -1;
  opt->flags = 0;
  opt->stream = nullptr;
  opt->device_status = nullptr;
  opt->pole_guard = 0.0;
  opt->mixed_order = 3;
}

const char *bgw_status_string(int status) {
  switch (status) {
    case BGW_OK: return "success";
    case BGW_ERR_INVALID_ARG: return "invalid argument";
    case BGW_ERR_INDEX: return "index out of range (inv_igp_index/indinv)";
    case BGW_ERR_CUDA: return "CUDA runtime error";
    case BGW_ERR_ALLOC: return "allocation failed";
    case BGW_ERR_NO_DEVICE: return "no usable CUDA device";
    case BGW_ERR_TIMEOUT: return "device-side wait timed out";
    case BGW_ERR_UNSUPPORTED: return "unsupported option combination";
    case BGW_ERR_CHECK: return "debug-build bounds check failed";
    default: return "unknown status";
  }
}

int bgw_abi_version(void) { return BGW_SIGMA_ABI_VERSION; }

int bgw_last_profile(bgw_profile *out) {
  if (!out) return BGW_ERR_INVALID_ARG;
  *out = bgw::t_last_profile;
  return BGW_OK;
}

uint64_t bgw_launch_count(void) { return bgw::g_launches.load(); }

int bgw_debug_inject_stall(int64_t step) {
  if (step < -1) return BGW_ERR_INVALID_ARG;
  bgw::g_stall_step.store((long long)step, std::memory_order_relaxed);
  return BGW_OK;
}

int bgw_release_workspace(int32_t device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
    (void)cudaGetLastError();
    return BGW_ERR_NO_DEVICE;
  }
  for (int d = 0; d < ndev && d < 64; ++d) {
    if (device >= 0 && d != device) continue;
    bgw::Workspace *ws = bgw::workspace_for(d);
    std::lock_guard<std::mutex> lk(ws->mu);
    BGW_CUDA_TRY(cudaSetDevice(d));
    BGW_CUDA_TRY(cudaDeviceSynchronize());
    for (int s = 0; s < bgw::SLOT_COUNT; ++s) {
      if (ws->buf[s]) BGW_CUDA_TRY(cudaFree(ws->buf[s]));
      ws->buf[s] = nullptr;
      ws->cap[s] = 0;
    }
    if (ws->pinned) BGW_CUDA_TRY(cudaFreeHost(ws->pinned));
    ws->pinned = nullptr;
    ws->pinned_cap = 0;
    if (ws->stage_slots) BGW_CUDA_TRY(cudaFreeHost(ws->stage_slots));
    ws->stage_slots = nullptr;
  }
  return BGW_OK;
}

}  // extern "C"
