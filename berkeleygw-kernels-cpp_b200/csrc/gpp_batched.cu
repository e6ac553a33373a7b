// gpp_batched.cu -- many GPP instances (q-points of uneven ncouls and
// number_bands) in one persistent launch, replayed from a CUDA graph.
//
// Work list.  Instance i contributes P_i x nchunk_i items (G' row, chunk of
// kE*256 G); items are numbered globally, instance after instance.  The list
// is cut into `grid` contiguous ranges of equal estimated cost (bands x
// elements), one per persistent CTA.  A CTA walks its range item by item
// (band loop: also band chunk by band chunk), staging each step's tiles with
// 1-D bulk copies exactly as the single-instance kernel does, and keeps the
// running sums in registers.  When the next item belongs to another
// instance -- or the range ends -- it folds the sums with a fixed-order block
// reduction into a fixed slot (CTA, instance - first instance of the CTA).
// A finalize kernel sums, per instance, its slots in CTA order.  No atomics:
// a replay is bitwise identical.
//
// Tuning.  The elements per thread (kE) and with it the chunk width and the
// occupancy are chosen per batch by timing the candidate kernels on a sample
// prefix of the work list (bgw_gpp_batch_create): FP64 8, 4 or 2 (8: one CTA
// per SM, the per-band combination amortised over 24 terms); choices are
// cached per batch signature for the process.  The mixed form (the hoisted
// expansion of the single-instance band loop, K = mixed_order) runs at 16
// elements per thread over 512-band steps, as the single-instance kernel does.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "bgw_internal.cuh"
#include "gpp_common.cuh"
#include "reduce.cuh"

namespace bgw {

// Device-side description of one instance (all pointers device memory).
struct BatchInst {
  const double2 *wt, *ie, *am, *an;
  const double *vc, *wx;
  const int32_t *inv, *indinv;
  double *out;           // achtemp, 6 doubles
  double2 *tab;          // band loop: sch_store1 [P][nb]; factored: S[P]
  double4 *wx4;          // band loop: per-band frequencies [nb]
  long long indinv_len, wx_stride;
  long long item0;       // first global item
  long long col0;        // first global G' column
  int nb, P, G, nchunk;  // nchunk: G chunks per row
  int b_lo, b_hi;        // CTAs whose ranges cover this instance's items
  int pad[2];
};

namespace {

constexpr int kBThreads = 256;

__device__ __forceinline__ int find_inst(const BatchInst *__restrict__ inst, int n, long long item) {
  int lo = 0, hi = n - 1;  // last instance with item0 <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (inst[mid].item0 <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int find_col_inst(const BatchInst *__restrict__ inst, int n, long long col) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (inst[mid].col0 <= col) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// sch_store1 table (band loop) or its band sum S (factored) of every column
// of every instance: one warp per global column.
__global__ void __launch_bounds__(256)
    batch_prep_kernel(const BatchInst *__restrict__ inst, int n, long long total_cols, int factored, int *status) {
  const int lane = threadIdx.x & 31;
  const long long warps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long col = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; col < total_cols; col += warps) {
    const int i = find_col_inst(inst, n, col);
    const BatchInst &I = inst[i];
    const int p = (int)(col - I.col0);
    const int g = resolve_igp(p, I.inv, I.indinv, I.indinv_len, I.G, status);
    double sr = 0.0, si = 0.0;
    for (int n1 = lane; n1 < I.nb; n1 += 32) {
      double2 s = make_double2(0.0, 0.0);
      if (g >= 0) s = store1(I.am, I.an, I.vc, I.wt, n1, p, g, I.G);
      if (!factored) I.tab[(size_t)p * I.nb + n1] = s;
      sr += s.x;
      si += s.y;
    }
    if (factored) {
      sr = warp_sum(sr);
      si = warp_sum(si);
      if (lane == 0) I.tab[p] = make_double2(sr, si);
    }
  }
}

// Per-band frequency rows of every instance (band loop).
__global__ void batch_wx_kernel(const BatchInst *__restrict__ inst, int n) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const BatchInst &I = inst[i];
    for (int n1 = threadIdx.x; n1 < I.nb; n1 += blockDim.x) {
      const double *w = I.wx + (size_t)n1 * I.wx_stride;
      I.wx4[n1] = make_double4(w[0], w[1], w[2], 0.0);
    }
  }
}

// The mixed form reads its elements from global memory (as the
// single-instance mixed band loop does) and stages only the band rows.
template <int BCH, int KE, bool MIXED>
struct BatchSmem {
  double2 wt[2][MIXED ? 1 : kBThreads * KE];
  double2 ie[2][MIXED ? 1 : kBThreads * KE];
  double2 st[2][BCH];
  double4 wx[2][BCH];
  unsigned long long bar[3];  // [2]: never arrived on (stall injection)
  double red[(kBThreads / 32) * 18];
  double xr_lo[kBThreads / 32], xr_hi[kBThreads / 32];  // MIXED: chunk frequency range
  RemRow rows[MIXED ? BCH : 1];                          // MIXED: per-band remainder rows
};

// Flushes the running sums of instance slot `seg` of this CTA.
__device__ __forceinline__ void flush(double (&acc_r)[3], double (&acc_i)[3], double (&lo_r)[3], double (&lo_i)[3],
                                      double *red, double *__restrict__ partials, int max_seg, int seg) {
  double v[6] = {acc_r[0] + lo_r[0], acc_i[0] + lo_i[0], acc_r[1] + lo_r[1],
                 acc_i[1] + lo_i[1], acc_r[2] + lo_r[2], acc_i[2] + lo_i[2]};
  block_sum<6, kBThreads>(v, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) partials[((size_t)blockIdx.x * max_seg + seg) * 6 + k] = v[k];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) acc_r[k] = acc_i[k] = lo_r[k] = lo_i[k] = 0.0;
}

// Band loop over this CTA's range [range[b], range[b+1]) of the global item
// list.  Steps are (item, band chunk); step s+1 is staged while s computes.
template <int BCH, int KE, bool MIXED, int K = 3>
__global__ void __launch_bounds__(kBThreads, KE >= 8 ? 1 : 2)
    batch_bandloop_kernel(const BatchInst *__restrict__ inst, int n, const long long *__restrict__ range,
                          int max_seg, double *__restrict__ partials, int *status, long long stall) {
  constexpr int kCH = kBThreads * KE;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  auto &sm = *reinterpret_cast<BatchSmem<BCH, KE, MIXED> *>(smem_raw);
  const int tid = threadIdx.x;
  const long long j0 = range[blockIdx.x], j1 = range[blockIdx.x + 1];
  if (j0 >= j1) return;  // uniform per CTA: no barrier is skipped by some threads only
  if (tid == 0) {
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[0]), 1);
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[1]), 1);
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[2]), 1);
    fence_mbar_init();
  }
  __syncthreads();
  const int inst_lo = find_inst(inst, n, j0);

  struct Step {
    long long j;
    int i, c;
  };
  auto nbc_of = [&](int i) { return max(1, (inst[i].nb + BCH - 1) / BCH); };
  auto next = [&](Step s) {
    Step t = s;
    if (s.c + 1 < nbc_of(s.i)) {
      t.c = s.c + 1;
    } else {
      t.j = s.j + 1;
      t.c = 0;
      while (t.i + 1 < n && inst[t.i + 1].item0 <= t.j) ++t.i;
    }
    return t;
  };
  auto issue = [&](Step s, int buf) {
    const BatchInst &I = inst[s.i];
    const long long local = s.j - I.item0;
    const int p = (int)(local / I.nchunk);
    const int g0 = (int)(local % I.nchunk) * kCH;
    const int nvalid = min(kCH, I.G - g0);
    const int b0 = s.c * BCH;
    const int nbv = max(0, min(BCH, I.nb - b0));
    uint64_t *bar = reinterpret_cast<uint64_t *>(&sm.bar[buf]);
    if (!BGW_CHECKED(s.i >= 0 && s.i < n && local >= 0 && p < I.P && nvalid > 0 && nvalid <= kCH &&
                         g0 + nvalid <= I.G && nbv <= BCH,
                     status, 31)) {
      mbar_expect_tx(bar, 0);
      return;
    }
    mbar_expect_tx(bar, (MIXED ? 0u : 2u * nvalid * 16u) + nbv * 48u);
    if constexpr (!MIXED) {
      bulk_g2s(sm.wt[buf], I.wt + (size_t)p * I.G + g0, nvalid * 16u, bar);
      bulk_g2s(sm.ie[buf], I.ie + (size_t)p * I.G + g0, nvalid * 16u, bar);
    }
    if (nbv > 0) {
      bulk_g2s(sm.st[buf], I.tab + (size_t)p * I.nb + b0, nbv * 16u, bar);
      bulk_g2s(sm.wx[buf], I.wx4 + b0, nbv * 32u, bar);
    }
  };

  double acc_r[3] = {0.0, 0.0, 0.0}, acc_i[3] = {0.0, 0.0, 0.0};
  double lo_r[3] = {0.0, 0.0, 0.0}, lo_i[3] = {0.0, 0.0, 0.0};
  Step cur{j0, inst_lo, 0};
  bool ok = true;
  long long s_fail = 0;     // the step whose wait ran out
  bool next_issued = false;  // whether step s_fail + 1 was staged
  if (tid == 0) issue(cur, 0);
  for (long long s = 0;; ++s) {
    const int buf = (int)(s & 1);
    const Step nx = next(cur);
    const bool more = nx.j < j1;
    if (tid == 0 && more) issue(nx, buf ^ 1);
    if (!staged_wait(reinterpret_cast<uint64_t *>(&sm.bar[buf]), s, stall,
                     reinterpret_cast<uint64_t *>(&sm.bar[2]))) {
      raise_status(status, BGW_ERR_TIMEOUT, blockIdx.x);
      ok = false;
    }
    if (__syncthreads_or(!ok)) {
      s_fail = s;
      next_issued = more;
      break;
    }
    const BatchInst &I = inst[cur.i];
    const long long local = cur.j - I.item0;
    const int g0 = (int)(local % I.nchunk) * kCH;
    int nvalid = min(kCH, I.G - g0);
    int nbv = max(0, min(BCH, I.nb - cur.c * BCH));
    if (!BGW_CHECKED(nvalid <= kCH && nbv <= BCH, status, 32)) nvalid = nbv = 0;
    // MIXED: elements near the chunk's frequencies are summed in FP64.
    if constexpr (MIXED) {
      const double2 *wt_g = I.wt + (size_t)(local / I.nchunk) * I.G + g0;
      const double2 *ie_g = I.ie + (size_t)(local / I.nchunk) * I.G + g0;
      const RemStep rs = rem_stage<kBThreads, K>(sm.wx[buf], sm.st[buf], nbv, sm.rows, sm.red, sm.xr_lo, sm.xr_hi);
      RemElems<KE> e;
      const uint32_t near = rem_elems<KE, K>(e, wt_g, ie_g, nvalid, kBThreads, tid, rs, 0.0, acc_r, acc_i);
      rem_sweep<KE>(e, sm.rows, nbv, acc_r, acc_i, lo_r, lo_i);
      if (near) near_sweep(near, wt_g, ie_g, kBThreads, tid, sm.wx[buf], sm.st[buf], nbv, 0.0, acc_r,
                           acc_i, lo_r, lo_i);
    } else {
      Elem<double> e[KE];
      load_elems<double, KE>(e, sm.wt[buf], sm.ie[buf], nvalid, kBThreads, tid);
      band_sweep<KE>(e, sm.wx[buf], sm.st[buf], nbv, acc_r, acc_i);
    }
    __syncthreads();  // buffer `buf` is free for step s + 2
    if (!more || nx.i != cur.i) flush(acc_r, acc_i, lo_r, lo_i, sm.red, partials, max_seg, cur.i - inst_lo);
    if (!more) break;
    cur = nx;
  }
  if (!ok && tid == 0) {
    // Copies still in flight (steps s_fail and, if staged, s_fail + 1) land
    // before the CTA's shared memory is released.
    drain_staged(reinterpret_cast<uint64_t *>(&sm.bar[0]), reinterpret_cast<uint64_t *>(&sm.bar[1]), s_fail,
                 next_issued);
  }
}

// Factored form over the CTA's item range: HBM-bound stream, 128-bit loads.
template <int KE>
__global__ void __launch_bounds__(kBThreads, 4)
    batch_factored_kernel(const BatchInst *__restrict__ inst, int n, const long long *__restrict__ range,
                          int max_seg, double *__restrict__ partials) {
  constexpr int kCH = kBThreads * KE;
  __shared__ double red[(kBThreads / 32) * 6];
  const int tid = threadIdx.x;
  const long long j0 = range[blockIdx.x], j1 = range[blockIdx.x + 1];
  if (j0 >= j1) return;
  int i = find_inst(inst, n, j0);
  const int inst_lo = i;
  double acc_r[3] = {0.0, 0.0, 0.0}, acc_i[3] = {0.0, 0.0, 0.0};
  double lo_r[3] = {0.0, 0.0, 0.0}, lo_i[3] = {0.0, 0.0, 0.0};
  // The current instance's fields, kept in registers.
  long long item0 = inst[i].item0, next0 = i + 1 < n ? inst[i + 1].item0 : LLONG_MAX;
  int G = inst[i].G, nchunk = inst[i].nchunk;
  const double2 *wt = inst[i].wt, *ie = inst[i].ie, *tab = inst[i].tab;
  double x[3] = {inst[i].wx[0], inst[i].wx[1], inst[i].wx[2]};
  for (long long j = j0; j < j1; ++j) {
    if (next0 <= j) {
      while (i + 1 < n && inst[i + 1].item0 <= j) ++i;
      item0 = inst[i].item0;
      next0 = i + 1 < n ? inst[i + 1].item0 : LLONG_MAX;
      G = inst[i].G;
      nchunk = inst[i].nchunk;
      wt = inst[i].wt;
      ie = inst[i].ie;
      tab = inst[i].tab;
      x[0] = inst[i].wx[0];
      x[1] = inst[i].wx[1];
      x[2] = inst[i].wx[2];
    }
    const long long local = j - item0;
    const int p = (int)(local / nchunk);
    const int g0 = (int)(local % nchunk) * kCH;
    // All of the item's loads first (streamed once: evict-first), then the math.
    double2 w[KE], v[KE];
#pragma unroll
    for (int k = 0; k < KE; ++k) {
      const int ig = g0 + k * kBThreads + tid;
      const size_t at = (size_t)p * G + min(ig, G - 1);
      w[k] = __ldcs(wt + at);
      v[k] = __ldcs(ie + at);
      if (ig >= G) {
        w[k] = make_double2(0.0, 1.0);
        v[k] = make_double2(0.0, 0.0);
      }
    }
    double tr[3] = {0.0, 0.0, 0.0}, ti[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < KE; ++k) {
      const double wi2 = w[k].y * w[k].y, a = -w[k].y * v[k].y, b = w[k].y * v[k].x;
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        const double dr = x[iw] - w[k].x;
        const double r = rcp_refined(fma(dr, dr, wi2));
        tr[iw] = fma(fma(dr, v[k].x, a), r, tr[iw]);
        ti[iw] = fma(fma(dr, v[k].y, b), r, ti[iw]);
      }
    }
    const double2 s = tab[p];
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) {
      acc_r[iw] = fma(tr[iw], s.x, acc_r[iw]);
      acc_r[iw] = fma(-ti[iw], s.y, acc_r[iw]);
      acc_i[iw] = fma(tr[iw], s.y, acc_i[iw]);
      acc_i[iw] = fma(ti[iw], s.x, acc_i[iw]);
    }
    const bool last = (j + 1 == j1) || next0 <= j + 1;
    if (last) flush(acc_r, acc_i, lo_r, lo_i, red, partials, max_seg, i - inst_lo);
  }
}

// achtemp of instance i = sum over its CTAs b (in order) of slot (b, i - first
// instance of b).  One block per instance.
__global__ void __launch_bounds__(256)
    batch_finalize_kernel(const BatchInst *__restrict__ inst, int n, const int *__restrict__ cta_inst_lo,
                          const long long *__restrict__ range, int max_seg, const double *__restrict__ partials) {
  __shared__ double red[8 * 6];
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const BatchInst &I = inst[i];
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (I.b_lo <= I.b_hi) {
      for (int b = I.b_lo + threadIdx.x; b <= I.b_hi; b += 256) {
        if (range[b] >= range[b + 1]) continue;  // an empty CTA range inside the span wrote nothing
        const double *src = partials + ((size_t)b * max_seg + (i - cta_inst_lo[b])) * 6;
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] += src[k];
      }
    }
    block_sum<6, 256>(v, red);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < 6; ++k) I.out[k] = v[k];
    }
  }
}

// ------------------------------------------------------------- host side --

struct Variant {
  int ke;          // elements per thread
  size_t smem;     // dynamic shared memory
  int per_sm;      // resident CTAs per SM
};

// Band rows per step: FP64 256 (with the staged elements), mixed 512.
template <bool MIXED>
constexpr int batch_bch() {
  return MIXED ? 512 : 256;
}

template <int KE, bool MIXED, int K = 3>
int band_variant(Variant *v) {
  v->ke = KE;
  v->smem = sizeof(BatchSmem<batch_bch<MIXED>(), KE, MIXED>);
  auto kfn = batch_bandloop_kernel<batch_bch<MIXED>(), KE, MIXED, K>;
  BGW_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v->smem));
  BGW_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v->per_sm, kfn, kBThreads, v->smem));
  return v->per_sm >= 1 ? BGW_OK : BGW_ERR_UNSUPPORTED;
}

template <int KE, bool MIXED, int K = 3>
void launch_band(cudaStream_t s, int grid, size_t smem, const BatchInst *inst, int n, const long long *range,
                 int max_seg, double *partials, int *status, long long stall) {
  batch_bandloop_kernel<batch_bch<MIXED>(), KE, MIXED, K><<<grid, kBThreads, smem, s>>>(inst, n, range, max_seg,
                                                                                        partials, status, stall);
}

std::mutex g_tune_mu;
std::map<std::string, int> g_tune_cache;  // batch signature -> chosen kE

}  // namespace
}  // namespace bgw

// Opaque batch handle of the C ABI.
struct bgw_gpp_batch {
  int device = 0;
  int n = 0;
  bool factored = false, mixed = false;
  int mixed_order = 3;
  int ke = 4;
  int grid = 1;
  int max_seg = 1;
  size_t smem = 0;
  long long total_items = 0, total_cols = 0;
  double flops = 0.0, bytes = 0.0;
  std::vector<bgw::BatchInst> h_inst;
  void *d_block = nullptr;  // one allocation: inst | range | cta_inst_lo | partials | status | tables
  bgw::BatchInst *d_inst = nullptr;
  long long *d_range = nullptr;
  int *d_cta_lo = nullptr;
  double *d_partials = nullptr;
  int *d_status = nullptr;
  cudaStream_t capture = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  char kernel_name[48] = {};
};

namespace bgw {
namespace {

// Cuts items [0, limit) into `grid` ranges of equal estimated cost (per item:
// bands x elements for the band loop, elements for the factored stream, plus
// a fixed per-item overhead).
void partition(const std::vector<BatchInst> &inst, bool factored, int kch, int bch, double step_bands,
               long long limit, int grid, std::vector<long long> *range) {
  const int n = (int)inst.size();
  std::vector<double> cum(n + 1, 0.0), per(n, 0.0);
  for (int i = 0; i < n; ++i) {
    const long long items = (long long)inst[i].P * inst[i].nchunk;
    const double elems = inst[i].nchunk > 0 ? (double)inst[i].G / inst[i].nchunk : 0.0;
    // The band loop sweeps every slot of a chunk, padding included (an item
    // costs kch x bands), plus a per-step set-up of step_bands bands' worth;
    // the factored stream skips the padding.
    const int nb = std::max(inst[i].nb, 1), steps = (nb + bch - 1) / bch;
    per[i] = factored ? elems + 0.25 * kch : (double)kch * (nb + step_bands * steps);
    const long long lim = std::max(0LL, std::min(items, limit - inst[i].item0));
    cum[i + 1] = cum[i] + per[i] * (double)lim;
  }
  range->assign(grid + 1, 0);
  const double total = cum[n];
  for (int b = 1; b < grid; ++b) {
    const double t = total * b / grid;
    int i = (int)(std::upper_bound(cum.begin(), cum.end(), t) - cum.begin()) - 1;
    i = std::min(std::max(i, 0), n - 1);
    long long j = inst[i].item0 + (per[i] > 0 ? (long long)std::ceil((t - cum[i]) / per[i]) : 0);
    j = std::min(j, limit);
    (*range)[b] = std::max((*range)[b - 1], j);
  }
  (*range)[grid] = limit;
}

int instance_of(const std::vector<BatchInst> &inst, long long item) {
  int lo = 0, hi = (int)inst.size() - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (inst[mid].item0 <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Fills b_lo/b_hi per instance, the first instance per CTA and the slots
// per CTA.
void assign_slots(std::vector<BatchInst> &inst, const std::vector<long long> &range, std::vector<int> *cta_lo,
                  int *max_seg) {
  const int grid = (int)range.size() - 1, n = (int)inst.size();
  cta_lo->assign(grid, 0);
  *max_seg = 1;
  for (auto &I : inst) {
    I.b_lo = 1;
    I.b_hi = 0;
  }
  for (int b = 0; b < grid; ++b) {
    if (range[b] >= range[b + 1]) {
      (*cta_lo)[b] = 0;
      continue;
    }
    const int lo = instance_of(inst, range[b]), hi = instance_of(inst, range[b + 1] - 1);
    (*cta_lo)[b] = lo;
    *max_seg = std::max(*max_seg, hi - lo + 1);
    for (int i = lo; i <= hi; ++i) {
      if ((long long)inst[i].P * inst[i].nchunk == 0) continue;  // no items: never flushed, result 0
      if (inst[i].b_lo > inst[i].b_hi) inst[i].b_lo = b;
      inst[i].b_hi = b;
    }
  }
  (void)n;
}

// stall: the band loop's injected stall step (-1 when tuning, so a test's
// stall never reaches the tuner's timings or its cache).
int enqueue_batch(bgw_gpp_batch *B, cudaStream_t s, long long stall = -1) {
  BGW_CUDA_TRY(cudaMemsetAsync(B->d_status, 0, sizeof(int32_t) * STATUS_WORDS, s));
  const int ninst = B->n;
  int pg = (int)std::min<long long>(std::max<long long>((B->total_cols + 7) / 8, 1), 148LL * 16);
  batch_prep_kernel<<<pg, 256, 0, s>>>(B->d_inst, ninst, B->total_cols, B->factored ? 1 : 0, B->d_status);
  BGW_CUDA_TRY(cudaGetLastError());
  if (!B->factored) {
    batch_wx_kernel<<<std::min(ninst, 1024), 256, 0, s>>>(B->d_inst, ninst);
    BGW_CUDA_TRY(cudaGetLastError());
    if (B->mixed) {
      auto *fn = B->mixed_order == 0   ? launch_band<16, true, 0>
                 : B->mixed_order == 1 ? launch_band<16, true, 1>
                 : B->mixed_order == 2 ? launch_band<16, true, 2>
                                       : launch_band<16, true, 3>;
      fn(s, B->grid, B->smem, B->d_inst, ninst, B->d_range, B->max_seg, B->d_partials, B->d_status, stall);
    } else {
      if (B->ke == 8) launch_band<8, false>(s, B->grid, B->smem, B->d_inst, ninst, B->d_range, B->max_seg,
                                           B->d_partials, B->d_status, stall);
      else if (B->ke == 4) launch_band<4, false>(s, B->grid, B->smem, B->d_inst, ninst, B->d_range, B->max_seg,
                                                B->d_partials, B->d_status, stall);
      else launch_band<2, false>(s, B->grid, B->smem, B->d_inst, ninst, B->d_range, B->max_seg, B->d_partials,
                                 B->d_status, stall);
    }
  } else {
    batch_factored_kernel<4><<<B->grid, kBThreads, 0, s>>>(B->d_inst, ninst, B->d_range, B->max_seg,
                                                            B->d_partials);
  }
  BGW_CUDA_TRY(cudaGetLastError());
  batch_finalize_kernel<<<std::min(ninst, 4096), 256, 0, s>>>(B->d_inst, ninst, B->d_cta_lo, B->d_range,
                                                              B->max_seg, B->d_partials);
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

}  // namespace
}  // namespace bgw

using namespace bgw;

extern "C" int bgw_gpp_batch_destroy(bgw_gpp_batch *B) {
  if (!B) return BGW_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(B->device);
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  if (B->capture) cudaStreamDestroy(B->capture);
  if (B->d_block) cudaFree(B->d_block);
  cudaSetDevice(prev);
  delete B;
  return BGW_OK;
}

extern "C" int bgw_gpp_batch_create(const bgw_gpp_instance *instances, int64_t n, const bgw_options *opt,
                                    bgw_gpp_batch **out) {
  if (!out || n <= 0 || n > (1 << 20) || !instances) return BGW_ERR_INVALID_ARG;
  *out = nullptr;
  CallEnv env;
  BGW_TRY(begin_call(opt, &env));
  if (env.host) return BGW_ERR_INVALID_ARG;  // device-resident instances only
  if (env.opt.flags & (BGW_FLAG_ASYNC | BGW_FLAG_PROFILE)) return BGW_ERR_INVALID_ARG;
  if (env.opt.pole_guard > 0.0) return BGW_ERR_UNSUPPORTED;  // near-pole cut-off: single calls only
  const bool mixed = env.opt.precision == BGW_PRECISION_MIXED;
  // Factored only when every wx is band-independent (and FP64).
  bool all_shared = true;
  for (int64_t i = 0; i < n; ++i) all_shared = all_shared && instances[i].wx_band_stride == 0;
  bool factored = env.opt.gpp_algorithm == BGW_GPP_FACTORED ||
                  (env.opt.gpp_algorithm == BGW_GPP_AUTO && all_shared && !mixed);
  if (factored && (mixed || !all_shared)) return BGW_ERR_UNSUPPORTED;

  // Validate and lay out.
  std::vector<BatchInst> h(n);
  size_t tab_elems = 0, wx4_elems = 0;
  for (int64_t i = 0; i < n; ++i) {
    const bgw_gpp_instance &q = instances[i];
    if (q.number_bands < 0 || q.ngpown < 0 || q.ncouls <= 0 || q.number_bands > INT32_MAX ||
        q.ngpown > INT32_MAX || q.ncouls > INT32_MAX || q.indinv_len <= 0 || q.wx_band_stride < 0 ||
        (q.wx_band_stride != 0 && q.wx_band_stride < 3) || !q.achtemp || !q.vcoul || !q.indinv ||
        (!q.wx_array && (q.number_bands > 0 || q.wx_band_stride == 0)))
      return BGW_ERR_INVALID_ARG;
    if (q.ngpown > 0 && (!q.inv_igp_index || !q.wtilde_array || !q.I_eps_array)) return BGW_ERR_INVALID_ARG;
    if (q.number_bands > 0 && q.ngpown > 0 && (!q.aqsmtemp || !q.aqsntemp)) return BGW_ERR_INVALID_ARG;
    if (((uintptr_t)q.wtilde_array | (uintptr_t)q.I_eps_array | (uintptr_t)q.aqsmtemp | (uintptr_t)q.aqsntemp) &
        15u)
      return BGW_ERR_INVALID_ARG;
    BatchInst &I = h[i];
    std::memset(&I, 0, sizeof(I));
    I.wt = (const double2 *)q.wtilde_array;
    I.ie = (const double2 *)q.I_eps_array;
    I.am = (const double2 *)q.aqsmtemp;
    I.an = (const double2 *)q.aqsntemp;
    I.vc = q.vcoul;
    I.wx = q.wx_array;
    I.inv = q.inv_igp_index;
    I.indinv = q.indinv;
    I.out = q.achtemp;
    I.indinv_len = q.indinv_len;
    I.wx_stride = q.wx_band_stride;
    I.nb = (int)q.number_bands;
    I.P = (int)q.ngpown;
    I.G = (int)q.ncouls;
    tab_elems += factored ? (size_t)I.P : (size_t)I.P * I.nb;
    wx4_elems += factored ? 0 : (size_t)I.nb;
  }

  // Candidate variants and the work list of each.
  Workspace *ws = env.ws;
  {
    std::lock_guard<std::mutex> lk(ws->mu);
    BGW_TRY(ws_acquire(ws, env.stream));  // creates the SM count on first use
  }
  std::vector<Variant> cands;
  if (factored) {
    cands.push_back({4, 0, 8});
  } else if (mixed) {
    Variant a;
    switch (env.opt.mixed_order) {
      case 0: BGW_TRY((band_variant<16, true, 0>(&a))); break;
      case 1: BGW_TRY((band_variant<16, true, 1>(&a))); break;
      case 2: BGW_TRY((band_variant<16, true, 2>(&a))); break;
      default: BGW_TRY((band_variant<16, true, 3>(&a))); break;
    }
    cands = {a};
  } else {
    Variant a, b, c;
    BGW_TRY((band_variant<8, false>(&a)));
    BGW_TRY((band_variant<4, false>(&b)));
    BGW_TRY((band_variant<2, false>(&c)));
    cands = {a, b, c};
  }

  bgw_gpp_batch *B = new (std::nothrow) bgw_gpp_batch();
  if (!B) return BGW_ERR_ALLOC;
  B->device = env.device;
  B->n = (int)n;
  B->factored = factored;
  B->mixed = mixed;
  B->mixed_order = env.opt.mixed_order;

  auto layout = [&](const Variant &v, long long limit, std::vector<long long> *range, std::vector<int> *cta_lo,
                    int *grid, int *max_seg) {
    const int kch = kBThreads * v.ke;
    long long item = 0, col = 0;
    for (auto &I : h) {
      I.nchunk = (I.G + kch - 1) / kch;
      I.item0 = item;
      I.col0 = col;
      item += (long long)I.P * I.nchunk;
      col += I.P;
    }
    B->total_items = item;
    B->total_cols = col;
    if (limit < 0 || limit > item) limit = item;
    *grid = (int)std::max<long long>(1, std::min<long long>((long long)ws->sm_count * v.per_sm,
                                                              std::max<long long>(limit, 1)));
    // Per-step set-up in bands' worth: FP64 staging ~2; mixed band moments,
    // FP64 hoisted terms and the element loads 32 (chosen by measurement on
    // the 64-instance batch: 0.99x over sequential calls at 16, 1.04x at 32).
    partition(h, factored, kch, mixed ? batch_bch<true>() : batch_bch<false>(), mixed ? 32.0 : 2.0, limit, *grid,
              range);
    assign_slots(h, *range, cta_lo, max_seg);
  };

  // Device block: inst | range | cta_lo | partials | status | tab | wx4.
  // Sized for the largest candidate grid.
  int max_grid = 1;
  for (auto &v : cands) max_grid = std::max(max_grid, ws->sm_count * v.per_sm);
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t off_inst = 0;
  const size_t off_range = off_inst + al(sizeof(BatchInst) * (size_t)n);
  const size_t off_cta = off_range + al(sizeof(long long) * ((size_t)max_grid + 1));
  const size_t off_part = off_cta + al(sizeof(int) * (size_t)max_grid);
  const size_t part_bytes = al(sizeof(double) * 6 * (size_t)max_grid * (size_t)std::min<int64_t>(n, 4096));
  const size_t off_status = off_part + part_bytes;
  const size_t off_tab = off_status + 256;
  const size_t off_wx4 = off_tab + al(sizeof(double2) * std::max<size_t>(tab_elems, 1));
  const size_t total = off_wx4 + al(sizeof(double4) * std::max<size_t>(wx4_elems, 1));
  if (cudaMalloc(&B->d_block, total) != cudaSuccess) {
    (void)cudaGetLastError();
    delete B;
    return BGW_ERR_ALLOC;
  }
  char *base = static_cast<char *>(B->d_block);
  B->d_inst = reinterpret_cast<BatchInst *>(base + off_inst);
  B->d_range = reinterpret_cast<long long *>(base + off_range);
  B->d_cta_lo = reinterpret_cast<int *>(base + off_cta);
  B->d_partials = reinterpret_cast<double *>(base + off_part);
  B->d_status = reinterpret_cast<int *>(base + off_status);
  {
    size_t t = 0, w = 0;
    for (auto &I : h) {
      I.tab = reinterpret_cast<double2 *>(base + off_tab) + t;
      I.wx4 = reinterpret_cast<double4 *>(base + off_wx4) + w;
      t += factored ? (size_t)I.P : (size_t)I.P * I.nb;
      w += factored ? 0 : (size_t)I.nb;
    }
  }
  const size_t max_slots = part_bytes / (sizeof(double) * 6);

  auto upload = [&](const std::vector<long long> &range, const std::vector<int> &cta_lo) -> int {
    BGW_CUDA_TRY(cudaMemcpy(B->d_inst, h.data(), sizeof(BatchInst) * h.size(), cudaMemcpyHostToDevice));
    BGW_CUDA_TRY(cudaMemcpy(B->d_range, range.data(), sizeof(long long) * range.size(), cudaMemcpyHostToDevice));
    BGW_CUDA_TRY(cudaMemcpy(B->d_cta_lo, cta_lo.data(), sizeof(int) * cta_lo.size(), cudaMemcpyHostToDevice));
    return BGW_OK;
  };

  // Autotune: time each candidate on a sample prefix (about 1/16 of the
  // items, at least one item per CTA) unless this signature is cached.
  std::string sig = std::string(factored ? "F" : (mixed ? "M" + std::to_string(env.opt.mixed_order) : "D")) +
                    std::to_string(env.device);
  for (auto &I : h) sig += ":" + std::to_string(I.nb) + "x" + std::to_string(I.P) + "x" + std::to_string(I.G);
  int chosen = -1;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(sig);
    if (it != g_tune_cache.end()) chosen = it->second;
  }
  int rc = BGW_OK;
  std::vector<long long> range;
  std::vector<int> cta_lo;
  if (chosen < 0) {
    float best = 1e30f;
    chosen = cands[0].ke;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cands.size() > 1 && cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
      for (auto &v : cands) {
        int grid = 1, mseg = 1;
        layout(v, 0, &range, &cta_lo, &grid, &mseg);
        const long long sample = std::max<long long>(B->total_items / 16, (long long)grid);
        layout(v, sample, &range, &cta_lo, &grid, &mseg);
        if ((size_t)grid * mseg > max_slots) continue;
        if ((rc = upload(range, cta_lo)) != BGW_OK) break;
        B->ke = v.ke;
        B->grid = grid;
        B->max_seg = mseg;
        B->smem = v.smem;
        if ((rc = enqueue_batch(B, env.stream)) != BGW_OK) break;  // warm-up: tables and caches
        cudaEventRecord(e0, env.stream);
        if ((rc = enqueue_batch(B, env.stream)) != BGW_OK) break;
        cudaEventRecord(e1, env.stream);
        if (cudaEventSynchronize(e1) != cudaSuccess) {
          rc = BGW_ERR_CUDA;
          break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
          best = ms;
          chosen = v.ke;
        }
      }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc == BGW_OK) {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune_cache[sig] = chosen;
    }
  }
  const Variant *pick = &cands[0];
  for (auto &v : cands)
    if (v.ke == chosen) pick = &v;
  int grid = 1, mseg = 1;
  if (rc == BGW_OK) {
    layout(*pick, -1, &range, &cta_lo, &grid, &mseg);
    if ((size_t)grid * mseg > max_slots) rc = BGW_ERR_UNSUPPORTED;
  }
  if (rc == BGW_OK) rc = upload(range, cta_lo);
  if (rc != BGW_OK) {
    bgw_gpp_batch_destroy(B);
    return rc;
  }
  B->ke = pick->ke;
  B->grid = grid;
  B->max_seg = mseg;
  B->smem = pick->smem;
  std::snprintf(B->kernel_name, sizeof(B->kernel_name), "%s<kE=%d>",
                factored ? "batch_factored_kernel" : (mixed ? "batch_bandloop_kernel<mixed>" : "batch_bandloop_kernel"),
                B->ke);
  for (auto &I : h) {
    B->flops += 63.0 * (double)I.nb * (double)I.P * (double)I.G;
    B->bytes += 32.0 * (double)I.P * (double)I.G;
  }
  B->h_inst = h;

  // Capture prep + persistent kernel + finalize into a graph.
  if (cudaStreamCreateWithFlags(&B->capture, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamBeginCapture(B->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    (void)cudaGetLastError();
    bgw_gpp_batch_destroy(B);
    return BGW_ERR_CUDA;
  }
  rc = enqueue_batch(B, B->capture, stall_step());
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(B->capture, &graph);
  if (rc != BGW_OK || ce != cudaSuccess || !graph ||
      cudaGraphInstantiate(&B->exec, graph, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    if (graph) cudaGraphDestroy(graph);
    bgw_gpp_batch_destroy(B);
    return rc != BGW_OK ? rc : BGW_ERR_CUDA;
  }
  B->graph = graph;
  *out = B;
  return BGW_OK;
}

extern "C" int bgw_gpp_batch_execute(bgw_gpp_batch *B, const bgw_options *opt) {
  if (!B) return BGW_ERR_INVALID_ARG;
  bgw_options o;
  bgw_options_init(&o);
  if (opt) {
    if (opt->struct_size < (int32_t)(offsetof(bgw_options, device_status) + sizeof(int32_t *)))
      return BGW_ERR_INVALID_ARG;
    std::memcpy(&o, opt, std::min<size_t>((size_t)opt->struct_size, sizeof(o)));
    o.struct_size = (int32_t)sizeof(o);
  }
  if ((o.flags & BGW_FLAG_ASYNC) && !o.device_status) return BGW_ERR_INVALID_ARG;
  BGW_CUDA_TRY(cudaSetDevice(B->device));
  cudaStream_t s = static_cast<cudaStream_t>(o.stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const bool prof = (o.flags & BGW_FLAG_PROFILE) && !(o.flags & BGW_FLAG_ASYNC);
  if (prof) {
    BGW_CUDA_TRY(cudaEventCreate(&e0));
    BGW_CUDA_TRY(cudaEventCreate(&e1));
    BGW_CUDA_TRY(cudaEventRecord(e0, s));
  }
  BGW_CUDA_TRY(cudaGraphLaunch(B->exec, s));
  count_launch(B->factored ? 3 : 4);
  if (o.flags & BGW_FLAG_ASYNC) {
    BGW_CUDA_TRY(cudaMemcpyAsync(o.device_status, B->d_status, sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    return BGW_OK;
  }
  if (prof) BGW_CUDA_TRY(cudaEventRecord(e1, s));
  int32_t st[STATUS_WORDS] = {0, 0, 0, 0};
  BGW_CUDA_TRY(cudaMemcpyAsync(st, B->d_status, sizeof(st), cudaMemcpyDeviceToHost, s));
  BGW_CUDA_TRY(cudaStreamSynchronize(s));
  if (prof) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    bgw_profile p = {};
    p.main_kernel_ms = ms;
    p.device_ms = ms;
    p.flops = B->flops;
    p.main_bytes = B->bytes;
    p.main_launches = 1;
    p.total_launches = B->factored ? 3 : 4;
    std::snprintf(p.main_kernel, sizeof(p.main_kernel), "%s", B->kernel_name);
    set_last_profile(p);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  return st[0];
}

extern "C" int bgw_gpp_batch_info(const bgw_gpp_batch *B, int32_t *elems_per_thread, int32_t *grid,
                                  int64_t *total_items) {
  if (!B) return BGW_ERR_INVALID_ARG;
  if (elems_per_thread) *elems_per_thread = B->ke;
  if (grid) *grid = B->grid;
  if (total_items) *total_items = B->total_items;
  return BGW_OK;
}
