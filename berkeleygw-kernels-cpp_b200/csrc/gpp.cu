// gpp.cu -- GPP self-energy summation (noflagOCC_solver, GPP/gpp.cpp:307-402)
// on sm_100a, FP64.
//
// Work decomposition.  The reference sum
//   achtemp[iw] = sum_{n1, p, ig} s(n1, p) * q(p, ig, iw; wx[n1][iw]),
//   s(n1, p)    = conj(aqsm[n1][igp]) aqsn[n1][igp] 0.5 vcoul[igp] wtilde[p][igp]
//                 (sch_store1, gpp.cpp:369-371),
//   q           = conj(wdiff) / |wdiff|^2 * I_eps[p][ig],  wdiff = wx - wtilde[p][ig]
//                 (gpp.cpp:374-380)
// is split into items (p, a chunk of CH consecutive ig).  An item's wtilde /
// I_eps chunk is staged once into shared memory by 1-D bulk copies (TMA
// engine, mbarrier completion, double-buffered across items) and lifted into
// registers; the CTA then sweeps every band n1 over it, so each element of
// the 1.7 GB wtilde / I_eps arrays is read from HBM once while the FP64 pipe
// evaluates nb * 3 quotients on it.  s(n1, p) is precomputed into a
// [p][n1] table by gpp_prep_kernel and staged per item alongside the chunk.
//
// Reduction.  Each thread accumulates its own 3 complex sums; a CTA folds
// them with warp butterflies and a fixed warp order into one partial; a
// single-block kernel sums the partials in a fixed order.  No atomics, so
// reruns are bitwise identical.
#include <algorithm>
#include <numeric>
#include <cstdio>
#include <cstring>
#include <functional>
#include <thread>
#include <type_traits>
#include <vector>

#include "bgw_internal.cuh"
#include "gpp_common.cuh"
#include "reduce.cuh"

namespace bgw {
namespace {

constexpr int kThreads = 256;
constexpr int kElems = 4;                 // ig elements per thread
constexpr int kChunk = kThreads * kElems;  // ig per item


// ---------------------------------------------------------------- prep --
// st[p][n1] = sch_store1(n1, p); wx4[n1] = (wx[n1][0..2], 0); S[p] (if
// requested) = sum_n1 st[p][n1] in a fixed order.  Indices are checked: an
// out-of-range inv_igp_index / indinv entry raises BGW_ERR_INDEX and that
// column contributes zero (no out-of-bounds read is ever issued).
// One warp per column p: st row (if st != nullptr) and S[p] (if S != nullptr).
// gstride > 0: am / an / vc were gathered on the host to the columns
// igp(p) (am[n1 * gstride + p], vc[p]); wtilde is always read at igp(p).
// S_occ (optional): the same sum over the first nv bands only (the occupied
// bands of the screened exchange); S is unaffected by it.
__global__ void __launch_bounds__(256) gpp_prep_kernel(int nb, int P, int G, const int *__restrict__ inv,
                                                       const int *__restrict__ indinv, long long indinv_len,
                                                       const double2 *__restrict__ wt, const double2 *__restrict__ am,
                                                       const double2 *__restrict__ an, const double *__restrict__ vc,
                                                       double2 *__restrict__ st, double2 *__restrict__ S,
                                                       int *status, long long gstride, int nv = 0,
                                                       double2 *__restrict__ S_occ = nullptr) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < P; p += warps) {
    int g = resolve_igp(p, inv, indinv, indinv_len, G, status);
    double sr = 0.0, si = 0.0, or_ = 0.0, oi = 0.0;
    for (int n1 = lane; n1 < nb; n1 += 32) {
      double2 s = make_double2(0.0, 0.0);
      if (g >= 0 && gstride > 0) {
        double2 m = am[(size_t)n1 * gstride + p];
        m.y = -m.y;
        double2 r = cmul(m, an[(size_t)n1 * gstride + p]);  // same operation order as store1
        r.x *= 0.5;
        r.y *= 0.5;
        const double v = vc[p];
        r.x *= v;
        r.y *= v;
        s = cmul(r, wt[(size_t)p * G + g]);
      } else if (g >= 0) {
        s = store1(am, an, vc, wt, n1, p, g, G);
      }
      if (st) st[(size_t)p * nb + n1] = s;
      sr += s.x;
      si += s.y;
      if (n1 < nv) {
        or_ += s.x;
        oi += s.y;
      }
    }
    if (S) {
      sr = warp_sum(sr);
      si = warp_sum(si);
      if (lane == 0) S[p] = make_double2(sr, si);
    }
    if (S_occ) {
      or_ = warp_sum(or_);
      oi = warp_sum(oi);
      if (lane == 0) S_occ[p] = make_double2(or_, oi);
    }
  }
}

__global__ void gpp_wx_kernel(int nb, const double *__restrict__ wx, long long stride, double4 *__restrict__ wx4) {
  for (int n1 = blockIdx.x * blockDim.x + threadIdx.x; n1 < nb; n1 += gridDim.x * blockDim.x) {
    const double *w = wx + (size_t)n1 * stride;
    wx4[n1] = make_double4(w[0], w[1], w[2], 0.0);
  }
}

// ------------------------------------------------------------ band loop --
// Per element (wtilde = wr + i wi, I_eps = Ir + i Ii) the band-independent
// constants are kept in registers:  wi^2, a = -wi*Ii, b = wi*Ir, so that for
// a frequency x:
//   dr  = x - wr,  |wdiff|^2 = dr^2 + wi^2,
//   conj(wdiff) * I_eps = (dr*Ir + a) + i (dr*Ii + b).
// Elements per thread: FP64 8 (a longer run per band amortises the per-band
// combination with sch_store1: 53.6 ms at 8 vs 58.0 ms at 4 and 55.8 ms at 6
// on the 512-band benchmark); mixed 16 (more independent work per thread,
// the per-band multiply over 48 terms).  256 threads per CTA, one CTA per
// SM.  FP64: the step's wtilde / I_eps chunk is staged in shared memory with
// the band rows (210 registers, 153 KB).  Mixed: the elements are read once
// per step from global memory (the item's chunk stays in L2 across its band
// chunks), which leaves the shared memory to 512-band steps: the per-step
// set-up (band moments, FP64 hoisted terms) is then amortised over every
// band of a 512-band problem (~123 KB with the remainder rows).
template <bool MIXED>
struct BandCfg {
  static constexpr int kE = MIXED ? 16 : 8;
  static constexpr int kNT = kThreads;
  static constexpr int kCH = kNT * kE;
};

template <int BCH, bool MIXED>
struct BandSmem {
  double2 wt[2][MIXED ? 1 : BandCfg<MIXED>::kCH];  // FP64 only: staged elements
  double2 ie[2][MIXED ? 1 : BandCfg<MIXED>::kCH];
  double2 st[2][BCH];
  double4 wx[2][BCH];
  unsigned long long bar[3];  // [2]: never arrived on (stall injection)
  double red[(BandCfg<MIXED>::kNT / 32) * 18];
  double xr_lo[BandCfg<MIXED>::kNT / 32], xr_hi[BandCfg<MIXED>::kNT / 32];  // MIXED: chunk frequency range
  RemRow rows[MIXED ? BCH : 1];                                               // MIXED: per-band remainder rows
};

// Every band reads its own frequencies from the staged wx4 rows (for the
// reference's band-independent wx the rows repeat one triple), so each
// (band, G', G, frequency) quotient is evaluated, as in gpp.cpp:343-390.
// MIXED: each step's quotients are expanded about the centre of the step's
// frequencies; K Taylor terms are hoisted into FP64 per element (rem_stage /
// rem_elems) and the remainder, |t|^K of each term, is a per-term complex
// quotient in packed FP32 (rem_sweep) whose group sums are accumulated in
// FP64 with TwoSum.  Elements near a pole take the FP64 path (near_sweep),
// which also applies the pole_guard cut-off.
// GUARD (FP64): near-pole cut-off, terms with |wdiff|^2 < guard2 contribute
// zero.  MIXED applies the guard in its FP64 near path; GUARD is not used.
template <int BCH, bool MIXED, bool GUARD, int K = 3>
__global__ void __launch_bounds__(BandCfg<MIXED>::kNT, 1)
    gpp_bandloop_kernel(int nb, int G, long long items, int nchunks_g, const double2 *__restrict__ wtilde,
                        const double2 *__restrict__ ieps, const double2 *__restrict__ st,
                        const double4 *__restrict__ wx4, double *__restrict__ partials, int *status,
                        double guard2, long long stall) {
  constexpr int kE = BandCfg<MIXED>::kE;
  constexpr int kCH = BandCfg<MIXED>::kCH;
  constexpr int kThreads = BandCfg<MIXED>::kNT;  // shadows the file-wide 256
  extern __shared__ __align__(128) unsigned char smem_raw[];
  using Smem = BandSmem<BCH, MIXED>;
  Smem &sm = *reinterpret_cast<Smem *>(smem_raw);
  const int tid = threadIdx.x;
  const int nbc = (nb + BCH - 1) / BCH;

  long long my_items = 0;
  if ((long long)blockIdx.x < items) my_items = (items - 1 - blockIdx.x) / gridDim.x + 1;
  const long long nsteps = my_items * nbc;

  if (tid == 0) {
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[0]), 1);
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[1]), 1);
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[2]), 1);
    fence_mbar_init();
  }
  __syncthreads();

  // Thread 0 stages step j into buffer j & 1.
  auto issue = [&](long long j) {
    const long long item = blockIdx.x + (j / nbc) * (long long)gridDim.x;
    const int c = (int)(j % nbc);
    const long long p = item / nchunks_g;
    const int g0 = (int)(item % nchunks_g) * kCH;
    const int nvalid = min(kCH, G - g0);
    const int b0 = c * BCH;
    const int nbv = min(BCH, nb - b0);
    const int buf = (int)(j & 1);
    uint32_t bytes = (MIXED ? 0u : 2u * nvalid * 16u) + nbv * 16u + nbv * 32u;
    uint64_t *bar = reinterpret_cast<uint64_t *>(&sm.bar[buf]);
    // Debug build: the step's source ranges and the staging capacity.
    if (!BGW_CHECKED(item < items && nvalid > 0 && nvalid <= kCH && g0 + nvalid <= G && nbv > 0 && nbv <= BCH &&
                         b0 + nbv <= nb,
                     status, 11)) {
      mbar_expect_tx(bar, 0);  // completes the phase without copies
      return;
    }
    mbar_expect_tx(bar, bytes);
    if constexpr (!MIXED) {
      bulk_g2s(sm.wt[buf], wtilde + p * G + g0, nvalid * 16u, bar);
      bulk_g2s(sm.ie[buf], ieps + p * G + g0, nvalid * 16u, bar);
    }
    bulk_g2s(sm.st[buf], st + p * nb + b0, nbv * 16u, bar);
    bulk_g2s(sm.wx[buf], wx4 + b0, nbv * 32u, bar);
  };

  double acc_r[3] = {0.0, 0.0, 0.0}, acc_i[3] = {0.0, 0.0, 0.0};
  double lo_r[3] = {0.0, 0.0, 0.0}, lo_i[3] = {0.0, 0.0, 0.0};  // TwoSum tails (MIXED)
  bool ok = true;
  long long j_fail = 0;  // the step whose wait ran out
  if (tid == 0 && nsteps > 0) issue(0);

  for (long long j = 0; j < nsteps; ++j) {
    if (tid == 0 && j + 1 < nsteps) issue(j + 1);
    const int buf = (int)(j & 1);
    if (!staged_wait(reinterpret_cast<uint64_t *>(&sm.bar[buf]), j, stall,
                     reinterpret_cast<uint64_t *>(&sm.bar[2]))) {
      raise_status(status, BGW_ERR_TIMEOUT, blockIdx.x);
      ok = false;
    }
    // Every thread must agree before leaving the loop.
    if (__syncthreads_or(!ok)) {
      j_fail = j;
      break;
    }

    const long long item = blockIdx.x + (j / nbc) * (long long)gridDim.x;
    const int c = (int)(j % nbc);
    const int g0 = (int)(item % nchunks_g) * kCH;
    int nvalid = min(kCH, G - g0);
    const int b0 = c * BCH;
    int nbv = min(BCH, nb - b0);
    if (!BGW_CHECKED(nvalid <= kCH && nbv <= BCH, status, 12)) nvalid = nbv = 0;

    if constexpr (MIXED) {
      const long long p = item / nchunks_g;
      const double2 *wt_g = wtilde + p * G + g0, *ie_g = ieps + p * G + g0;
      const RemStep rs = rem_stage<kThreads, K>(sm.wx[buf], sm.st[buf], nbv, sm.rows, sm.red, sm.xr_lo, sm.xr_hi);
      RemElems<kE> e;
      const uint32_t near = rem_elems<kE, K>(e, wt_g, ie_g, nvalid, kThreads, tid, rs, guard2, acc_r, acc_i);
      rem_sweep<kE>(e, sm.rows, nbv, acc_r, acc_i, lo_r, lo_i);
      if (near) near_sweep(near, wt_g, ie_g, kThreads, tid, sm.wx[buf], sm.st[buf], nbv, guard2, acc_r, acc_i, lo_r,
                           lo_i);
    } else {
      Elem<double> e[kE];
      load_elems<double, kE>(e, sm.wt[buf], sm.ie[buf], nvalid, kThreads, tid);
      band_sweep<kE, GUARD>(e, sm.wx[buf], sm.st[buf], nbv, acc_r, acc_i, guard2);
    }
    __syncthreads();  // buffer `buf` is free for step j + 2
  }
  if (!ok && tid == 0) {
    // Copies still in flight (steps j_fail and j_fail + 1) land before the
    // CTA's shared memory is released.
    drain_staged(reinterpret_cast<uint64_t *>(&sm.bar[0]), reinterpret_cast<uint64_t *>(&sm.bar[1]), j_fail,
                 j_fail + 1 < nsteps);
  }

  double v[6] = {acc_r[0] + lo_r[0], acc_i[0] + lo_i[0], acc_r[1] + lo_r[1],
                 acc_i[1] + lo_i[1], acc_r[2] + lo_r[2], acc_i[2] + lo_i[2]};
  block_sum<6, kThreads>(v, sm.red);
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) partials[(size_t)blockIdx.x * 6 + k] = v[k];
  }
}

// ------------------------------------------------------------- factored --
// Band-independent wx: achtemp[iw] = sum_p S(p) * sum_ig q(p, ig, iw).
// HBM-bound stream over wtilde / I_eps with 128-bit loads; one item =
// (p, chunk of kChunk ig); per-thread sums are folded per CTA.
// GUARD: near-pole cut-off as in the band loop.
// SX: also the screened exchange of the occupied bands in the same pass over
// wtilde / I_eps: the sums at -wx are formed beside those at +wx, and
// asxtemp = -sum_p S_occ(p) (T(p, wx) + T(p, -wx)) (partial fractions of
// wtilde / (wx^2 - wtilde^2)); partials then hold 12 doubles per CTA,
// achtemp's 6 (bitwise the same as without SX) and asxtemp's 6.
template <bool GUARD, bool SX = false>
__global__ void __launch_bounds__(kThreads, SX ? 2 : 4)
    gpp_factored_kernel(int G, long long items, int nchunks_g, const double2 *__restrict__ wtilde,
                        const double2 *__restrict__ ieps, const double2 *__restrict__ S,
                        const double *__restrict__ wx3, double *__restrict__ partials, double guard2,
                        const double2 *__restrict__ S_occ = nullptr) {
  constexpr int W = SX ? 12 : 6;
  __shared__ double red[(kThreads / 32) * W];
  const int tid = threadIdx.x;
  const double x[3] = {wx3[0], wx3[1], wx3[2]};
  double acc_r[3] = {0.0, 0.0, 0.0}, acc_i[3] = {0.0, 0.0, 0.0};
  double ax_r[3] = {0.0, 0.0, 0.0}, ax_i[3] = {0.0, 0.0, 0.0};  // SX
  auto load = [&](long long item, double2 (&w)[kElems], double2 (&v)[kElems]) {
    const long long p = item / nchunks_g;
    const int g0 = (int)(item % nchunks_g) * kChunk;
#pragma unroll
    for (int k = 0; k < kElems; ++k) {
      const int ig = g0 + k * kThreads + tid;
      if (ig < G) {
        w[k] = __ldcs(wtilde + p * G + ig);
        v[k] = __ldcs(ieps + p * G + ig);
      } else {
        w[k] = make_double2(0.0, 1.0);
        v[k] = make_double2(0.0, 0.0);
      }
    }
  };
  // SX (twice the arithmetic per element): the next item's elements are
  // loaded before the current item is evaluated, so its loads are in flight
  // during the math.
  double2 wn[kElems], vn[kElems];
  if constexpr (SX) {
    if ((long long)blockIdx.x < items) load(blockIdx.x, wn, vn);
  }
  for (long long item = blockIdx.x; item < items; item += gridDim.x) {
    const long long p = item / nchunks_g;
    double2 w[kElems], v[kElems];
    if constexpr (SX) {
#pragma unroll
      for (int k = 0; k < kElems; ++k) {
        w[k] = wn[k];
        v[k] = vn[k];
      }
      if (item + gridDim.x < items) load(item + gridDim.x, wn, vn);
    } else {
      load(item, w, v);
    }
    double tr[3] = {0.0, 0.0, 0.0}, ti[3] = {0.0, 0.0, 0.0};
    double ur[3] = {0.0, 0.0, 0.0}, ui[3] = {0.0, 0.0, 0.0};  // SX: at -wx
#pragma unroll
    for (int k = 0; k < kElems; ++k) {
      const double wi2 = w[k].y * w[k].y, a = -w[k].y * v[k].y, b = w[k].y * v[k].x;
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        const double dr = x[iw] - w[k].x;
        const double den = fma(dr, dr, wi2);
        double r = rcp_refined(den);
        if constexpr (GUARD) r = den < guard2 ? 0.0 : r;
        tr[iw] = fma(fma(dr, v[k].x, a), r, tr[iw]);
        ti[iw] = fma(fma(dr, v[k].y, b), r, ti[iw]);
        if constexpr (SX) {
          const double dn = -x[iw] - w[k].x;
          const double dn2 = fma(dn, dn, wi2);
          double rn = rcp_refined(dn2);
          if constexpr (GUARD) rn = dn2 < guard2 ? 0.0 : rn;
          ur[iw] = fma(fma(dn, v[k].x, a), rn, ur[iw]);
          ui[iw] = fma(fma(dn, v[k].y, b), rn, ui[iw]);
        }
      }
    }
    const double2 s = S[p];
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) {
      acc_r[iw] = fma(tr[iw], s.x, acc_r[iw]);
      acc_r[iw] = fma(-ti[iw], s.y, acc_r[iw]);
      acc_i[iw] = fma(tr[iw], s.y, acc_i[iw]);
      acc_i[iw] = fma(ti[iw], s.x, acc_i[iw]);
    }
    if constexpr (SX) {
      const double2 so = S_occ[p];
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        const double qr = tr[iw] + ur[iw], qi = ti[iw] + ui[iw];
        ax_r[iw] = fma(-qr, so.x, ax_r[iw]);
        ax_r[iw] = fma(qi, so.y, ax_r[iw]);
        ax_i[iw] = fma(-qr, so.y, ax_i[iw]);
        ax_i[iw] = fma(-qi, so.x, ax_i[iw]);
      }
    }
  }
  double vv[W];
#pragma unroll
  for (int iw = 0; iw < 3; ++iw) {
    vv[2 * iw] = acc_r[iw];
    vv[2 * iw + 1] = acc_i[iw];
    if constexpr (SX) {
      vv[6 + 2 * iw] = ax_r[iw];
      vv[6 + 2 * iw + 1] = ax_i[iw];
    }
  }
  block_sum<W, kThreads>(vv, red);
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < W; ++k) partials[(size_t)blockIdx.x * W + k] = vv[k];
  }
}

template <int BCH, bool MIXED, bool GUARD = false, int K = 3>
int bandloop_per_sm(int *per_sm) {
  using Smem = BandSmem<BCH, MIXED>;
  const size_t smem = sizeof(Smem);
  auto kfn = gpp_bandloop_kernel<BCH, MIXED, GUARD, K>;
  BGW_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  BGW_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kfn, BandCfg<MIXED>::kNT, smem));
  return *per_sm >= 1 ? BGW_OK : BGW_ERR_UNSUPPORTED;
}

// Launches the band loop over rows [0, P) of the given (already offset)
// arrays; writes `grid` partials (6 doubles each) starting at `partials`.
template <int BCH, bool MIXED, bool GUARD, int K = 3>
int launch_bandloop(cudaStream_t stream, int max_grid, int nb, int G, const double2 *wt, const double2 *ie,
                    const double2 *st, const double4 *wx4, int64_t P, double *partials, int *grid_out,
                    int *status, double guard2) {
  using Smem = BandSmem<BCH, MIXED>;
  const size_t smem = sizeof(Smem);
  const int nchunks_g = (int)((G + BandCfg<MIXED>::kCH - 1) / BandCfg<MIXED>::kCH);
  const long long items = (long long)P * nchunks_g;
  long long grid = std::min<long long>(items, (long long)max_grid);
  if (grid < 1) grid = 1;
  *grid_out = (int)grid;
  gpp_bandloop_kernel<BCH, MIXED, GUARD, K><<<(int)grid, BandCfg<MIXED>::kNT, smem, stream>>>(
      nb, G, items, nchunks_g, wt, ie, st, wx4, partials, status, guard2, stall_step());
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

// Band chunk of the mixed form (the FP64 form stages 256 bands per step).
constexpr int kMixBCH = 512;

// The instantiation a call's options select: FP64 (guarded or not) or mixed
// with K = opt.mixed_order hoisted terms.
int bandloop_per_sm_for(const bgw_options &o, int *per_sm) {
  if (o.precision == BGW_PRECISION_MIXED) {
    switch (o.mixed_order) {
      case 0: return bandloop_per_sm<kMixBCH, true, false, 0>(per_sm);
      case 1: return bandloop_per_sm<kMixBCH, true, false, 1>(per_sm);
      case 2: return bandloop_per_sm<kMixBCH, true, false, 2>(per_sm);
      default: return bandloop_per_sm<kMixBCH, true, false, 3>(per_sm);
    }
  }
  if (o.pole_guard > 0.0) return bandloop_per_sm<256, false, true>(per_sm);
  return bandloop_per_sm<256, false, false>(per_sm);
}

int launch_bandloop_for(const bgw_options &o, cudaStream_t stream, int max_grid, int nb, int G, const double2 *wt,
                        const double2 *ie, const double2 *st, const double4 *wx4, int64_t P, double *partials,
                        int *grid_out, int *status) {
  const double guard2 = o.pole_guard * o.pole_guard;
  if (o.precision == BGW_PRECISION_MIXED) {
    switch (o.mixed_order) {
      case 0:
        return launch_bandloop<kMixBCH, true, false, 0>(stream, max_grid, nb, G, wt, ie, st, wx4, P, partials, grid_out,
                                                    status, guard2);
      case 1:
        return launch_bandloop<kMixBCH, true, false, 1>(stream, max_grid, nb, G, wt, ie, st, wx4, P, partials, grid_out,
                                                    status, guard2);
      case 2:
        return launch_bandloop<kMixBCH, true, false, 2>(stream, max_grid, nb, G, wt, ie, st, wx4, P, partials, grid_out,
                                                    status, guard2);
      default:
        return launch_bandloop<kMixBCH, true, false, 3>(stream, max_grid, nb, G, wt, ie, st, wx4, P, partials, grid_out,
                                                    status, guard2);
    }
  }
  if (o.pole_guard > 0.0)
    return launch_bandloop<256, false, true>(stream, max_grid, nb, G, wt, ie, st, wx4, P, partials, grid_out, status,
                                             guard2);
  return launch_bandloop<256, false, false>(stream, max_grid, nb, G, wt, ie, st, wx4, P, partials, grid_out, status,
                                            0.0);
}

}  // namespace

// Rows [p0[c], p0[c + 1]) of wtilde / I_eps form chunk c; the compute stream
// waits for ready[c] (may be null) before using chunk c.  One chunk with no
// event covers device-resident inputs.
struct RowChunks {
  static constexpr int kMax = 16;
  int n = 1;
  int64_t p0[kMax + 1] = {};
  cudaEvent_t ready[kMax] = {};
};

// Enqueues the GPP sum on env->stream.  All pointers are device pointers;
// wx holds 3 doubles (wx_stride == 0) or nb rows of wx_stride doubles.
// achtemp_dev receives 6 doubles (3 complex).
// `issue(c)` (optional) is called before chunk c is enqueued and may issue
// chunk c's copies: with pageable host memory cudaMemcpyAsync returns only
// after staging the source, so interleaving keeps the GPU busy on chunk c-1.
int gpp_enqueue_chunks(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                       int64_t indinv_len, const double *wx, int64_t wx_stride, const double2 *wt,
                       const double2 *am, const double2 *an, const double2 *ie, const double *vc,
                       double *achtemp_dev, RowChunks &rc, const std::function<int(int)> &issue = nullptr,
                       long long gstride = 0) {
  Workspace *ws = env->ws;
  cudaStream_t stream = env->stream;
  const bool factored = env->opt.gpp_algorithm == BGW_GPP_FACTORED ||
                        (env->opt.gpp_algorithm == BGW_GPP_AUTO && wx_stride == 0 &&
                         env->opt.precision == BGW_PRECISION_FP64);
  if (factored && env->opt.precision == BGW_PRECISION_MIXED) return BGW_ERR_UNSUPPORTED;
  if (factored && wx_stride != 0) return BGW_ERR_UNSUPPORTED;  // needs a band-independent wx
  const bool mixed = env->opt.precision == BGW_PRECISION_MIXED;
  const bool guard = env->opt.pole_guard > 0.0;
  const double guard2 = env->opt.pole_guard * env->opt.pole_guard;
  auto prep_grid_for = [&](int64_t rows) {
    return (int)std::max<long long>(1, std::min<long long>((rows + 7) / 8, (long long)ws->sm_count * 16));
  };

  // Partials: an upper bound of every chunk's grid, reserved up front.
  int per_launch = 0;
  if (factored) {
    per_launch = ws->sm_count * 8;
  } else {
    int per_sm = 0;
    // Also sets the launched instantiation's shared-memory limit.
    BGW_TRY(bandloop_per_sm_for(env->opt, &per_sm));
    per_launch = ws->sm_count * per_sm;
  }
  void *partials_v = nullptr, *tab = nullptr, *wx4 = nullptr;
  BGW_TRY(ws_reserve(ws, SLOT_PARTIALS, sizeof(double) * 6 * (size_t)per_launch * rc.n, &partials_v));
  double *partials = static_cast<double *>(partials_v);
  const size_t tab_elems = factored ? (size_t)std::max<int64_t>(P, 1) : (size_t)std::max<int64_t>(P * nb, 1);
  BGW_TRY(ws_reserve(ws, SLOT_TABLE0, sizeof(double2) * tab_elems, &tab));
  if (!factored) {
    // Per-band frequency rows (stride 0: the one triple repeated per band).
    BGW_TRY(ws_reserve(ws, SLOT_TABLE1, sizeof(double4) * (size_t)std::max<int64_t>(nb, 1), &wx4));
  }

  int total = 0;  // partials written so far
  for (int c = 0; c < rc.n; ++c) {
    if (issue) BGW_TRY(issue(c));
    if (rc.ready[c]) BGW_CUDA_TRY(cudaStreamWaitEvent(stream, rc.ready[c], 0));
    const int64_t p0 = rc.p0[c], rows = rc.p0[c + 1] - rc.p0[c];
    if (c == 0 && !factored && nb > 0) {
      int g = (int)std::min<int64_t>((nb + 255) / 256, 1024);
      gpp_wx_kernel<<<std::max(g, 1), 256, 0, stream>>>((int)nb, wx, wx_stride, (double4 *)wx4);
      count_launch();
      BGW_CUDA_TRY(cudaGetLastError());
    }
    if (rows <= 0 && rc.n > 1) continue;
    const double2 *wt_c = wt + (size_t)p0 * G, *ie_c = ie + (size_t)p0 * G;
    double *part_c = partials + (size_t)total * 6;
    if (factored) {
      double2 *S_c = static_cast<double2 *>(tab) + p0;
      gpp_prep_kernel<<<prep_grid_for(rows), 256, 0, stream>>>(
          (int)nb, (int)rows, (int)G, inv + p0, indinv, indinv_len, wt_c, gstride ? am + p0 : am,
          gstride ? an + p0 : an, gstride ? vc + p0 : vc, nullptr, S_c, env->d_status, gstride);
      count_launch();
      BGW_CUDA_TRY(cudaGetLastError());
      const int nchunks_g = (int)((G + kChunk - 1) / kChunk);
      const long long items = (long long)rows * nchunks_g;
      const int grid = (int)std::min<long long>(std::max<long long>(items, 1), (long long)per_launch);
      if (c == 0) BGW_TRY(prof_mark(env, 1));
      if (guard)
        gpp_factored_kernel<true><<<grid, kThreads, 0, stream>>>((int)G, items, nchunks_g, wt_c, ie_c, S_c, wx,
                                                                 part_c, guard2);
      else
        gpp_factored_kernel<false><<<grid, kThreads, 0, stream>>>((int)G, items, nchunks_g, wt_c, ie_c, S_c, wx,
                                                                  part_c, 0.0);
      count_launch();
      BGW_CUDA_TRY(cudaGetLastError());
      total += grid;
    } else {
      double2 *st_c = static_cast<double2 *>(tab) + (size_t)p0 * nb;
      gpp_prep_kernel<<<prep_grid_for(rows), 256, 0, stream>>>(
          (int)nb, (int)rows, (int)G, inv + p0, indinv, indinv_len, wt_c, gstride ? am + p0 : am,
          gstride ? an + p0 : an, gstride ? vc + p0 : vc, st_c, nullptr, env->d_status, gstride);
      count_launch();
      BGW_CUDA_TRY(cudaGetLastError());
      if (c == 0) BGW_TRY(prof_mark(env, 1));
      int grid = 0;
      BGW_TRY(launch_bandloop_for(env->opt, stream, per_launch, (int)nb, (int)G, wt_c, ie_c, st_c,
                                  (const double4 *)wx4, rows, part_c, &grid, env->d_status));
      total += grid;
    }
  }
  BGW_TRY(prof_mark(env, 2));
  if (factored) {
    env->prof.main_bytes = 32.0 * (double)P * (double)G + 16.0 * (double)P;
    std::snprintf(env->prof.main_kernel, sizeof(env->prof.main_kernel), "gpp_factored_kernel");
  } else {
    env->prof.main_bytes = 32.0 * (double)P * (double)G + 16.0 * (double)P * (double)nb + 32.0 * (double)nb;
    std::snprintf(env->prof.main_kernel, sizeof(env->prof.main_kernel),
                  mixed ? "gpp_bandloop_kernel<mixed>" : "gpp_bandloop_kernel");
  }
  env->prof.main_launches = rc.n;
  reduce_partials_kernel<6><<<1, 256, 0, stream>>>(partials, std::max(total, 1), achtemp_dev);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

int gpp_enqueue(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                int64_t indinv_len, const double *wx, int64_t wx_stride, const double2 *wt, const double2 *am,
                const double2 *an, const double2 *ie, const double *vc, double *achtemp_dev) {
  RowChunks rc;
  rc.n = 1;
  rc.p0[0] = 0;
  rc.p0[1] = P;
  return gpp_enqueue_chunks(env, nb, P, G, inv, indinv, indinv_len, wx, wx_stride, wt, am, an, ie, vc,
                            achtemp_dev, rc);
}

// Host-resident inputs: the copies run on the workspace's copy stream in
// G'-row chunks, and chunk c's kernels start as soon as its rows have landed,
// so the H2D transfer of chunk c+1 overlaps the compute of chunk c.  The
// chunking is a fixed function of the sizes, so results stay deterministic.
int gpp_run_host(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                 int64_t indinv_len, const double *wx, size_t wx_n, int64_t wx_stride, const double *wt,
                 const double *am, const double *an, const double *ie, const double *vc, double *achtemp_dev) {
  Workspace *ws = env->ws;
  cudaStream_t cs = nullptr;
  BGW_TRY(ws_copy_stream(ws, &cs));
  // The copy stream starts after everything already queued on the compute
  // stream (earlier users of the staging buffers).
  BGW_CUDA_TRY(cudaEventRecord(ws->copy_start, env->stream));
  BGW_CUDA_TRY(cudaStreamWaitEvent(cs, ws->copy_start, 0));
  const size_t pg = (size_t)P * (size_t)G * 16;
  const size_t nbp = (size_t)nb * (size_t)P;
  void *d_inv, *d_ind, *d_wx, *d_vc, *d_am, *d_an, *d_wt, *d_ie;
  BGW_TRY(ws_reserve(ws, SLOT_IN0, sizeof(int32_t) * (size_t)P, &d_inv));
  BGW_TRY(ws_reserve(ws, SLOT_IN1, sizeof(int32_t) * (size_t)indinv_len, &d_ind));
  BGW_TRY(ws_reserve(ws, SLOT_IN2, sizeof(double) * wx_n, &d_wx));
  BGW_TRY(ws_reserve(ws, SLOT_IN7, sizeof(double) * (size_t)std::max<int64_t>(P, 1), &d_vc));
  BGW_TRY(ws_reserve(ws, SLOT_IN4, nbp * 16, &d_am));
  BGW_TRY(ws_reserve(ws, SLOT_IN5, nbp * 16, &d_an));
  BGW_TRY(ws_reserve(ws, SLOT_IN3, pg, &d_wt));
  BGW_TRY(ws_reserve(ws, SLOT_IN6, pg, &d_ie));
  auto h2d = [&](void *dst, const void *src, size_t bytes) -> int {
    if (bytes) BGW_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, cs));
    return BGW_OK;
  };
  // Up to 16 chunks of at least 64 rows.
  RowChunks rc;
  rc.n = (int)std::max<int64_t>(1, std::min<int64_t>(RowChunks::kMax, P / 64));
  for (int c = 0; c <= rc.n; ++c) rc.p0[c] = P * c / rc.n;
  // With the band loop each chunk is one launch of `ctas` persistent CTAs
  // over rows x ng items (ng G chunks per row).  Chunks whose item count is a
  // multiple of ctas end without a partial last round: 1638 rows, 16 G chunks
  // and 148 CTAs give a first chunk of 37 rows (4 rounds) and 15 of 111 rows
  // (12 rounds each; the last one shorter) instead of 16 of about 102 rows
  // (11.07 rounds each, an 8 % tail per launch).
  const bool factored = env->opt.gpp_algorithm == BGW_GPP_FACTORED ||
                        (env->opt.gpp_algorithm == BGW_GPP_AUTO && wx_stride == 0 &&
                         env->opt.precision == BGW_PRECISION_FP64);
  if (!factored && rc.n > 1) {
    const bool mixed = env->opt.precision == BGW_PRECISION_MIXED;
    int per_sm = 0;
    BGW_TRY(bandloop_per_sm_for(env->opt, &per_sm));
    const int64_t ctas = (int64_t)ws->sm_count * std::max(per_sm, 1);
    const int64_t kch = mixed ? BandCfg<true>::kCH : BandCfg<false>::kCH;
    const int64_t ng = std::max<int64_t>(1, (G + kch - 1) / kch);
    const int64_t m = ctas / std::gcd(ng, ctas);  // rows per full round set
    const int64_t even = (P + rc.n - 1) / rc.n;
    const int64_t rows = std::max<int64_t>(1, (even + m / 2) / m) * m;
    const int64_t n = (P + rows - 1) / rows;
    // The first chunk is one round set (m rows): its copy is the part of the
    // H2D transfer that no computation hides.
    const int64_t n0 = rows > m ? 1 + (P - m + rows - 1) / rows : n;
    if (rows > m && P > m && n0 >= 2 && n0 <= RowChunks::kMax) {
      rc.n = (int)n0;
      rc.p0[0] = 0;
      for (int c = 1; c <= rc.n; ++c) rc.p0[c] = std::min<int64_t>(P, m + (int64_t)(c - 1) * rows);
    } else if (n >= 2 && n <= RowChunks::kMax) {
      rc.n = (int)n;
      for (int c = 0; c <= rc.n; ++c) rc.p0[c] = std::min<int64_t>(P, (int64_t)c * rows);
    }
  }
  for (int c = 0; c < rc.n; ++c) rc.ready[c] = ws->chunk_ready[c];
  // Pageable wtilde / I_eps (the reference drivers' new[] buffers) are
  // staged through two page-locked slots filled by several host threads:
  // the memcpy of chunk c+1 overlaps the DMA of chunk c, instead of the
  // driver's single-threaded staging of every byte.
  const bool staged = P > 0 && G > 0 && (is_pageable(wt) || is_pageable(ie));
  int64_t max_rows = 0;
  for (int c = 0; c < rc.n; ++c) max_rows = std::max<int64_t>(max_rows, rc.p0[c + 1] - rc.p0[c]);
  const size_t slot_bytes = staged ? 2 * (size_t)max_rows * G * 16 : 0;
  const size_t gather_bytes = ((2 * nbp * 16 + (size_t)P * 8) + 255) & ~size_t(255);
  void *pinned = nullptr;
  BGW_TRY(ws_reserve_pinned(ws, gather_bytes + 2 * slot_bytes, &pinned));
  unsigned char *slots = static_cast<unsigned char *>(pinned) + gather_bytes;
  auto copy_rows = [&](int c) -> int {
    const size_t off = (size_t)rc.p0[c] * G * 16, bytes = (size_t)(rc.p0[c + 1] - rc.p0[c]) * G * 16;
    if (!staged) {
      BGW_TRY(h2d(static_cast<char *>(d_wt) + off, reinterpret_cast<const char *>(wt) + off, bytes));
      BGW_TRY(h2d(static_cast<char *>(d_ie) + off, reinterpret_cast<const char *>(ie) + off, bytes));
      return BGW_OK;
    }
    const int slot = c & 1;
    if (c >= 2) BGW_CUDA_TRY(cudaEventSynchronize(ws->stage_free[slot]));  // DMA of chunk c-2 done
    unsigned char *dst = slots + (size_t)slot * slot_bytes;
    const unsigned char *sw = reinterpret_cast<const unsigned char *>(wt) + off;
    const unsigned char *si = reinterpret_cast<const unsigned char *>(ie) + off;
    const int64_t blocks = (int64_t)((2 * bytes + (1 << 20) - 1) >> 20);  // 1 MiB pieces of wt | ie
    parallel_ranges(blocks, host_threads(blocks, 4), [&](int64_t b0, int64_t b1) {
      for (int64_t b = b0; b < b1; ++b) {
        const size_t lo = (size_t)b << 20, hi = std::min<size_t>(2 * bytes, lo + (1 << 20));
        for (size_t x = lo; x < hi;) {  // a piece may straddle the wt / ie boundary
          const bool in_wt = x < bytes;
          const size_t end = in_wt ? std::min(hi, bytes) : hi;
          std::memcpy(dst + x, (in_wt ? sw + x : si + (x - bytes)), end - x);
          x = end;
        }
      }
    });
    BGW_TRY(h2d(static_cast<char *>(d_wt) + off, dst, bytes));
    BGW_TRY(h2d(static_cast<char *>(d_ie) + off, dst + bytes, bytes));
    BGW_CUDA_TRY(cudaEventRecord(ws->stage_free[slot], cs));
    return BGW_OK;
  };
  // Chunk 0's wtilde / I_eps rows go first, so the copy engine works while
  // the host gathers the aqs columns below.
  BGW_TRY(copy_rows(0));

  // The kernels read aqsmtemp / aqsntemp / vcoul only at the columns
  // igp(p) = indinv[inv_igp_index[p]]: those are gathered into a page-locked
  // buffer ([nb][P] complex twice, then P doubles), so nb*P instead of nb*G
  // values cross PCIe.  With the band loop the gather and its copies go chunk
  // by chunk (columns [p0[c], p0[c+1])), so chunk c's columns are gathered
  // while the GPU works on chunk c-1 and chunk 0 waits only for its own.  An
  // out-of-range index gathers zeros; the device still resolves and checks
  // every index and reports BGW_ERR_INDEX as for device-memory inputs.
  double2 *g_am = static_cast<double2 *>(pinned), *g_an = g_am + nbp;
  double *g_vc = reinterpret_cast<double *>(g_an + nbp);
  std::vector<int64_t> igp((size_t)P);
  std::vector<int32_t> order;  // valid columns by chunk, ascending igp within a chunk
  std::vector<size_t> order_at((size_t)rc.n + 1, 0);
  order.reserve((size_t)P);
  for (int64_t p = 0; p < P; ++p) {
    const int32_t a = inv[p];
    const int64_t g = (a >= 0 && (int64_t)a < indinv_len) ? (int64_t)indinv[a] : -1;
    igp[(size_t)p] = (g >= 0 && g < G) ? g : -1;
    g_vc[p] = igp[(size_t)p] >= 0 ? vc[igp[(size_t)p]] : 0.0;
    if (igp[(size_t)p] < 0)
      for (int64_t n1 = 0; n1 < nb; ++n1) g_am[(size_t)n1 * P + p] = g_an[(size_t)n1 * P + p] = double2{0.0, 0.0};
  }
  for (int c = 0; c < rc.n; ++c) {
    order_at[(size_t)c] = order.size();
    for (int64_t p = rc.p0[c]; p < rc.p0[c + 1]; ++p)
      if (igp[(size_t)p] >= 0) order.push_back((int32_t)p);
    std::sort(order.begin() + (std::ptrdiff_t)order_at[(size_t)c], order.end(),
              [&](int32_t x, int32_t y) { return igp[(size_t)x] < igp[(size_t)y]; });
  }
  order_at[(size_t)rc.n] = order.size();
  const double2 *am2 = reinterpret_cast<const double2 *>(am), *an2 = reinterpret_cast<const double2 *>(an);
  // Gathers the columns of chunks [c0, c1) and queues their copies.
  auto gather_cols = [&](int c0, int c1) -> int {
    const int64_t p0 = rc.p0[c0], w = rc.p0[c1] - p0;
    if (w <= 0) return BGW_OK;
    const int32_t *ob = order.data() + order_at[(size_t)c0], *oe = order.data() + order_at[(size_t)c1];
    auto gather = [&](int64_t b0, int64_t b1) {
      for (int64_t n1 = b0; n1 < b1; ++n1) {
        const double2 *ra = am2 + (size_t)n1 * G, *rn = an2 + (size_t)n1 * G;
        double2 *da = g_am + (size_t)n1 * P, *dn = g_an + (size_t)n1 * P;
        for (const int32_t *q = ob; q < oe; ++q) {
          const int64_t g = igp[(size_t)*q];
          da[*q] = ra[g];
          dn[*q] = rn[g];
        }
      }
    };
    parallel_ranges(nb, host_threads(nb * w, 4096), gather);  // scattered reads: many threads
    if (nb > 0) {
      const size_t pitch = (size_t)P * 16;
      BGW_CUDA_TRY(cudaMemcpy2DAsync(static_cast<double2 *>(d_am) + p0, pitch, g_am + p0, pitch, (size_t)w * 16,
                                     (size_t)nb, cudaMemcpyHostToDevice, cs));
      BGW_CUDA_TRY(cudaMemcpy2DAsync(static_cast<double2 *>(d_an) + p0, pitch, g_an + p0, pitch, (size_t)w * 16,
                                     (size_t)nb, cudaMemcpyHostToDevice, cs));
    }
    BGW_TRY(h2d(static_cast<double *>(d_vc) + p0, g_vc + p0, sizeof(double) * (size_t)w));
    return BGW_OK;
  };
  BGW_TRY(h2d(d_inv, inv, sizeof(int32_t) * (size_t)P));
  BGW_TRY(h2d(d_ind, indinv, sizeof(int32_t) * (size_t)indinv_len));
  BGW_TRY(h2d(d_wx, wx, sizeof(double) * wx_n));
  // Band loop: chunk by chunk, hidden behind the previous chunk's kernels.
  // Factored (PCIe-bound, little GPU work per chunk): all columns at once, so
  // the host's staging of later chunks is not held up by gathers.
  BGW_TRY(gather_cols(0, factored ? rc.n : 1));
  BGW_CUDA_TRY(cudaEventRecord(ws->chunk_ready[0], cs));  // chunk 0 and the per-band inputs
  auto issue = [&](int c) -> int {
    if (c == 0) return BGW_OK;
    BGW_TRY(copy_rows(c));
    if (!factored) BGW_TRY(gather_cols(c, c + 1));
    BGW_CUDA_TRY(cudaEventRecord(ws->chunk_ready[c], cs));
    return BGW_OK;
  };
  return gpp_enqueue_chunks(env, nb, P, G, (const int32_t *)d_inv, (const int32_t *)d_ind, indinv_len,
                            (const double *)d_wx, wx_stride, (const double2 *)d_wt, (const double2 *)d_am,
                            (const double2 *)d_an, (const double2 *)d_ie, (const double *)d_vc, achtemp_dev, rc,
                            issue, (long long)P);
}

// ------------------------------------------------- screened exchange (SX) --
//
// bgw_gpp_sigma's asxtemp (the GPP model's screened exchange over the
// occupied bands; not in the reference, which has no flagOCC branch).  With
// Omega^2 / wtilde = I_eps wtilde[p][igp] (the reference's Coulomb-hole
// weight) the SX term is -2 sch_store1 I_eps wtilde / (wx^2 - wtilde^2), and
// by partial fractions wtilde / (wx^2 - wtilde^2) = (1/(wx - wtilde) -
// 1/(wx + wtilde)) / 2, so
//   asxtemp(wx) = -( Sigma_occ(wx) + Sigma_occ(-wx) ),
// Sigma_occ being the Coulomb-hole sum of the plain kernels restricted to the
// occupied bands.  The two evaluations reuse gpp_enqueue; these kernels negate
// wx and combine the results.
namespace {
__global__ void gpp_negate_kernel(const double *__restrict__ in, double *__restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = -in[i];
}
__global__ void gpp_sx_combine_kernel(const double *__restrict__ a, const double *__restrict__ b,
                                      double *__restrict__ out) {
  if (threadIdx.x < 6) out[threadIdx.x] = -(a[threadIdx.x] + b[threadIdx.x]);
}
}  // namespace

namespace {
__global__ void gpp_split12_kernel(const double *__restrict__ in, double *__restrict__ ach, double *__restrict__ asx) {
  const int k = threadIdx.x;
  if (k < 6 && ach) ach[k] = in[k];
  if (k < 6 && asx) asx[k] = in[6 + k];
}
}  // namespace

// Factored form (band-independent wx, FP64) of bgw_gpp_sigma: one prep pass
// forms S(p) over all bands and S_occ(p) over the first nv, one pass over
// wtilde / I_eps forms both outputs (gpp_factored_kernel<., true>).
// achtemp is bitwise that of gpp_enqueue's factored path.
int gpp_sigma_factored_enqueue(CallEnv *env, int64_t nb, int64_t nv, int64_t P, int64_t G, const int32_t *inv,
                               const int32_t *indinv, int64_t indinv_len, const double *wx, const double2 *wt,
                               const double2 *am, const double2 *an, const double2 *ie, const double *vc,
                               double *ach_dev, double *asx_dev) {
  Workspace *ws = env->ws;
  cudaStream_t stream = env->stream;
  const bool guard = env->opt.pole_guard > 0.0;
  const double guard2 = env->opt.pole_guard * env->opt.pole_guard;
  const int per_launch = ws->sm_count * 8;
  void *partials_v = nullptr, *tab = nullptr, *out12 = nullptr;
  BGW_TRY(ws_reserve(ws, SLOT_PARTIALS, sizeof(double) * 12 * (size_t)per_launch, &partials_v));
  BGW_TRY(ws_reserve(ws, SLOT_TABLE0, sizeof(double2) * 2 * (size_t)std::max<int64_t>(P, 1), &tab));
  BGW_TRY(ws_reserve(ws, SLOT_IN10, sizeof(double) * 12, &out12));
  double2 *S = static_cast<double2 *>(tab), *S_occ = S + std::max<int64_t>(P, 1);
  const int prep_grid = (int)std::max<long long>(1, std::min<long long>((P + 7) / 8, (long long)ws->sm_count * 16));
  gpp_prep_kernel<<<prep_grid, 256, 0, stream>>>((int)nb, (int)P, (int)G, inv, indinv, indinv_len, wt, am, an, vc,
                                                 nullptr, S, env->d_status, 0LL, (int)nv, S_occ);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  const int nchunks_g = (int)((G + kChunk - 1) / kChunk);
  const long long items = (long long)P * nchunks_g;
  // The grid of gpp_enqueue's factored launch: the same CTA partition, so
  // achtemp's partial sums (and the result) are bitwise the same.
  const int grid = (int)std::min<long long>(std::max<long long>(items, 1), (long long)per_launch);
  double *partials = static_cast<double *>(partials_v);
  BGW_TRY(prof_mark(env, 1));
  if (guard)
    gpp_factored_kernel<true, true><<<grid, kThreads, 0, stream>>>((int)G, items, nchunks_g, wt, ie, S, wx,
                                                                   partials, guard2, S_occ);
  else
    gpp_factored_kernel<false, true><<<grid, kThreads, 0, stream>>>((int)G, items, nchunks_g, wt, ie, S, wx,
                                                                    partials, 0.0, S_occ);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  BGW_TRY(prof_mark(env, 2));
  env->prof.main_bytes = 32.0 * (double)P * (double)G + 32.0 * (double)P;
  std::snprintf(env->prof.main_kernel, sizeof(env->prof.main_kernel), "gpp_factored_kernel<sx>");
  env->prof.main_launches = 1;
  reduce_partials_kernel<12><<<1, 256, 0, stream>>>(partials, grid, static_cast<double *>(out12));
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  gpp_split12_kernel<<<1, 32, 0, stream>>>(static_cast<const double *>(out12), ach_dev, asx_dev);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

int gpp_sx_enqueue(CallEnv *env, int64_t nvband, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                   int64_t indinv_len, const double *wx, size_t wx_n, int64_t wx_stride, const double2 *wt,
                   const double2 *am, const double2 *an, const double2 *ie, const double *vc, double *asx_dev) {
  void *tmp = nullptr, *wxn = nullptr;
  BGW_TRY(ws_reserve(env->ws, SLOT_IN10, sizeof(double) * 12, &tmp));
  BGW_TRY(ws_reserve(env->ws, SLOT_IN11, sizeof(double) * std::max<size_t>(wx_n, 1), &wxn));
  double *t_pos = static_cast<double *>(tmp), *t_neg = t_pos + 6;
  const int g = (int)std::min<size_t>((wx_n + 255) / 256, 1024);
  gpp_negate_kernel<<<std::max(g, 1), 256, 0, env->stream>>>(wx, static_cast<double *>(wxn), (long long)wx_n);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  BGW_TRY(gpp_enqueue(env, nvband, P, G, inv, indinv, indinv_len, wx, wx_stride, wt, am, an, ie, vc, t_pos));
  BGW_TRY(gpp_enqueue(env, nvband, P, G, inv, indinv, indinv_len, static_cast<const double *>(wxn), wx_stride, wt,
                      am, an, ie, vc, t_neg));
  gpp_sx_combine_kernel<<<1, 32, 0, env->stream>>>(t_pos, t_neg, asx_dev);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

// ------------------------------------------------------ no-allocation path --
//
// bgw_noflagOCC_solver_noalloc (include/bgw_sigma.h) serves callers that
// cannot allocate GPU memory: it evaluates the factored GPP sum with the
// kernels above, and all its scratch -- the status words, the per-column
// sums S[ngpown] and the per-CTA partials -- lives in one static device
// array compiled into the library.  The host never dereferences the array's
// name: on a device's first call the address is fetched with
// cudaGetSymbolAddress (with that device current) and cached for the life of
// the process (it belongs to the primary context; a cudaDeviceReset would
// invalidate it, which the header documents).
namespace {

constexpr int64_t kNoAllocMaxNgpown = BGW_NOALLOC_MAX_NGPOWN;
constexpr int kNoAllocMaxGrid = 2048;  // grid-stride kernel: any grid works
constexpr size_t kNoAllocStatusOff = 0;
constexpr size_t kNoAllocSOff = 256;
constexpr size_t kNoAllocPartialOff = kNoAllocSOff + sizeof(double2) * (size_t)kNoAllocMaxNgpown;
constexpr size_t kNoAllocBytes = kNoAllocPartialOff + sizeof(double) * 6 * (size_t)kNoAllocMaxGrid;
static_assert(kNoAllocBytes == BGW_NOALLOC_SCRATCH_BYTES, "scratch size must match the header");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char *g_noalloc_base[kNoAllocMaxDevices] = {};
int g_noalloc_sms[kNoAllocMaxDevices] = {};

// Once per device, with `dev` current: the device address of the scratch
// array and the SM count.
int noalloc_setup(int dev, unsigned char **base, int *sms) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_base[dev]) {
    void *p = nullptr;
    BGW_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    int n = 0;
    BGW_CUDA_TRY(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    g_noalloc_sms[dev] = n;
    g_noalloc_base[dev] = static_cast<unsigned char *>(p);
  }
  *base = g_noalloc_base[dev];
  *sms = g_noalloc_sms[dev];
  return BGW_OK;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace

}  // namespace bgw

extern "C" int bgw_noflagOCC_solver_noalloc(int64_t number_bands, int64_t ngpown, int64_t ncouls,
                                            const int32_t *inv_igp_index, const int32_t *indinv,
                                            int64_t indinv_len, const double *wx_array,
                                            const double *wtilde_array, const double *aqsmtemp,
                                            const double *aqsntemp, const double *I_eps_array,
                                            const double *vcoul, double *achtemp, int32_t device, void *stream) {
  using namespace bgw;
  const int64_t nb = number_bands, P = ngpown, G = ncouls;
  if (nb < 0 || P < 0 || G <= 0 || nb > INT32_MAX || G > INT32_MAX) return BGW_ERR_INVALID_ARG;
  if (P > kNoAllocMaxNgpown) return BGW_ERR_INVALID_ARG;  // beyond the static scratch
  if (indinv_len <= 0 || indinv_len > INT32_MAX) return BGW_ERR_INVALID_ARG;
  if (!achtemp || !wx_array || !vcoul || !indinv) return BGW_ERR_INVALID_ARG;
  if (P > 0 && (!inv_igp_index || !wtilde_array || !I_eps_array)) return BGW_ERR_INVALID_ARG;
  if (nb > 0 && P > 0 && (!aqsmtemp || !aqsntemp)) return BGW_ERR_INVALID_ARG;
  if (!aligned16(wtilde_array) || !aligned16(I_eps_array) || !aligned16(aqsmtemp) || !aligned16(aqsntemp))
    return BGW_ERR_INVALID_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
    (void)cudaGetLastError();
    return BGW_ERR_NO_DEVICE;
  }
  int dev = device;
  if (dev < 0) BGW_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= ndev || dev >= kNoAllocMaxDevices) return BGW_ERR_INVALID_ARG;
  BGW_CUDA_TRY(cudaSetDevice(dev));
  unsigned char *base = nullptr;
  int sms = 0;
  BGW_TRY(noalloc_setup(dev, &base, &sms));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int *status = reinterpret_cast<int *>(base + kNoAllocStatusOff);
  double2 *S = reinterpret_cast<double2 *>(base + kNoAllocSOff);
  double *partials = reinterpret_cast<double *>(base + kNoAllocPartialOff);

  // The scratch keeps the previous call's contents: only the status words
  // must start at zero (S and the partials are fully rewritten below).
  BGW_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int32_t) * STATUS_WORDS, s));
  const int nchunks_g = (int)((G + kChunk - 1) / kChunk);
  const long long items = (long long)P * nchunks_g;
  int prep_grid = (int)std::min<long long>((P + 7) / 8, (long long)sms * 16);
  if (prep_grid < 1) prep_grid = 1;
  gpp_prep_kernel<<<prep_grid, 256, 0, s>>>((int)nb, (int)P, (int)G, inv_igp_index, indinv, indinv_len,
                                            reinterpret_cast<const double2 *>(wtilde_array),
                                            reinterpret_cast<const double2 *>(aqsmtemp),
                                            reinterpret_cast<const double2 *>(aqsntemp), vcoul, nullptr, S, status,
                                            0LL);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  int grid = (int)std::min<long long>(std::max<long long>(items, 1), (long long)sms * 8);
  grid = std::min(grid, kNoAllocMaxGrid);
  gpp_factored_kernel<false><<<grid, kThreads, 0, s>>>((int)G, items, nchunks_g,
                                                reinterpret_cast<const double2 *>(wtilde_array),
                                                reinterpret_cast<const double2 *>(I_eps_array), S, wx_array,
                                                partials, 0.0);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  reduce_partials_kernel<6><<<1, 256, 0, s>>>(partials, grid, achtemp);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  int32_t st[STATUS_WORDS] = {0, 0, 0, 0};
  BGW_CUDA_TRY(cudaMemcpyAsync(st, status, sizeof(st), cudaMemcpyDeviceToHost, s));
  BGW_CUDA_TRY(cudaStreamSynchronize(s));
  return st[0];
}
