// gpp_adjoint.cu -- analytic adjoint of the GPP sum (noflagOCC_solver,
// GPP/gpp.cpp:307-402) on sm_100a, FP64.
//
// With q = conj(d) / |d|^2 = 1 / d, d = wx[iw] - wtilde[p][ig] (gpp.cpp:374-378),
//   Sigma_iw = sum_p S(p) T(p, iw),  T(p, iw) = sum_ig I_eps[p][ig] q_iw(p, ig),
//   S(p) = C(p) wtilde[p][igp],      C(p) = sum_n1 conj(aqsm[n1][igp]) aqsn[n1][igp] 0.5 vcoul[igp].
// Sigma is holomorphic in wtilde and I_eps, so for a real loss
// L = sum_iw Re(conj(G_iw) Sigma_iw)  (G_iw = dL/dRe Sigma_iw + i dL/dIm Sigma_iw)
// the complex gradient dL/dRe z + i dL/dIm z equals sum_iw G_iw conj(dSigma_iw/dz):
//   dSigma_iw/dI_eps[p][ig]  = S(p) q_iw
//   dSigma_iw/dwtilde[p][ig] = S(p) I_eps[p][ig] q_iw^2   (+ C(p) T(p, iw) at ig = igp)
//   dSigma_iw/domega         = - sum_{p, ig} S(p) I_eps[p][ig] q_iw^2
// The quotients are recomputed (nothing of size bands x G' x G is stored).
// This is the factored form: valid for the reference's band-independent wx.
//
// One CTA streams whole G' rows (round robin, staged in chunks by bulk
// copies): it writes both gradient rows,
// reduces T(p, .) over the row with a fixed-order block sum and adds the
// sch_store1 term at (p, igp) itself, so no second pass over the row is
// needed.  dSigma/domega is reduced per CTA, then in a fixed order.
#include <algorithm>
#include <cstdio>

#include "bgw_internal.cuh"
#include "gpp_common.cuh"
#include "reduce.cuh"

namespace bgw {
namespace {

constexpr int kAdjThreads = 256;

// C(p), S(p) = C(p) wtilde[p][igp] and igp(p) (-1 if out of range).  One
// warp per column, fixed-order band sum.
__global__ void __launch_bounds__(256)
    gpp_adjoint_prep_kernel(int nb, int P, int G, const int *__restrict__ inv, const int *__restrict__ indinv,
                            long long indinv_len, const double2 *__restrict__ wt, const double2 *__restrict__ am,
                            const double2 *__restrict__ an, const double *__restrict__ vc, double2 *__restrict__ Cp,
                            double2 *__restrict__ Sp, int *__restrict__ igp_out, int *status) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < P; p += warps) {
    const int g = resolve_igp(p, inv, indinv, indinv_len, G, status);
    double cr = 0.0, ci = 0.0;
    if (g >= 0) {
      for (int n1 = lane; n1 < nb; n1 += 32) {
        double2 m = am[(size_t)n1 * G + g];
        m.y = -m.y;
        double2 r = cmul(m, an[(size_t)n1 * G + g]);
        const double v = 0.5 * vc[g];
        cr += r.x * v;
        ci += r.y * v;
      }
    }
    cr = warp_sum(cr);
    ci = warp_sum(ci);
    if (lane == 0) {
      const double2 c = make_double2(cr, ci);
      Cp[p] = c;
      Sp[p] = g >= 0 ? cmul(c, wt[(size_t)p * G + g]) : make_double2(0.0, 0.0);
      igp_out[p] = g;
    }
  }
}

__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

constexpr int kAdjChunk = 1024;  // G elements of a row per staged step

struct AdjSmem {
  double2 wt[2][kAdjChunk];
  double2 ie[2][kAdjChunk];
  unsigned long long bar[3];  // [2]: never arrived on (stall injection)
  double red[(kAdjThreads / 32) * 6];
};

// grad_wt / grad_ie may be null (not requested).  partials: 6 doubles per
// CTA (dSigma_iw/domega, re/im).  The CTA's rows are walked in chunks of
// kAdjChunk elements; thread 0 stages chunk j + 1 of wtilde / I_eps into
// shared memory with 1-D bulk copies (TMA engine, mbarrier completion,
// double-buffered) while the block computes chunk j, so HBM reads are in
// flight without costing registers.  Every wait is bounded.
__global__ void __launch_bounds__(kAdjThreads, 2)
    gpp_adjoint_kernel(int P, int G, const double2 *__restrict__ wtilde, const double2 *__restrict__ ieps,
                       const double2 *__restrict__ Cp, const double2 *__restrict__ Sp, const int *__restrict__ igp,
                       const double *__restrict__ wx3, const double2 *__restrict__ gcot,
                       double2 *__restrict__ grad_wt, double2 *__restrict__ grad_ie, double *__restrict__ partials,
                       int *status, long long stall) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  AdjSmem &sm = *reinterpret_cast<AdjSmem *>(smem_raw);
  const int tid = threadIdx.x;
  const double x[3] = {wx3[0], wx3[1], wx3[2]};
  // conj(G_iw): the cotangents enter as sum_iw conj(G_iw) dSigma_iw/dz.
  const double2 cg[3] = {cconj(gcot[0]), cconj(gcot[1]), cconj(gcot[2])};
  double dw_r[3] = {0.0, 0.0, 0.0}, dw_i[3] = {0.0, 0.0, 0.0};  // sum S I q^2 (sign applied at the end)

  const int nch = (G + kAdjChunk - 1) / kAdjChunk;
  const long long my_rows = (long long)blockIdx.x < P ? (P - 1 - (long long)blockIdx.x) / gridDim.x + 1 : 0;
  const long long nsteps = my_rows * nch;
  if (tid == 0) {
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[0]), 1);
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[1]), 1);
    mbar_init(reinterpret_cast<uint64_t *>(&sm.bar[2]), 1);
    fence_mbar_init();
  }
  __syncthreads();
  auto issue = [&](long long j) {
    const long long p = blockIdx.x + (j / nch) * (long long)gridDim.x;
    const int g0 = (int)(j % nch) * kAdjChunk;
    const int nvalid = min(kAdjChunk, G - g0);
    const int buf = (int)(j & 1);
    uint64_t *bar = reinterpret_cast<uint64_t *>(&sm.bar[buf]);
    if (!BGW_CHECKED(p < P && nvalid > 0 && nvalid <= kAdjChunk && g0 + nvalid <= G, status, 21)) {
      mbar_expect_tx(bar, 0);
      return;
    }
    mbar_expect_tx(bar, 2u * (uint32_t)nvalid * 16u);
    bulk_g2s(sm.wt[buf], wtilde + p * G + g0, (uint32_t)nvalid * 16u, bar);
    bulk_g2s(sm.ie[buf], ieps + p * G + g0, (uint32_t)nvalid * 16u, bar);
  };
  bool ok = true;
  long long j_fail = 0;  // the step whose wait ran out
  if (tid == 0 && nsteps > 0) issue(0);
  double t_r[3] = {0.0, 0.0, 0.0}, t_i[3] = {0.0, 0.0, 0.0};  // T(p, iw) (this thread)
  double u_r[3] = {0.0, 0.0, 0.0}, u_i[3] = {0.0, 0.0, 0.0};  // sum_ig I q^2 (this thread)
  for (long long j = 0; j < nsteps; ++j) {
    if (tid == 0 && j + 1 < nsteps) issue(j + 1);
    const int buf = (int)(j & 1);
    if (!staged_wait(reinterpret_cast<uint64_t *>(&sm.bar[buf]), j, stall,
                     reinterpret_cast<uint64_t *>(&sm.bar[2]))) {
      raise_status(status, BGW_ERR_TIMEOUT, blockIdx.x);
      ok = false;
    }
    if (__syncthreads_or(!ok)) {  // every thread agrees before leaving
      j_fail = j;
      break;
    }
    const long long p = blockIdx.x + (j / nch) * (long long)gridDim.x;
    const int c = (int)(j % nch);
    const int g0 = c * kAdjChunk;
    const int nvalid = min(kAdjChunk, G - g0);
    const double2 S = Sp[p];
#pragma unroll 1
    for (int k = 0; k < kAdjChunk / kAdjThreads; ++k) {
      const int idx = k * kAdjThreads + tid;
      if (idx >= nvalid) break;
      const double2 w = sm.wt[buf][idx], v = sm.ie[buf][idx];
      double2 hI = make_double2(0.0, 0.0), hW = make_double2(0.0, 0.0);
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        const double dr = x[iw] - w.x;
        const double r = rcp_refined(fma(dr, dr, w.y * w.y));
        const double2 q = make_double2(dr * r, w.y * r);  // 1 / (x - w)
        const double2 iq = cmul(v, q);                     // I q
        const double2 iq2 = cmul(iq, q);                   // I q^2
        t_r[iw] += iq.x;
        t_i[iw] += iq.y;
        u_r[iw] += iq2.x;
        u_i[iw] += iq2.y;
        hI = cadd(hI, cmul(cg[iw], q));
        hW = cadd(hW, cmul(cg[iw], iq2));
      }
      // grad = conj(sum_iw conj(G_iw) dSigma_iw/dz)
      const size_t at = (size_t)p * G + g0 + idx;
      if (grad_ie) __stcs(grad_ie + at, cconj(cmul(S, hI)));
      if (grad_wt) __stcs(grad_wt + at, cconj(cmul(S, hW)));
    }
    __syncthreads();  // buffer `buf` is free for step j + 2
    if (c == nch - 1) {
      // Row done: S u into dSigma/domega, then T(p, .) over the whole row and
      // the sch_store1 term at (p, igp): dSigma_iw/dwtilde[p][igp] += C(p) T(p, iw).
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        const double2 su = cmul(S, make_double2(u_r[iw], u_i[iw]));
        dw_r[iw] += su.x;
        dw_i[iw] += su.y;
      }
      double tv[6] = {t_r[0], t_i[0], t_r[1], t_i[1], t_r[2], t_i[2]};
      block_sum<6, kAdjThreads>(tv, sm.red);
      if (tid == 0 && grad_wt) {
        const int g = igp[p];
        if (g >= 0) {
          double2 h = make_double2(0.0, 0.0);
#pragma unroll
          for (int iw = 0; iw < 3; ++iw) h = cadd(h, cmul(cg[iw], make_double2(tv[2 * iw], tv[2 * iw + 1])));
          const double2 add = cconj(cmul(Cp[p], h));
          const double2 cur = grad_wt[(size_t)p * G + g];
          grad_wt[(size_t)p * G + g] = cadd(cur, add);
        }
      }
      __syncthreads();
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) t_r[iw] = t_i[iw] = u_r[iw] = u_i[iw] = 0.0;
    }
  }
  if (!ok && tid == 0) {
    // Copies still in flight (steps j_fail and j_fail + 1) land before the
    // CTA's shared memory is released.
    drain_staged(reinterpret_cast<uint64_t *>(&sm.bar[0]), reinterpret_cast<uint64_t *>(&sm.bar[1]), j_fail,
                 j_fail + 1 < nsteps);
  }
  double vv[6] = {-dw_r[0], -dw_i[0], -dw_r[1], -dw_i[1], -dw_r[2], -dw_i[2]};
  block_sum<6, kAdjThreads>(vv, sm.red);
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) partials[(size_t)blockIdx.x * 6 + k] = vv[k];
  }
}

// ------------------------------------------------- band-loop adjoint --
// For a band-dependent wx (wx[n1][iw]) nothing factors over bands.  With
// s(n1, p) = C(n1, p) wtilde[p][igp], C(n1, p) = conj(aqsm[n1][igp])
// aqsn[n1][igp] 0.5 vcoul[igp] and q = 1 / (wx[n1][iw] - wtilde[p][ig]):
//   dSigma_iw/dI_eps[p][ig]  = wtilde[p][igp] A'_iw,   A'_iw = sum_n1 C q
//   dSigma_iw/dwtilde[p][ig] = wtilde[p][igp] I_eps B'_iw,  B'_iw = sum_n1 C q^2
//                              (+ D_iw(p) = sum_ig I_eps A'_iw at ig = igp)
//   dSigma_iw/domega         = - sum_{p, ig} wtilde[p][igp] I_eps B'_iw.
// One item = (row p, kAbChunk elements); a thread keeps its kAbE elements
// and their A', B' in registers and walks all bands, whose C values and
// frequency rows are staged per chunk of kAbBCH bands by bulk copies
// (double-buffered, bounded waits).  The quotients are recomputed per band:
// nothing of size bands x G' x G is stored.  D_iw(p) is summed per item
// (Dpart) and added to grad_wtilde[p][igp] by gpp_adjoint_diag_kernel, in a
// fixed order.
constexpr int kAbBCH = 256;
constexpr int kAbE = 4;  // one CTA per SM (255 registers): 98 ms vs 102 ms at 2 and 101 ms at 3
constexpr int kAbChunk = kAdjThreads * kAbE;

// C(n1, p) table [P][nb], wtilde[p][igp] and igp(p) (-1 if out of range).
__global__ void __launch_bounds__(256)
    gpp_adjoint_band_prep_kernel(int nb, int P, int G, const int *__restrict__ inv, const int *__restrict__ indinv,
                                 long long indinv_len, const double2 *__restrict__ wt,
                                 const double2 *__restrict__ am, const double2 *__restrict__ an,
                                 const double *__restrict__ vc, double2 *__restrict__ Ctab,
                                 double2 *__restrict__ wpp, int *__restrict__ igp_out, int *status) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int p = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < P; p += warps) {
    const int g = resolve_igp(p, inv, indinv, indinv_len, G, status);
    for (int n1 = lane; n1 < nb; n1 += 32) {
      double2 c = make_double2(0.0, 0.0);
      if (g >= 0) {
        double2 m = am[(size_t)n1 * G + g];
        m.y = -m.y;
        c = cmul(m, an[(size_t)n1 * G + g]);
        c.x *= 0.5;
        c.y *= 0.5;
        const double v = vc[g];
        c.x *= v;
        c.y *= v;
      }
      Ctab[(size_t)p * nb + n1] = c;
    }
    if (lane == 0) {
      wpp[p] = g >= 0 ? wt[(size_t)p * G + g] : make_double2(0.0, 0.0);
      igp_out[p] = g;
    }
  }
}

__global__ void gpp_adjoint_wx_kernel(int nb, const double *__restrict__ wx, long long stride,
                                      double4 *__restrict__ wx4) {
  for (int n1 = blockIdx.x * blockDim.x + threadIdx.x; n1 < nb; n1 += gridDim.x * blockDim.x) {
    const double *w = wx + (size_t)n1 * stride;
    wx4[n1] = make_double4(w[0], w[1], w[2], 0.0);
  }
}

struct AdjBandSmem {
  double2 C[2][kAbBCH];
  double4 wx[2][kAbBCH];
  unsigned long long bar[3];  // [2]: never arrived on (stall injection)
  double red[(kAdjThreads / 32) * 6];
};

__global__ void __launch_bounds__(kAdjThreads, 1)
    gpp_adjoint_bandloop_kernel(int nb, int G, long long items, int nchunk_e, const double2 *__restrict__ wtilde,
                                const double2 *__restrict__ ieps, const double2 *__restrict__ Ctab,
                                const double2 *__restrict__ wpp, const double4 *__restrict__ wx4,
                                const double2 *__restrict__ gcot, double2 *__restrict__ grad_wt,
                                double2 *__restrict__ grad_ie, double *__restrict__ Dpart,
                                double *__restrict__ partials, int *status, long long stall) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  AdjBandSmem &sm = *reinterpret_cast<AdjBandSmem *>(smem_raw);
  const int tid = threadIdx.x;
  const double2 cg[3] = {cconj(gcot[0]), cconj(gcot[1]), cconj(gcot[2])};
  const int nbc = (nb + kAbBCH - 1) / kAbBCH;
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
  auto issue = [&](long long j) {
    const long long item = blockIdx.x + (j / nbc) * (long long)gridDim.x;
    const long long p = item / nchunk_e;
    const int b0 = (int)(j % nbc) * kAbBCH;
    const int nbv = min(kAbBCH, nb - b0);
    const int buf = (int)(j & 1);
    uint64_t *bar = reinterpret_cast<uint64_t *>(&sm.bar[buf]);
    if (!BGW_CHECKED(item < items && nbv > 0 && nbv <= kAbBCH && b0 + nbv <= nb, status, 22)) {
      mbar_expect_tx(bar, 0);
      return;
    }
    mbar_expect_tx(bar, (uint32_t)nbv * 48u);
    bulk_g2s(sm.C[buf], Ctab + p * nb + b0, (uint32_t)nbv * 16u, bar);
    bulk_g2s(sm.wx[buf], wx4 + b0, (uint32_t)nbv * 32u, bar);
  };
  bool ok = true;
  long long j_fail = 0;  // the step whose wait ran out
  if (tid == 0 && nsteps > 0) issue(0);
  double dw_r[3] = {0.0, 0.0, 0.0}, dw_i[3] = {0.0, 0.0, 0.0};  // sum wpp I B' (sign at the end)
  double2 w[kAbE], v[kAbE];
  double ar[kAbE][3], ai[kAbE][3], br[kAbE][3], bi[kAbE][3];
  for (long long j = 0; j < nsteps; ++j) {
    if (tid == 0 && j + 1 < nsteps) issue(j + 1);
    const int buf = (int)(j & 1);
    if (!staged_wait(reinterpret_cast<uint64_t *>(&sm.bar[buf]), j, stall,
                     reinterpret_cast<uint64_t *>(&sm.bar[2]))) {
      raise_status(status, BGW_ERR_TIMEOUT, blockIdx.x);
      ok = false;
    }
    if (__syncthreads_or(!ok)) {  // every thread agrees before leaving
      j_fail = j;
      break;
    }
    const long long item = blockIdx.x + (j / nbc) * (long long)gridDim.x;
    const long long p = item / nchunk_e;
    const int g0 = (int)(item % nchunk_e) * kAbChunk;
    const int c = (int)(j % nbc);
    int nbv = min(kAbBCH, nb - c * kAbBCH);
    if (!BGW_CHECKED(nbv <= kAbBCH, status, 23)) nbv = 0;
    if (c == 0) {
#pragma unroll
      for (int k = 0; k < kAbE; ++k) {
        const int ig = g0 + k * kAdjThreads + tid;
        if (ig < G) {
          w[k] = __ldcs(wtilde + p * G + ig);
          v[k] = __ldcs(ieps + p * G + ig);
        } else {
          w[k] = make_double2(0.0, 1.0);  // |wdiff| >= 1: finite, and v = 0 adds nothing
          v[k] = make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int iw = 0; iw < 3; ++iw) ar[k][iw] = ai[k][iw] = br[k][iw] = bi[k][iw] = 0.0;
      }
    }
    for (int bb = 0; bb < nbv; ++bb) {
      const double2 cb = sm.C[buf][bb];
      const double4 x4 = sm.wx[buf][bb];
      const double x[3] = {x4.x, x4.y, x4.z};
#pragma unroll
      for (int k = 0; k < kAbE; ++k) {
        const double wi2 = w[k].y * w[k].y;
#pragma unroll
        for (int iw = 0; iw < 3; ++iw) {
          const double dr = x[iw] - w[k].x;
          const double r = rcp_refined(fma(dr, dr, wi2));
          const double qr = dr * r, qi = w[k].y * r;  // q = 1 / (x - w)
          ar[k][iw] = fma(cb.x, qr, fma(-cb.y, qi, ar[k][iw]));
          ai[k][iw] = fma(cb.x, qi, fma(cb.y, qr, ai[k][iw]));
          const double q2r = fma(qr, qr, -qi * qi), q2i = 2.0 * qr * qi;
          br[k][iw] = fma(cb.x, q2r, fma(-cb.y, q2i, br[k][iw]));
          bi[k][iw] = fma(cb.x, q2i, fma(cb.y, q2r, bi[k][iw]));
        }
      }
    }
    __syncthreads();  // buffer `buf` is free for step j + 2
    if (c == nbc - 1) {
      // Item done: both gradients of its elements, its share of D(p, .) and
      // of dSigma/domega.
      const double2 wp = wpp[p];
      double dv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int k = 0; k < kAbE; ++k) {
        const int ig = g0 + k * kAdjThreads + tid;
        double2 hI = make_double2(0.0, 0.0), hW = make_double2(0.0, 0.0);
#pragma unroll
        for (int iw = 0; iw < 3; ++iw) {
          const double2 A1 = make_double2(ar[k][iw], ai[k][iw]);
          const double2 iB = cmul(v[k], cmul(wp, make_double2(br[k][iw], bi[k][iw])));  // I B
          hI = cadd(hI, cmul(cg[iw], cmul(wp, A1)));
          hW = cadd(hW, cmul(cg[iw], iB));
          const double2 iA = cmul(v[k], A1);
          dv[2 * iw] += iA.x;
          dv[2 * iw + 1] += iA.y;
          dw_r[iw] += iB.x;
          dw_i[iw] += iB.y;
        }
        if (ig < G) {
          const size_t at = (size_t)p * G + ig;
          if (grad_ie) __stcs(grad_ie + at, cconj(hI));
          if (grad_wt) __stcs(grad_wt + at, cconj(hW));
        }
      }
      block_sum<6, kAdjThreads>(dv, sm.red);
      if (tid == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) Dpart[(size_t)item * 6 + k] = dv[k];
      }
    }
  }
  if (!ok && tid == 0) {
    // Copies still in flight (steps j_fail and j_fail + 1) land before the
    // CTA's shared memory is released.
    drain_staged(reinterpret_cast<uint64_t *>(&sm.bar[0]), reinterpret_cast<uint64_t *>(&sm.bar[1]), j_fail,
                 j_fail + 1 < nsteps);
  }
  double vv[6] = {-dw_r[0], -dw_i[0], -dw_r[1], -dw_i[1], -dw_r[2], -dw_i[2]};
  block_sum<6, kAdjThreads>(vv, sm.red);
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < 6; ++k) partials[(size_t)blockIdx.x * 6 + k] = vv[k];
  }
}

// grad_wtilde[p][igp] += conj(sum_iw conj(G_iw) D_iw(p)), D summed over the
// row's items in order.  One thread per row.
__global__ void gpp_adjoint_diag_kernel(int P, int G, int nchunk_e, const double *__restrict__ Dpart,
                                        const int *__restrict__ igp, const double2 *__restrict__ gcot,
                                        double2 *__restrict__ grad_wt) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
    const int g = igp[p];
    if (g < 0) continue;
    double d[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int e = 0; e < nchunk_e; ++e) {
#pragma unroll
      for (int k = 0; k < 6; ++k) d[k] += Dpart[((size_t)p * nchunk_e + e) * 6 + k];
    }
    double2 h = make_double2(0.0, 0.0);
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) h = cadd(h, cmul(cconj(gcot[iw]), make_double2(d[2 * iw], d[2 * iw + 1])));
    const size_t at = (size_t)p * G + g;
    grad_wt[at] = cadd(grad_wt[at], cconj(h));
  }
}

}  // namespace

// Band-loop adjoint (any wx_band_stride).  Device pointers; wx holds nb rows
// of wx_stride doubles (or one shared triple when wx_stride == 0).
int gpp_adjoint_bandloop_enqueue(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv,
                                 const int32_t *indinv, int64_t indinv_len, const double *wx, int64_t wx_stride,
                                 const double2 *wt, const double2 *am, const double2 *an, const double2 *ie,
                                 const double *vc, const double2 *gcot, double2 *grad_wt, double2 *grad_ie,
                                 double *domega) {
  Workspace *ws = env->ws;
  cudaStream_t stream = env->stream;
  void *scratch_out = nullptr;
  if (!domega) {
    BGW_TRY(ws_reserve(ws, SLOT_OUT, sizeof(double) * 6, &scratch_out));
    domega = static_cast<double *>(scratch_out);
  }
  if (nb == 0 || P == 0) {  // Sigma is identically zero
    if (grad_wt) BGW_CUDA_TRY(cudaMemsetAsync(grad_wt, 0, sizeof(double2) * (size_t)P * G, stream));
    if (grad_ie) BGW_CUDA_TRY(cudaMemsetAsync(grad_ie, 0, sizeof(double2) * (size_t)P * G, stream));
    BGW_CUDA_TRY(cudaMemsetAsync(domega, 0, sizeof(double) * 6, stream));
    return BGW_OK;
  }
  const int nchunk_e = (int)((G + kAbChunk - 1) / kAbChunk);
  const long long items = (long long)P * nchunk_e;
  void *tab = nullptr, *wx4v = nullptr, *dpart = nullptr, *partials = nullptr;
  const size_t np = (size_t)P;
  // C[P][nb] | wpp[P] (double2) | igp[P] (int)
  BGW_TRY(ws_reserve(ws, SLOT_TABLE0, sizeof(double2) * (np * (size_t)nb + np) + sizeof(int) * np, &tab));
  double2 *Ctab = static_cast<double2 *>(tab);
  double2 *wpp = Ctab + np * (size_t)nb;
  int *igp = reinterpret_cast<int *>(wpp + np);
  BGW_TRY(ws_reserve(ws, SLOT_TABLE1, sizeof(double4) * (size_t)nb, &wx4v));
  BGW_TRY(ws_reserve(ws, SLOT_TABLE2, sizeof(double) * 6 * (size_t)items, &dpart));
  int prep_grid = (int)std::min<long long>((P + 7) / 8, (long long)ws->sm_count * 16);
  gpp_adjoint_band_prep_kernel<<<std::max(prep_grid, 1), 256, 0, stream>>>(
      (int)nb, (int)P, (int)G, inv, indinv, indinv_len, wt, am, an, vc, Ctab, wpp, igp, env->d_status);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  const int wgrid = (int)std::min<int64_t>((nb + 255) / 256, 1024);
  gpp_adjoint_wx_kernel<<<std::max(wgrid, 1), 256, 0, stream>>>((int)nb, wx, wx_stride, (double4 *)wx4v);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  int per_sm = 0;
  const size_t smem = sizeof(AdjBandSmem);
  BGW_CUDA_TRY(cudaFuncSetAttribute(gpp_adjoint_bandloop_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  BGW_CUDA_TRY(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gpp_adjoint_bandloop_kernel, kAdjThreads, smem));
  const int grid = (int)std::min<long long>(items, (long long)ws->sm_count * std::max(per_sm, 1));
  BGW_TRY(ws_reserve(ws, SLOT_PARTIALS, sizeof(double) * 6 * (size_t)grid, &partials));
  BGW_TRY(prof_mark(env, 1));
  gpp_adjoint_bandloop_kernel<<<grid, kAdjThreads, smem, stream>>>(
      (int)nb, (int)G, items, nchunk_e, wt, ie, Ctab, wpp, (const double4 *)wx4v, gcot, grad_wt, grad_ie,
      (double *)dpart, (double *)partials, env->d_status, stall_step());
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  BGW_TRY(prof_mark(env, 2));
  env->prof.main_launches = 1;
  env->prof.main_bytes = 32.0 * (double)P * (double)G * (1.0 + (grad_wt ? 0.5 : 0.0) + (grad_ie ? 0.5 : 0.0)) +
                         16.0 * (double)P * (double)nb;
  std::snprintf(env->prof.main_kernel, sizeof(env->prof.main_kernel), "gpp_adjoint_bandloop_kernel");
  if (grad_wt) {
    const int dgrid = (int)std::min<int64_t>((P + 255) / 256, 1024);
    gpp_adjoint_diag_kernel<<<std::max(dgrid, 1), 256, 0, stream>>>((int)P, (int)G, nchunk_e,
                                                                    (const double *)dpart, igp, gcot, grad_wt);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
  }
  reduce_partials_kernel<6><<<1, 256, 0, stream>>>((const double *)partials, grid, domega);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

// Enqueues the adjoint.  Device pointers; gcot: 3 complex cotangents;
// grad_wt / grad_ie / domega may be null.
int gpp_adjoint_enqueue(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                        int64_t indinv_len, const double *wx, const double2 *wt, const double2 *am,
                        const double2 *an, const double2 *ie, const double *vc, const double2 *gcot,
                        double2 *grad_wt, double2 *grad_ie, double *domega) {
  Workspace *ws = env->ws;
  cudaStream_t stream = env->stream;
  void *tab = nullptr, *partials = nullptr, *scratch_out = nullptr;
  const size_t np = (size_t)std::max<int64_t>(P, 1);
  // C[P] | S[P] (double2) | igp[P] (int)
  BGW_TRY(ws_reserve(ws, SLOT_TABLE0, np * (2 * sizeof(double2) + sizeof(int)), &tab));
  double2 *Cp = static_cast<double2 *>(tab);
  double2 *Sp = Cp + np;
  int *igp = reinterpret_cast<int *>(Sp + np);
  int prep_grid = (int)std::min<long long>((P + 7) / 8, (long long)ws->sm_count * 16);
  gpp_adjoint_prep_kernel<<<std::max(prep_grid, 1), 256, 0, stream>>>((int)nb, (int)P, (int)G, inv, indinv,
                                                                       indinv_len, wt, am, an, vc, Cp, Sp, igp,
                                                                       env->d_status);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  int per_sm = 0;
  const size_t smem = sizeof(AdjSmem);
  BGW_CUDA_TRY(cudaFuncSetAttribute(gpp_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  BGW_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gpp_adjoint_kernel, kAdjThreads, smem));
  int grid = (int)std::min<long long>(std::max<int64_t>(P, 1), (long long)ws->sm_count * std::max(per_sm, 1));
  BGW_TRY(ws_reserve(ws, SLOT_PARTIALS, sizeof(double) * 6 * (size_t)grid, &partials));
  if (!domega) {
    BGW_TRY(ws_reserve(ws, SLOT_OUT, sizeof(double) * 6, &scratch_out));
    domega = static_cast<double *>(scratch_out);
  }
  BGW_TRY(prof_mark(env, 1));
  gpp_adjoint_kernel<<<grid, kAdjThreads, smem, stream>>>((int)P, (int)G, wt, ie, Cp, Sp, igp, wx, gcot, grad_wt,
                                                          grad_ie, (double *)partials, env->d_status,
                                                          stall_step());
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  BGW_TRY(prof_mark(env, 2));
  env->prof.main_launches = 1;
  env->prof.main_bytes = 32.0 * (double)P * (double)G * (1.0 + (grad_wt ? 0.5 : 0.0) + (grad_ie ? 0.5 : 0.0));
  std::snprintf(env->prof.main_kernel, sizeof(env->prof.main_kernel), "gpp_adjoint_kernel");
  reduce_partials_kernel<6><<<1, 256, 0, stream>>>((const double *)partials, grid, domega);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

}  // namespace bgw
