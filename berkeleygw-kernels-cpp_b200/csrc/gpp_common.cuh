// gpp_common.cuh -- device helpers shared by the GPP forward and adjoint.
#pragma once

#include <type_traits>

#include "bgw_internal.cuh"

namespace bgw {

// igp = indinv[inv_igp_index[p]] (GPP/gpp.cpp:362-363) with bounds checks:
// an out-of-range entry raises BGW_ERR_INDEX and returns -1 (the caller
// then treats the column as zero; no out-of-bounds read is issued).
__device__ __forceinline__ int resolve_igp(int p, const int *__restrict__ inv, const int *__restrict__ indinv,
                                           long long indinv_len, int G, int *status) {
  int a = inv[p];
  if (a < 0 || (long long)a >= indinv_len) {
    raise_status(status, BGW_ERR_INDEX, p);
    return -1;
  }
  int g = indinv[a];
  if (g < 0 || g >= G) {
    raise_status(status, BGW_ERR_INDEX, p);
    return -1;
  }
  return g;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ double2 store1(const double2 *__restrict__ am, const double2 *__restrict__ an,
                                          const double *__restrict__ vc, const double2 *__restrict__ wt, int n1,
                                          int p, int g, int G) {
  double2 m = am[(size_t)n1 * G + g];
  m.y = -m.y;
  double2 r = cmul(m, an[(size_t)n1 * G + g]);
  r.x *= 0.5;
  r.y *= 0.5;
  double v = vc[g];
  r.x *= v;
  r.y *= v;
  return cmul(r, wt[(size_t)p * G + g]);
}

// Band-independent per-element constants of the band loop (see gpp.cu).
template <typename T>
struct Elem {
  T wr, wi2, Ir, Ii, a, b;
};

// Error-free transformation of a + b (Knuth's TwoSum, TAOCP vol. 2,
// 4.2.2): hi + lo == a + b exactly, no ordering assumption.
__device__ __forceinline__ void two_sum_acc(double &hi, double &lo, double b) {
  const double s = hi + b;
  const double bb = s - hi;
  const double err = (hi - (s - bb)) + (b - bb);
  hi = s;
  lo += err;
}


// Lifts this thread's kE elements of a staged chunk into registers
// (element k of thread t is chunk index k * nthreads + t).  Padding past
// nvalid contributes exactly zero and keeps |wdiff|^2 >= 1.
template <typename T, int kE>
__device__ __forceinline__ void load_elems(Elem<T> (&e)[kE], const double2 *__restrict__ wt,
                                           const double2 *__restrict__ ie, int nvalid, int nthreads, int tid) {
#pragma unroll
  for (int k = 0; k < kE; ++k) {
    const int idx = k * nthreads + tid;
    if (idx < nvalid) {
      const double2 w = wt[idx], v = ie[idx];
      e[k].wr = (T)w.x;
      e[k].wi2 = (T)(w.y * w.y);
      e[k].Ir = (T)v.x;
      e[k].Ii = (T)v.y;
      e[k].a = (T)(-w.y * v.y);
      e[k].b = (T)(w.y * v.x);
    } else {
      e[k].wr = (T)0;
      e[k].wi2 = (T)1;
      e[k].Ir = e[k].Ii = e[k].a = e[k].b = (T)0;
    }
  }
}

// The band sweep of the FP64 GPP band loop (gpp.cpp:360-390): for each of
// nbv bands, the kE x 3 quotients q = conj(wdiff) I_eps / |wdiff|^2 of this
// thread's elements are summed (reciprocal by rcp_refined) and multiplied by
// sch_store1 (st[b]), and the product is accumulated per frequency.  (The
// mixed form is rem_stage / rem_elems / rem_sweep below.)
// GUARD: a term with |wdiff|^2 < guard2 contributes zero (near-pole cut-off;
// the select discards the reciprocal, so a zero |wdiff| yields no NaN).
template <int kE, bool GUARD = false>
__device__ __forceinline__ void band_sweep(const Elem<double> (&e)[kE], const double4 *__restrict__ wx,
                                           const double2 *__restrict__ st, int nbv, double (&acc_r)[3],
                                           double (&acc_i)[3], double guard2 = 0.0) {
  for (int bb = 0; bb < nbv; ++bb) {
    const double4 w4 = wx[bb];
    const double x[3] = {w4.x, w4.y, w4.z};
    const double2 s = st[bb];
    double tr[3] = {0.0, 0.0, 0.0}, ti[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < kE; ++k) {
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        const double dr = x[iw] - e[k].wr;
        const double den = fma(dr, dr, e[k].wi2);
        double r = rcp_refined(den);
        if constexpr (GUARD) r = den < guard2 ? 0.0 : r;
        const double nr = fma(dr, e[k].Ir, e[k].a);
        const double ni = fma(dr, e[k].Ii, e[k].b);
        tr[iw] = fma(nr, r, tr[iw]);
        ti[iw] = fma(ni, r, ti[iw]);
      }
    }
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) {
      acc_r[iw] = fma(tr[iw], s.x, acc_r[iw]);
      acc_r[iw] = fma(-ti[iw], s.y, acc_r[iw]);
      acc_i[iw] = fma(tr[iw], s.y, acc_i[iw]);
      acc_i[iw] = fma(ti[iw], s.x, acc_i[iw]);
    }
  }
}

// ----------------------------------- mixed band loop: hoisted expansion --
//
// The mixed-precision band loop evaluates each element's quotients about a
// centre c of the step's band-chunk frequencies.  With w = wtilde[p][ig],
// I = I_eps[p][ig], u = 1 / (c - w), Q0 = I u, delta = x - c and t = delta u,
//   q = I / (x - w) = Q0 / (1 + t)
//     = Q0 sum_{k<K} (-t)^k + (-t)^K Q0 / (1 + t)             (exact, any K),
// so the band sum of a (p, ig) element is
//   sum_b s_b q_b = Q0 sum_{k<K} (-u)^k S_k + sum_b s_b (-delta_b)^K (X + delta_b Y) / |1 + t_b|^2,
// with band moments S_k = sum_b s_b delta_b^k (FP64, once per step),
// X = Q0 u^K, Y = X conj(u) (per element) and |1 + t|^2 = 1 + 2 delta Re u +
// delta^2 |u|^2.  The first part (the K hoisted Taylor terms) is evaluated in
// FP64 once per element and step; the remainder is a per-term complex
// quotient evaluated in FP32, whose value is |t|^K of the term, so its
// FP32 rounding costs ~eps32 |t|^K of the term instead of eps32.  K = 0 is a
// plain FP32 quotient.  Elements with |t| > kRemTau for some term of the
// step (near a pole) take the FP64 path (near_sweep), as do elements a
// pole_guard cut could reach.
//
// The remainder's denominators lie in [(1 - tau)^2, (1 + tau)^2], so one
// reciprocal serves two frequencies of an element: R = 1 / (d0 d1),
// 1/d0 = d1 R, 1/d1 = d0 R (no overflow or underflow can occur in that
// range); the third has its own.  Two elements are processed per packed
// f32x2 instruction.  (An f32x2 FMA occupies both halves of the FMA pipe, so
// packing saves issue slots, not pipe time; the measured limits are the FMA
// pipe and dependent-instruction latency, hence two accumulator sets.)
constexpr double kRemTau = 0.125;

// Per band of a step: (2 delta, 2 delta), (delta^2, delta^2), (delta, delta)
// for each frequency, and the band multiplier m = s_b (-delta)^K split into
// (Re m, Re m), (Im m, Im m), (-Im m, -Im m) (pairs: operands of f32x2 ops).
struct RemRow {
  float2 d2x[3], dd[3], d[3], mr[3], mi[3], nmi[3];
};

// Centre, half-width and FP64 band moments of a step.
struct RemStep {
  double c, dmax;
  double2 S[3][3];  // S[k][iw] = sum_b s_b delta_b^k (k < 3)
};

// Every thread calls: folds the frequency range of the step's nbv bands,
// writes rows[b] and returns the centre, half-width and moments (identical
// in every thread; fixed summation order).  red: (kThreads / 32) * 18
// doubles; s_lo / s_hi: kThreads / 32 doubles each.
template <int kThreads, int K>
__device__ __forceinline__ RemStep rem_stage(const double4 *__restrict__ wx, const double2 *__restrict__ st, int nbv,
                                             RemRow *rows, double *red, double *s_lo, double *s_hi) {
  constexpr int kW = kThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double lo = INFINITY, hi = -INFINITY;
  for (int b = threadIdx.x; b < nbv; b += kThreads) {
    const double4 w = wx[b];
    lo = fmin(lo, fmin(w.x, fmin(w.y, w.z)));
    hi = fmax(hi, fmax(w.x, fmax(w.y, w.z)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if (lane == 0) {
    s_lo[warp] = lo;
    s_hi[warp] = hi;
  }
  __syncthreads();
#pragma unroll
  for (int w = 0; w < kW; ++w) {
    lo = fmin(lo, s_lo[w]);
    hi = fmax(hi, s_hi[w]);
  }
  RemStep r;
  r.c = 0.5 * (lo + hi);
  r.dmax = 0.5 * (hi - lo);
  // Moments: v[(k * 3 + iw) * 2 + {re, im}] = sum_b s_b delta^k.
  double v[18];
#pragma unroll
  for (int i = 0; i < 18; ++i) v[i] = 0.0;
  for (int b = threadIdx.x; b < nbv; b += kThreads) {
    const double4 w4 = wx[b];
    const double x[3] = {w4.x, w4.y, w4.z};
    const double2 sb = st[b];
    RemRow row;
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) {
      const double d = x[iw] - r.c, d2 = d * d;
      double pk = 1.0;  // (-delta)^K
#pragma unroll
      for (int k = 0; k < K; ++k) pk *= -d;
      const float fd = (float)d, fd2 = (float)d2, f2d = (float)(2.0 * d);
      row.d2x[iw] = make_float2(f2d, f2d);
      row.dd[iw] = make_float2(fd2, fd2);
      row.d[iw] = make_float2(fd, fd);
      const float mr = (float)(sb.x * pk), mi = (float)(sb.y * pk);
      row.mr[iw] = make_float2(mr, mr);
      row.mi[iw] = make_float2(mi, mi);
      row.nmi[iw] = make_float2(-mi, -mi);
      v[(0 * 3 + iw) * 2 + 0] += sb.x;
      v[(0 * 3 + iw) * 2 + 1] += sb.y;
      v[(1 * 3 + iw) * 2 + 0] += sb.x * d;
      v[(1 * 3 + iw) * 2 + 1] += sb.y * d;
      v[(2 * 3 + iw) * 2 + 0] += sb.x * d2;
      v[(2 * 3 + iw) * 2 + 1] += sb.y * d2;
    }
    rows[b] = row;
  }
  // Every thread forms the same totals: warp butterflies, then the warp
  // partials in warp order.
#pragma unroll
  for (int i = 0; i < 18; ++i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
  }
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < 18; ++i) red[warp * 18 + i] = v[i];
  }
  __syncthreads();  // also publishes rows[]
#pragma unroll
  for (int i = 0; i < 18; ++i) {
    double t = red[i];
    for (int w = 1; w < kW; ++w) t += red[w * 18 + i];
    v[i] = t;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) r.S[k][iw] = make_double2(v[(k * 3 + iw) * 2], v[(k * 3 + iw) * 2 + 1]);
  return r;
}

// Per-element FP32 constants of the remainder, two elements per pair.
template <int kE>
struct RemElems {
  float2 ur[kE / 2], uu[kE / 2], Xr[kE / 2], Xi[kE / 2], Yr[kE / 2], Yi[kE / 2];
};

__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // a * conj(b)
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// This thread's kE elements of the staged chunk (element k is chunk index
// k * nthreads + tid): the FP64 hoisted part is added to acc_r / acc_i, the
// FP32 constants of the remainder are set, and the near elements (returned
// as a bit mask) get zero constants (their remainder then adds exactly
// zero).  guard2 > 0: elements a pole_guard cut could reach are near too.
template <int kE, int K>
__device__ __forceinline__ uint32_t rem_elems(RemElems<kE> &e, const double2 *__restrict__ wt,
                                              const double2 *__restrict__ ie, int nvalid, int nthreads, int tid,
                                              const RemStep &r, double guard2, double (&acc_r)[3],
                                              double (&acc_i)[3]) {
  uint32_t near = 0;
  const double tau2 = kRemTau * kRemTau, far2 = (1.0 - kRemTau) * (1.0 - kRemTau);
#pragma unroll
  for (int k = 0; k < kE; ++k) {
    float ur = 0.f, uu = 0.f, xr = 0.f, xi = 0.f, yr = 0.f, yi = 0.f;
    const int idx = k * nthreads + tid;
    if (idx < nvalid) {
      const double2 w = wt[idx], v = ie[idx];
      const double dr = r.c - w.x;
      const double D = fma(dr, dr, w.y * w.y);  // |c - w|^2
      const double rD = rcp_refined(D);
      // |t| <= dmax |u| <= tau for every term; a guard cut needs
      // |x - w| >= (1 - tau) / |u| < delta.  (D = 0 is near: rD = inf.)
      const bool is_near = !(r.dmax * r.dmax * rD <= tau2) || (guard2 > 0.0 && guard2 * rD > far2);
      if (is_near) {
        near |= 1u << k;
      } else {
        const double2 u = make_double2(dr * rD, w.y * rD);  // 1 / (c - w)
        const double2 Q0 = cmul(v, u);
        const double2 mu = make_double2(-u.x, -u.y);
#pragma unroll
        for (int iw = 0; iw < 3; ++iw) {
          // Q0 (S_0 + (-u) (S_1 + (-u) S_2)) truncated to K terms (Horner).
          double2 h = make_double2(0.0, 0.0);
#pragma unroll
          for (int j = K - 1; j >= 0; --j) {
            const double2 t = cmul(mu, h);
            h = make_double2(r.S[j][iw].x + t.x, r.S[j][iw].y + t.y);
          }
          const double2 p = cmul(Q0, h);
          acc_r[iw] += p.x;
          acc_i[iw] += p.y;
        }
        double2 X = Q0;
#pragma unroll
        for (int j = 0; j < K; ++j) X = cmul(X, u);
        const double2 Y = cmulc(X, u);
        ur = (float)u.x;
        uu = (float)rD;  // |u|^2 = 1 / |c - w|^2
        xr = (float)X.x;
        xi = (float)X.y;
        yr = (float)Y.x;
        yi = (float)Y.y;
      }
    }
    if (k & 1) {
      e.ur[k >> 1].y = ur, e.uu[k >> 1].y = uu, e.Xr[k >> 1].y = xr, e.Xi[k >> 1].y = xi;
      e.Yr[k >> 1].y = yr, e.Yi[k >> 1].y = yi;
    } else {
      e.ur[k >> 1].x = ur, e.uu[k >> 1].x = uu, e.Xr[k >> 1].x = xr, e.Xi[k >> 1].x = xi;
      e.Yr[k >> 1].x = yr, e.Yi[k >> 1].x = yi;
    }
  }
  return near;
}

// The remainder's band sweep: for each band, T_iw = sum over this thread's
// elements of (X + delta Y) / |1 + t|^2 (packed FP32, two reciprocals per
// element for the three frequencies), times the band multiplier m; the
// products are summed in FP32 over groups of kRemGroup bands and each group
// sum is added to the FP64 accumulators with TwoSum.
constexpr int kRemGroup = 8;

__device__ __forceinline__ float rcp_f32(float d) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
  return y;
}

template <int kE>
__device__ __forceinline__ void rem_sweep(const RemElems<kE> &e, const RemRow *__restrict__ rows, int nbv,
                                          double (&acc_r)[3], double (&acc_i)[3], double (&lo_r)[3],
                                          double (&lo_i)[3]) {
  const float2 one = make_float2(1.f, 1.f);
  for (int b0 = 0; b0 < nbv; b0 += kRemGroup) {
    const int b1 = min(b0 + kRemGroup, nbv);
    float2 gr[3], gi[3];
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) gr[iw] = gi[iw] = make_float2(0.f, 0.f);
    for (int b = b0; b < b1; ++b) {
      const RemRow &R = rows[b];
      // Two accumulator sets (even / odd element pairs) shorten the chains of
      // dependent FMAs.
      float2 tr[2][3], ti[2][3];
#pragma unroll
      for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int iw = 0; iw < 3; ++iw) tr[h][iw] = ti[h][iw] = make_float2(0.f, 0.f);
#pragma unroll
      for (int q = 0; q < kE / 2; ++q) {
        float2 den[3];
#pragma unroll
        for (int iw = 0; iw < 3; ++iw) den[iw] = __ffma2_rn(R.dd[iw], e.uu[q], __ffma2_rn(R.d2x[iw], e.ur[q], one));
        const float2 P = __fmul2_rn(den[0], den[1]);
        const float2 Ri = make_float2(rcp_f32(P.x), rcp_f32(P.y));
        float2 rc[3];
        rc[0] = __fmul2_rn(den[1], Ri);
        rc[1] = __fmul2_rn(den[0], Ri);
        rc[2] = make_float2(rcp_f32(den[2].x), rcp_f32(den[2].y));
#pragma unroll
        for (int iw = 0; iw < 3; ++iw) {
          const float2 nr = __ffma2_rn(R.d[iw], e.Yr[q], e.Xr[q]);
          const float2 ni = __ffma2_rn(R.d[iw], e.Yi[q], e.Xi[q]);
          tr[q & 1][iw] = __ffma2_rn(nr, rc[iw], tr[q & 1][iw]);
          ti[q & 1][iw] = __ffma2_rn(ni, rc[iw], ti[q & 1][iw]);
        }
      }
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        tr[0][iw] = __fadd2_rn(tr[0][iw], tr[1][iw]);
        ti[0][iw] = __fadd2_rn(ti[0][iw], ti[1][iw]);
      }
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        gr[iw] = __ffma2_rn(R.mr[iw], tr[0][iw], __ffma2_rn(R.nmi[iw], ti[0][iw], gr[iw]));
        gi[iw] = __ffma2_rn(R.mr[iw], ti[0][iw], __ffma2_rn(R.mi[iw], tr[0][iw], gi[iw]));
      }
    }
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) {
      two_sum_acc(acc_r[iw], lo_r[iw], (double)gr[iw].x + (double)gr[iw].y);
      two_sum_acc(acc_i[iw], lo_i[iw], (double)gi[iw].x + (double)gi[iw].y);
    }
  }
}

// ------------------------------------------- mixed band loop near poles --
// The FP64 sum of the near elements over the chunk's bands, each product
// with sch_store1 added to the TwoSum accumulators; terms with |wdiff|^2 <
// guard2 are skipped (guard2 = 0: none).
__device__ __forceinline__ void near_sweep(uint32_t near, const double2 *__restrict__ wt, const double2 *__restrict__ ie,
                                        int nthreads, int tid, const double4 *__restrict__ wx,
                                        const double2 *__restrict__ st, int nbv, double guard2, double (&acc_r)[3],
                                        double (&acc_i)[3], double (&lo_r)[3], double (&lo_i)[3]) {
  while (near) {
    const int k = __ffs(near) - 1;
    near &= near - 1;
    const int idx = k * nthreads + tid;
    const double2 w = wt[idx], v = ie[idx];
    const double wi2 = w.y * w.y, a = -w.y * v.y, b = w.y * v.x;
    for (int bb = 0; bb < nbv; ++bb) {
      const double4 w4 = wx[bb];
      const double x[3] = {w4.x, w4.y, w4.z};
      const double2 s = st[bb];
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        const double dr = x[iw] - w.x;
        const double den = fma(dr, dr, wi2);
        if (den < guard2) continue;
        const double r = rcp_refined(den);
        const double qr = fma(dr, v.x, a) * r, qi = fma(dr, v.y, b) * r;
        two_sum_acc(acc_r[iw], lo_r[iw], fma(qr, s.x, -qi * s.y));
        two_sum_acc(acc_i[iw], lo_i[iw], fma(qr, s.y, qi * s.x));
      }
    }
  }
}

}  // namespace bgw
