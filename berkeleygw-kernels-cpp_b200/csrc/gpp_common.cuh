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

__device__ __forceinline__ float rcp_approx_f32(float d) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
  return y;
}

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

// The band sweep of the GPP band loop (gpp.cpp:360-390): for each of nbv
// bands, the kE x 3 quotients q = conj(wdiff) I_eps / |wdiff|^2 of this
// thread's elements are summed and multiplied by sch_store1 (st[b]), and the
// product is accumulated per frequency.  FP64: reciprocal by rcp_refined.
// MIXED: quotients and their per-band partial in FP32, the product and the
// accumulation in FP64 with TwoSum tails (lo_r / lo_i).
// GUARD: a term with |wdiff|^2 < guard2 contributes zero (near-pole cut-off;
// the select discards the reciprocal, so a zero |wdiff| yields no NaN).
template <bool MIXED, int kE, bool GUARD = false>
__device__ __forceinline__ void band_sweep(const Elem<typename std::conditional<MIXED, float, double>::type> (&e)[kE],
                                           const double4 *__restrict__ wx, const double2 *__restrict__ st, int nbv,
                                           double (&acc_r)[3], double (&acc_i)[3], double (&lo_r)[3],
                                           double (&lo_i)[3], double guard2 = 0.0) {
  using T = typename std::conditional<MIXED, float, double>::type;
  for (int bb = 0; bb < nbv; ++bb) {
    const double4 w4 = wx[bb];
    const T x[3] = {(T)w4.x, (T)w4.y, (T)w4.z};
    const double2 s = st[bb];
    T tr[3] = {(T)0, (T)0, (T)0}, ti[3] = {(T)0, (T)0, (T)0};
#pragma unroll
    for (int k = 0; k < kE; ++k) {
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        const T dr = x[iw] - e[k].wr;
        const T den = fma(dr, dr, e[k].wi2);
        T r;
        if constexpr (MIXED) {
          r = rcp_approx_f32(den);
        } else {
          r = rcp_refined(den);
        }
        if constexpr (GUARD) r = den < (T)guard2 ? (T)0 : r;
        const T nr = fma(dr, e[k].Ir, e[k].a);
        const T ni = fma(dr, e[k].Ii, e[k].b);
        tr[iw] = fma(nr, r, tr[iw]);
        ti[iw] = fma(ni, r, ti[iw]);
      }
    }
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) {
      const double trd = (double)tr[iw], tid_ = (double)ti[iw];
      if constexpr (MIXED) {
        two_sum_acc(acc_r[iw], lo_r[iw], fma(trd, s.x, -tid_ * s.y));
        two_sum_acc(acc_i[iw], lo_i[iw], fma(trd, s.y, tid_ * s.x));
      } else {
        acc_r[iw] = fma(trd, s.x, acc_r[iw]);
        acc_r[iw] = fma(-tid_, s.y, acc_r[iw]);
        acc_i[iw] = fma(trd, s.y, acc_i[iw]);
        acc_i[iw] = fma(tid_, s.x, acc_i[iw]);
      }
    }
  }
}

// ------------------------------------------- mixed band loop near poles --
// The FP32 quotient's error grows like eps32 (|x| + |wr|) / |x - wr|: near a
// pole the subtraction cancels.  The mixed band loop therefore sends every
// element whose wtilde real part wr lies near the band chunk's frequency
// range to an FP64 path.  With the chunk's frequencies in [lo, hi], an
// element is "far" when
//   wr >= hi + max(kNearFrac |hi|, delta)   or   wr <= lo - max(kNearFrac |lo|, delta);
// then every term has |x - wr| >= kNearFrac |x| (so the FP32 relative error
// is at most eps32 (2 / kNearFrac + 1)) and |wdiff| >= |x - wr| >= delta (so
// the near-pole guard cannot fire and the FP32 path needs no test).  Near
// elements are zeroed in the FP32 copy and summed in FP64, guard included.
constexpr double kNearFrac = 0.25;

// [lo, hi] of the frequencies of the chunk's nbv bands, broadcast to every
// thread (all threads must call; two warp-level folds and one barrier).
template <int kThreads>
__device__ __forceinline__ double2 chunk_wx_range(const double4 *__restrict__ wx, int nbv, double *s_lo,
                                                  double *s_hi) {
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
  if ((threadIdx.x & 31) == 0) {
    s_lo[threadIdx.x >> 5] = lo;
    s_hi[threadIdx.x >> 5] = hi;
  }
  __syncthreads();
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) {
    lo = fmin(lo, s_lo[w]);
    hi = fmax(hi, s_hi[w]);
  }
  return make_double2(lo, hi);
}

// Marks this thread's near elements (bit k for element k) and zeroes their
// FP32 copies (the padding values: they then add exactly zero).
template <int kE>
__device__ __forceinline__ uint32_t near_elems(Elem<float> (&e)[kE], const double2 *__restrict__ wt, int nvalid,
                                               int nthreads, int tid, double2 xr, double guard_d) {
  const double m = 1.0 + 1e-9;  // covers the rounding of the bounds below
  const double blo = xr.x - fmax(kNearFrac * fabs(xr.x), guard_d) * m;
  const double bhi = xr.y + fmax(kNearFrac * fabs(xr.y), guard_d) * m;
  uint32_t near = 0;
#pragma unroll
  for (int k = 0; k < kE; ++k) {
    const int idx = k * nthreads + tid;
    if (idx < nvalid) {
      const double wr = wt[idx].x;
      if (wr > blo && wr < bhi) {
        near |= 1u << k;
        e[k].wr = 0.f;
        e[k].wi2 = 1.f;
        e[k].Ir = e[k].Ii = e[k].a = e[k].b = 0.f;
      }
    }
  }
  return near;
}

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
