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
template <bool MIXED, int kE>
__device__ __forceinline__ void band_sweep(const Elem<typename std::conditional<MIXED, float, double>::type> (&e)[kE],
                                           const double4 *__restrict__ wx, const double2 *__restrict__ st, int nbv,
                                           double (&acc_r)[3], double (&acc_i)[3], double (&lo_r)[3],
                                           double (&lo_i)[3]) {
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

}  // namespace bgw
