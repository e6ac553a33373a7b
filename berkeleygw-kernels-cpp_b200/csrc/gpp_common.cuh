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

// The band sweep of the FP64 GPP band loop (gpp.cpp:360-390): for each of
// nbv bands, the kE x 3 quotients q = conj(wdiff) I_eps / |wdiff|^2 of this
// thread's elements are summed (reciprocal by rcp_refined) and multiplied by
// sch_store1 (st[b]), and the product is accumulated per frequency.  (The
// mixed form is band_sweep_mixed below.)
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

// Per step of the mixed band loop: FP32 copies of the chunk's nbv frequency
// rows (xf) and sch_store1 values (sf), and [lo, hi] of its frequencies,
// broadcast to every thread (all threads must call; two warp-level folds and
// one barrier, which also publishes xf / sf).
template <int kThreads>
__device__ __forceinline__ double2 stage_mixed_rows(const double4 *__restrict__ wx, const double2 *__restrict__ st,
                                                    int nbv, float4 *xf, float2 *sf, double *s_lo, double *s_hi) {
  double lo = INFINITY, hi = -INFINITY;
  for (int b = threadIdx.x; b < nbv; b += kThreads) {
    const double4 w = wx[b];
    const double2 v = st[b];
    xf[b] = make_float4((float)w.x, (float)w.y, (float)w.z, 0.f);
    sf[b] = make_float2((float)v.x, (float)v.y);
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

// The band sweep of the mixed band loop: the quotients of band_sweep in
// FP32 (rcp.approx.ftz.f32), their products with sch_store1 summed in FP32
// over groups of kGroup bands, each group sum added to the FP64 accumulators
// with TwoSum (one conversion and two TwoSums per kGroup bands and
// frequency: the XU and FP64 pipes stay free for the reciprocals, which
// bound this loop).
template <int kE>
__device__ __forceinline__ void band_sweep_mixed(const Elem<float> (&e)[kE], const float4 *__restrict__ xf,
                                                 const float2 *__restrict__ sf, int nbv, double (&acc_r)[3],
                                                 double (&acc_i)[3], double (&lo_r)[3], double (&lo_i)[3]) {
  constexpr int kGroup = 8;
  for (int b0 = 0; b0 < nbv; b0 += kGroup) {
    const int b1 = min(b0 + kGroup, nbv);
    float gr[3] = {0.f, 0.f, 0.f}, gi[3] = {0.f, 0.f, 0.f};
    for (int bb = b0; bb < b1; ++bb) {
      const float4 w4 = xf[bb];
      const float x[3] = {w4.x, w4.y, w4.z};
      const float2 s = sf[bb];
      float tr[3] = {0.f, 0.f, 0.f}, ti[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int k = 0; k < kE; ++k) {
#pragma unroll
        for (int iw = 0; iw < 3; ++iw) {
          const float dr = x[iw] - e[k].wr;
          const float r = rcp_approx_f32(fmaf(dr, dr, e[k].wi2));
          tr[iw] = fmaf(fmaf(dr, e[k].Ir, e[k].a), r, tr[iw]);
          ti[iw] = fmaf(fmaf(dr, e[k].Ii, e[k].b), r, ti[iw]);
        }
      }
#pragma unroll
      for (int iw = 0; iw < 3; ++iw) {
        gr[iw] = fmaf(tr[iw], s.x, gr[iw]);
        gr[iw] = fmaf(-ti[iw], s.y, gr[iw]);
        gi[iw] = fmaf(tr[iw], s.y, gi[iw]);
        gi[iw] = fmaf(ti[iw], s.x, gi[iw]);
      }
    }
#pragma unroll
    for (int iw = 0; iw < 3; ++iw) {
      two_sum_acc(acc_r[iw], lo_r[iw], (double)gr[iw]);
      two_sum_acc(acc_i[iw], lo_i[iw], (double)gi[iw]);
    }
  }
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
