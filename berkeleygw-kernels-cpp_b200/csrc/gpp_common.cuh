// gpp_common.cuh -- device helpers shared by the GPP forward and adjoint.
#pragma once

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

}  // namespace bgw
