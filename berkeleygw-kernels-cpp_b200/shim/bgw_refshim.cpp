// bgw_refshim.cpp -- link-time drop-in for the reference kernels.
//
// Defines, with the reference's exact C++ signatures (and therefore the
// same mangled symbol names), the four functions its drivers call:
//   noflagOCC_solver     common/Defines.h:50-62, GPP/gpp.cpp:307-312
//   achsDtemp_Kernel     FF/ff.cpp:171-175
//   asxDtemp_Kernel      FF/ff.cpp:211-217
//   achDtemp_cor_Kernel  FF/ff.cpp:295-302
// Each unpacks the ArrayMD arguments into pointers and extents and calls the
// C ABI of libbgwsigma.so (include/bgw_sigma.h) with host-memory options.
// The reference functions return void and have no error channel, so a
// failing call throws std::runtime_error carrying bgw_status_string().
//
// Compiled as C++11 like the reference (its headers do not build as C++14,
// arrayMD/arrayMD.h:23-24).  It does not include the reference headers: the
// ArrayMD template below repeats only what the ABI needs -- the template
// name and parameter kinds (which fix the mangled names) and the data
// member layout (arrayMD/arrayMD.h:156-163: m_offsets, d_offsets, size,
// subarray_offset, dptr).  Element type std::complex<double> is the
// reference's ComplexType (common/Defines.h:21-25, every build defines
// std_complex).
#include <array>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "bgw_sigma.h"

template <typename T, size_t dim, size_t device>
struct ArrayMD {
  std::array<size_t, dim> m_offsets;  // extents, slowest first
  size_t *d_offsets;
  size_t size;
  size_t subarray_offset;
  T *dptr;
};

namespace {

typedef std::complex<double> Cplx;
const size_t kCpu = 1;  // Device::cpu (arrayMD/arrayMD.h:32-36)

template <typename T, size_t D>
const double *dbl(ArrayMD<T, D, kCpu> &a) {
  return reinterpret_cast<const double *>(a.dptr);
}

void check(int status, const char *fn) {
  if (status != BGW_OK)
    throw std::runtime_error(std::string("libbgwsigma: ") + fn + ": " + bgw_status_string(status));
}

bgw_options host_options() {
  bgw_options o;
  bgw_options_init(&o);
  return o;
}

}  // namespace

void noflagOCC_solver(size_t number_bands, size_t ngpown, size_t ncouls, ArrayMD<int, 1, kCpu> &inv_igp_index,
                      ArrayMD<int, 1, kCpu> &indinv, ArrayMD<double, 1, kCpu> &wx_array,
                      ArrayMD<Cplx, 2, kCpu> &wtilde_array, ArrayMD<Cplx, 2, kCpu> &aqsmtemp,
                      ArrayMD<Cplx, 2, kCpu> &aqsntemp, ArrayMD<Cplx, 2, kCpu> &I_eps_array,
                      ArrayMD<double, 1, kCpu> &vcoul, ArrayMD<Cplx, 1, kCpu> &achtemp) {
  bgw_options o = host_options();
  double out[6];
  check(bgw_noflagOCC_solver((int64_t)number_bands, (int64_t)ngpown, (int64_t)ncouls, inv_igp_index.dptr,
                             indinv.dptr, (int64_t)indinv.m_offsets[0], wx_array.dptr, dbl(wtilde_array),
                             dbl(aqsmtemp), dbl(aqsntemp), dbl(I_eps_array), vcoul.dptr, out, &o),
        "noflagOCC_solver");
  for (int iw = 0; iw < 3; ++iw) achtemp.dptr[iw] = Cplx(out[2 * iw], out[2 * iw + 1]);
}

void achsDtemp_Kernel(int number_bands, int ngpown, int ncouls, ArrayMD<int, 1, kCpu> &inv_igp_index,
                      ArrayMD<int, 1, kCpu> &indinv, ArrayMD<Cplx, 2, kCpu> &aqsntemp,
                      ArrayMD<Cplx, 2, kCpu> &aqsmtemp, ArrayMD<Cplx, 3, kCpu> &I_epsR_array,
                      ArrayMD<double, 1, kCpu> &vcoul, Cplx &achsDtemp) {
  bgw_options o = host_options();
  double out[2];
  check(bgw_achsDtemp_Kernel(number_bands, ngpown, ncouls, inv_igp_index.dptr, indinv.dptr,
                             (int64_t)indinv.m_offsets[0], dbl(aqsntemp), dbl(aqsmtemp), dbl(I_epsR_array),
                             (int64_t)I_epsR_array.m_offsets[0], vcoul.dptr, out, &o),
        "achsDtemp_Kernel");
  achsDtemp = Cplx(out[0], out[1]);
}

void asxDtemp_Kernel(int nvband, int nfreqeval, int ncouls, int ngpown, int nFreq, double freqevalmin,
                     double freqevalstep, double occ, ArrayMD<double, 1, kCpu> &ekq,
                     ArrayMD<double, 1, kCpu> &dFreqGrid, ArrayMD<int, 1, kCpu> &inv_igp_index,
                     ArrayMD<int, 1, kCpu> &indinv, ArrayMD<Cplx, 2, kCpu> &aqsmtemp,
                     ArrayMD<Cplx, 2, kCpu> &aqsntemp, ArrayMD<double, 1, kCpu> &vcoul,
                     ArrayMD<Cplx, 3, kCpu> &I_epsR_array, ArrayMD<Cplx, 3, kCpu> &I_epsA_array,
                     ArrayMD<Cplx, 1, kCpu> &asxDtemp) {
  bgw_options o = host_options();
  check(bgw_asxDtemp_Kernel(nvband, nfreqeval, ncouls, ngpown, nFreq, freqevalmin, freqevalstep, occ, ekq.dptr,
                            dFreqGrid.dptr, inv_igp_index.dptr, indinv.dptr, (int64_t)indinv.m_offsets[0],
                            dbl(aqsmtemp), dbl(aqsntemp), (int64_t)aqsmtemp.m_offsets[0], vcoul.dptr,
                            dbl(I_epsR_array), dbl(I_epsA_array), reinterpret_cast<double *>(asxDtemp.dptr), &o),
        "asxDtemp_Kernel");
}

void achDtemp_cor_Kernel(int number_bands, int nvband, int nfreqeval, int ncouls, int ngpown, int nFreq,
                         double freqevalmin, double freqevalstep, ArrayMD<double, 1, kCpu> &ekq,
                         ArrayMD<double, 1, kCpu> &dFreqGrid, ArrayMD<int, 1, kCpu> &inv_igp_index,
                         ArrayMD<int, 1, kCpu> &indinv, ArrayMD<Cplx, 2, kCpu> &aqsmtemp,
                         ArrayMD<Cplx, 2, kCpu> &aqsntemp, ArrayMD<double, 1, kCpu> &vcoul,
                         ArrayMD<Cplx, 3, kCpu> &I_epsR_array, ArrayMD<Cplx, 3, kCpu> &I_epsA_array,
                         ArrayMD<Cplx, 1, kCpu> &achDtemp_cor) {
  bgw_options o = host_options();
  check(bgw_achDtemp_cor_Kernel(number_bands, nvband, nfreqeval, ncouls, ngpown, nFreq, freqevalmin, freqevalstep,
                                ekq.dptr, dFreqGrid.dptr, inv_igp_index.dptr, indinv.dptr,
                                (int64_t)indinv.m_offsets[0], dbl(aqsmtemp), dbl(aqsntemp), vcoul.dptr,
                                dbl(I_epsR_array), dbl(I_epsA_array),
                                reinterpret_cast<double *>(achDtemp_cor.dptr), &o),
        "achDtemp_cor_Kernel");
}
