// ref_harness.cpp -- C entry points onto the reference's own kernels.
//
// TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline, never the
// product).  oracle/Makefile compiles the reference sources GPP/gpp.cpp and
// FF/ff.cpp unmodified, with the reference's own OpenMP 3.0 flags
// (Makefile.inc:289-323: g++ -Ofast -fstrict-aliasing -fopenmp -std=c++11
// -Dstd_complex) and `main` renamed, and links them with this file into
// oracle/_ref/libbgwref.so.  This file only wraps caller-owned buffers in
// non-owning ArrayMD views (arrayMD/arrayMD.h:156-163: the fields are public;
// size == 0 keeps the destructor from freeing, arrayMD.h:317-321) and calls
// the four reference functions through their own signatures
// (common/Defines.h:50-62, FF/ff.cpp:171-175, 211-217, 295-302).
//
// The headers compile only as C++11 (arrayMD.h:23-24 defines a global
// enable_if_t that collides with std::enable_if_t from C++14 on).
#include "common/Defines.h"

#include <array>
#include <complex>

void achsDtemp_Kernel(int number_bands, int ngpown, int ncouls,
                      ARRAY1D_int &inv_igp_index, ARRAY1D_int &indinv,
                      ARRAY2D &aqsntemp, ARRAY2D &aqsmtemp,
                      ARRAY3D &I_epsR_array, ARRAY1D_DataType &vcoul,
                      ComplexType &achsDtemp);
void asxDtemp_Kernel(int nvband, int nfreqeval, int ncouls, int ngpown,
                     int nFreq, double freqevalmin, double freqevalstep,
                     double occ, ARRAY1D_DataType &ekq,
                     ARRAY1D_DataType &dFreqGrid, ARRAY1D_int &inv_igp_index,
                     ARRAY1D_int &indinv, ARRAY2D &aqsmtemp, ARRAY2D &aqsntemp,
                     ARRAY1D_DataType &vcoul, ARRAY3D &I_epsR_array,
                     ARRAY3D &I_epsA_array, ARRAY1D &asxDtemp);
void achDtemp_cor_Kernel(int number_bands, int nvband, int nfreqeval,
                         int ncouls, int ngpown, int nFreq, double freqevalmin,
                         double freqevalstep, ARRAY1D_DataType &ekq,
                         ARRAY1D_DataType &dFreqGrid,
                         ARRAY1D_int &inv_igp_index, ARRAY1D_int &indinv,
                         ARRAY2D &aqsmtemp, ARRAY2D &aqsntemp,
                         ARRAY1D_DataType &vcoul, ARRAY3D &I_epsR_array,
                         ARRAY3D &I_epsA_array, ARRAY1D &achDtemp_cor);

namespace {

template <class T, size_t D>
struct View {
  ArrayMD<T, D, Device::cpu> a;
  View(T *p, std::array<size_t, D> ext) {
    a.m_offsets = ext;
    a.d_offsets = nullptr;
    a.size = 0;  // non-owning: ArrayMD::destroy_data frees only if size != 0
    a.subarray_offset = 0;
    a.dptr = p;
  }
};

typedef std::complex<double> cplx;

inline cplx *C(double *p) { return reinterpret_cast<cplx *>(p); }

}  // namespace

extern "C" {

// noflagOCC_solver (GPP/gpp.cpp:307-402).  achtemp: 3 complex (6 doubles).
void ref_gpp_noflagocc(long nb, long P, long G, int *inv_igp_index,
                       int *indinv, long indinv_len, double *wx_array,
                       double *wtilde, double *aqsm, double *aqsn,
                       double *I_eps, double *vcoul, double *achtemp) {
  View<int, 1> inv(inv_igp_index, {{(size_t)P}});
  View<int, 1> ind(indinv, {{(size_t)indinv_len}});
  View<double, 1> wx(wx_array, {{(size_t)(nend - nstart)}});
  View<cplx, 2> wt(C(wtilde), {{(size_t)P, (size_t)G}});
  View<cplx, 2> am(C(aqsm), {{(size_t)nb, (size_t)G}});
  View<cplx, 2> an(C(aqsn), {{(size_t)nb, (size_t)G}});
  View<cplx, 2> ie(C(I_eps), {{(size_t)P, (size_t)G}});
  View<double, 1> vc(vcoul, {{(size_t)G}});
  View<cplx, 1> out(C(achtemp), {{(size_t)(nend - nstart)}});
  noflagOCC_solver((size_t)nb, (size_t)P, (size_t)G, inv.a, ind.a, wx.a, wt.a,
                   am.a, an.a, ie.a, vc.a, out.a);
}

// achsDtemp_Kernel (FF/ff.cpp:171-209).  out: 1 complex.
void ref_ff_achs(long nb, long P, long G, long nFreq, int *inv_igp_index,
                 int *indinv, long indinv_len, double *aqsn, double *aqsm,
                 double *I_epsR, double *vcoul, double *out) {
  View<int, 1> inv(inv_igp_index, {{(size_t)P}});
  View<int, 1> ind(indinv, {{(size_t)indinv_len}});
  View<cplx, 2> an(C(aqsn), {{(size_t)nb, (size_t)G}});
  View<cplx, 2> am(C(aqsm), {{(size_t)nb, (size_t)G}});
  View<cplx, 3> R(C(I_epsR), {{(size_t)nFreq, (size_t)P, (size_t)G}});
  View<double, 1> vc(vcoul, {{(size_t)G}});
  cplx res(0.0, 0.0);
  achsDtemp_Kernel((int)nb, (int)P, (int)G, inv.a, ind.a, an.a, am.a, R.a,
                   vc.a, res);
  out[0] = res.real();
  out[1] = res.imag();
}

// asxDtemp_Kernel (FF/ff.cpp:211-293).  out: nfreqeval complex.
void ref_ff_asx(long nvband, long nfreqeval, long G, long P, long nFreq,
                double freqevalmin, double freqevalstep, double occ,
                double *ekq, long nb, double *dFreqGrid, int *inv_igp_index,
                int *indinv, long indinv_len, double *aqsm, double *aqsn,
                double *vcoul, double *I_epsR, double *I_epsA, double *out) {
  View<double, 1> e(ekq, {{(size_t)nb}});
  View<double, 1> grid(dFreqGrid, {{(size_t)nFreq}});
  View<int, 1> inv(inv_igp_index, {{(size_t)P}});
  View<int, 1> ind(indinv, {{(size_t)indinv_len}});
  View<cplx, 2> am(C(aqsm), {{(size_t)nb, (size_t)G}});
  View<cplx, 2> an(C(aqsn), {{(size_t)nb, (size_t)G}});
  View<double, 1> vc(vcoul, {{(size_t)G}});
  View<cplx, 3> R(C(I_epsR), {{(size_t)nFreq, (size_t)P, (size_t)G}});
  View<cplx, 3> A(C(I_epsA), {{(size_t)nFreq, (size_t)P, (size_t)G}});
  View<cplx, 1> o(C(out), {{(size_t)nfreqeval}});
  asxDtemp_Kernel((int)nvband, (int)nfreqeval, (int)G, (int)P, (int)nFreq,
                  freqevalmin, freqevalstep, occ, e.a, grid.a, inv.a, ind.a,
                  am.a, an.a, vc.a, R.a, A.a, o.a);
}

// achDtemp_cor_Kernel (FF/ff.cpp:295-379).  out: nfreqeval complex.
void ref_ff_cor(long nb, long nvband, long nfreqeval, long G, long P,
                long nFreq, double freqevalmin, double freqevalstep,
                double *ekq, double *dFreqGrid, int *inv_igp_index,
                int *indinv, long indinv_len, double *aqsm, double *aqsn,
                double *vcoul, double *I_epsR, double *I_epsA, double *out) {
  View<double, 1> e(ekq, {{(size_t)nb}});
  View<double, 1> grid(dFreqGrid, {{(size_t)nFreq}});
  View<int, 1> inv(inv_igp_index, {{(size_t)P}});
  View<int, 1> ind(indinv, {{(size_t)indinv_len}});
  View<cplx, 2> am(C(aqsm), {{(size_t)nb, (size_t)G}});
  View<cplx, 2> an(C(aqsn), {{(size_t)nb, (size_t)G}});
  View<double, 1> vc(vcoul, {{(size_t)G}});
  View<cplx, 3> R(C(I_epsR), {{(size_t)nFreq, (size_t)P, (size_t)G}});
  View<cplx, 3> A(C(I_epsA), {{(size_t)nFreq, (size_t)P, (size_t)G}});
  View<cplx, 1> o(C(out), {{(size_t)nfreqeval}});
  achDtemp_cor_Kernel((int)nb, (int)nvband, (int)nfreqeval, (int)G, (int)P,
                      (int)nFreq, freqevalmin, freqevalstep, e.a, grid.a,
                      inv.a, ind.a, am.a, an.a, vc.a, R.a, A.a, o.a);
}

// Number of OpenMP threads the reference build will use.
int ref_num_threads(void) {
#if defined(_OPENMP)
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
