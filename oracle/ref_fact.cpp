// ref_fact.cpp -- the reference's own compute_fact (FF/ff.cpp:103-152) made
// callable for the golden probe table.
//
// TEST INFRASTRUCTURE ONLY.  compute_fact is an inline helper of ff.cpp with
// no symbol of its own, so this translation unit includes FF/ff.cpp
// unmodified (oracle/Makefile compiles it with the reference's flags and
// -I$(REF)/FF).  `main` and the three kernels are renamed by macros first:
// their definitions for libbgwref.so come from ff_ref.o, and this file adds
// only the probe below.
#define main bgw_ref_fact_unused_main
#define achsDtemp_Kernel bgw_ref_fact_unused_achs
#define asxDtemp_Kernel bgw_ref_fact_unused_asx
#define achDtemp_cor_Kernel bgw_ref_fact_unused_cor
#include "ff.cpp"
#undef main
#undef achsDtemp_Kernel
#undef asxDtemp_Kernel
#undef achDtemp_cor_Kernel

// (ifreq, fact1, fact2) of compute_fact(wx, nFreq, grid, ., ., ., loop,
// flag_occ), the outputs starting at 0 as at the reference's call sites
// (FF/ff.cpp:247-252, 338-342).  grid: nFreq doubles (a non-owning ArrayMD
// view, arrayMD/arrayMD.h:156-163, 317-321).
extern "C" void ref_compute_fact(double wx, int nFreq, double *grid, int loop, int flag_occ, int *ifreq,
                                 double *fact1, double *fact2) {
  ARRAY1D_DataType g;
  g.m_offsets = {(size_t)nFreq};
  g.d_offsets = nullptr;
  g.size = 0;
  g.subarray_offset = 0;
  g.dptr = grid;
  double f1 = 0.00, f2 = 0.00;
  int i = 0;
  compute_fact(wx, nFreq, g, f1, f2, i, loop, flag_occ != 0);
  g.dptr = nullptr;
  *ifreq = i;
  *fact1 = f1;
  *fact2 = f2;
}
