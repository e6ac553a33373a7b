/*
 * bgw_oracle.c -- CPU oracle for the GPP and full-frequency self-energy sums.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load the library built from it.  The product path (libbgwsigma.so) never
 * links or calls anything here.
 *
 * It restates, in long double (x87 80-bit) arithmetic, the algorithms of the
 * reference mini-apps (rgayatri23/BerkeleyGW-Kernels-CPP):
 *   - GPP  noflagOCC_solver             GPP/gpp.cpp:307-402
 *   - FF   compute_fact                 FF/ff.cpp:103-152
 *   - FF   achsDtemp_Kernel             FF/ff.cpp:171-209
 *   - FF   asxDtemp_Kernel (+ssxDittt)  FF/ff.cpp:154-169, 211-293
 *   - FF   achDtemp_cor_Kernel (+schDttt_corKernel1/2)  FF/ff.cpp:295-451
 * and the analytic gradient of the GPP sum (orc_gpp_backward), which the
 * reference does not have; that gradient is pinned by central finite
 * differences of the long-double forward (tests/test_adjoint.py).
 *
 * Every sum is accumulated in long double and combined in a fixed order, so
 * the result does not depend on the OpenMP thread count.  The oracle is
 * pinned (i) against closed-form known answers of the reference's own uniform
 * fills and (ii) against the reference sources compiled unmodified into
 * oracle/_ref/libbgwref.so (see oracle/Makefile and tests/golden/).
 *
 * Complex arrays are interleaved (re, im) doubles, row-major with the last
 * index fastest, exactly the memory image of ArrayMD<std::complex<double>>
 * (arrayMD/arrayMD.h:156-184).
 *
 * All functions return 0 on success and -1 on an out-of-range size or index,
 * without touching memory outside the stated extents.
 */
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

typedef long double ld;

/* Resolve igp = indinv[inv_igp_index[p]] with bounds checks (gpp.cpp:362-363,
 * ff.cpp:183-184).  Returns -1 if an index is out of range. */
static int resolve_igp(long P, long G, const int *inv_igp_index,
                       const int *indinv, long indinv_len, long *igp_out) {
  for (long p = 0; p < P; ++p) {
    int a = inv_igp_index[p];
    if (a < 0 || (long)a >= indinv_len) return -1;
    int b = indinv[a];
    if (b < 0 || (long)b >= G) return -1;
    igp_out[p] = b;
  }
  return 0;
}

/* ------------------------------------------------------------------ GPP -- */

/* sch_store1 of gpp.cpp:369-371:
 *   conj(aqsm[n1][igp]) * aqsn[n1][igp] * 0.5 * vcoul[igp] * wtilde[p][igp] */
static void gpp_store1(const double *am, const double *an, double vc,
                       const double *wt, ld *sr, ld *si) {
  ld ar = am[0], ai = -(ld)am[1];       /* conj(aqsm) */
  ld br = an[0], bi = an[1];
  ld r = ar * br - ai * bi, i = ar * bi + ai * br;
  r *= 0.5L; i *= 0.5L;
  r *= (ld)vc; i *= (ld)vc;
  ld cr = wt[0], ci = wt[1];
  *sr = r * cr - i * ci;
  *si = r * ci + i * cr;
}

/* Near-pole guard (not in the reference, which has none; specified from
 * first principles): with delta > 0 a pole term 1/(w - wtilde) whose
 * |w - wtilde|^2 is below delta^2 is left out of the sum.  0 (the default)
 * keeps every term, as the reference does.  Set by orc_set_pole_guard; read
 * by gpp_quot and sx_term. */
static ld g_pole_guard2 = 0.0L;

void orc_set_pole_guard(double delta) { g_pole_guard2 = (ld)delta * (ld)delta; }

static int guarded(ld dr, ld di) { return g_pole_guard2 > 0.0L && dr * dr + di * di < g_pole_guard2; }

/* One (my_igp, ig, iw) quotient of gpp.cpp:374-380 without sch_store1:
 *   conj(wdiff) / |wdiff|^2 * I_eps,  wdiff = wx - wtilde. */
static void gpp_quot(double wx, const double *wt, const double *ie, ld *qr,
                     ld *qi) {
  ld dr = (ld)wx - (ld)wt[0];
  ld di = -(ld)wt[1];
  if (guarded(dr, di)) { *qr = 0.0L; *qi = 0.0L; return; }
  ld rcp = 1.0L / (dr * dr + di * di);
  ld cr = dr * rcp, ci = -di * rcp;      /* conj(wdiff) * rcp */
  ld er = ie[0], ei = ie[1];
  *qr = cr * er - ci * ei;
  *qi = cr * ei + ci * er;
}

/* Direct restatement of the n1 x my_igp x ig x iw loop of gpp.cpp:343-390.
 * wx is read as wx[n1 * wx_band_stride + iw]; stride 0 is the reference
 * (wx_array has no band index, gpp.cpp:239).  achtemp receives 3 complex
 * values (6 doubles).  Cost O(nb * P * G * 3): small sizes only. */
static int gpp_direct_ld(long nb, long P, long G, const int *inv_igp_index,
                         const int *indinv, long indinv_len, const double *wx,
                         long wx_band_stride, const double *wtilde,
                         const double *aqsm, const double *aqsn,
                         const double *I_eps, const double *vcoul, ld *out) {
  if (nb < 0 || P < 0 || G <= 0 || wx_band_stride < 0) return -1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(nb > 0 ? nb : 1) * 6, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (long n1 = 0; n1 < nb; ++n1) {
    ld acc[6] = {0, 0, 0, 0, 0, 0};
    for (long p = 0; p < P; ++p) {
      long g = igp[p];
      ld sr, si;
      gpp_store1(aqsm + 2 * (n1 * G + g), aqsn + 2 * (n1 * G + g), vcoul[g],
                 wtilde + 2 * (p * G + g), &sr, &si);
      for (long ig = 0; ig < G; ++ig) {
        const double *wt = wtilde + 2 * (p * G + ig);
        const double *ie = I_eps + 2 * (p * G + ig);
        for (int iw = 0; iw < 3; ++iw) {
          ld qr, qi;
          gpp_quot(wx[n1 * wx_band_stride + iw], wt, ie, &qr, &qi);
          acc[2 * iw] += qr * sr - qi * si;
          acc[2 * iw + 1] += qr * si + qi * sr;
        }
      }
    }
    for (int k = 0; k < 6; ++k) part[6 * n1 + k] = acc[k];
  }
  ld tot[6] = {0, 0, 0, 0, 0, 0};
  for (long n1 = 0; n1 < nb; ++n1)
    for (int k = 0; k < 6; ++k) tot[k] += part[6 * n1 + k];
  for (int k = 0; k < 6; ++k) out[k] = tot[k];
  free(igp); free(part);
  return 0;
}

int orc_gpp_direct(long nb, long P, long G, const int *inv_igp_index,
                   const int *indinv, long indinv_len, const double *wx,
                   long wx_band_stride, const double *wtilde,
                   const double *aqsm, const double *aqsn,
                   const double *I_eps, const double *vcoul,
                   double *achtemp) {
  ld out[6];
  const int st = gpp_direct_ld(nb, P, G, inv_igp_index, indinv, indinv_len, wx, wx_band_stride, wtilde, aqsm,
                               aqsn, I_eps, vcoul, out);
  if (st) return st;
  for (int k = 0; k < 6; ++k) achtemp[k] = (double)out[k];
  return 0;
}

/* The same sum with long-double outputs (finite differences of the band-
 * dependent form). */
int orc_gpp_direct_ld(long nb, long P, long G, const int *inv_igp_index,
                      const int *indinv, long indinv_len, const double *wx,
                      long wx_band_stride, const double *wtilde,
                      const double *aqsm, const double *aqsn,
                      const double *I_eps, const double *vcoul, ld *out) {
  return gpp_direct_ld(nb, P, G, inv_igp_index, indinv, indinv_len, wx, wx_band_stride, wtilde, aqsm, aqsn,
                       I_eps, vcoul, out);
}

/* Screened exchange (SX, the GPP `flagOCC` branch) -- NOT in the reference,
 * so its parity is unpinned: specified here from the GPP model
 *   eps^-1_GG'(w) = delta_GG' + Omega^2 / (w^2 - wtilde^2),
 * with the Coulomb-hole weight the reference uses, Omega^2 / wtilde =
 * I_eps[p][ig] wtilde[p][igp] (sch_store1 already carries 0.5 conj(aqsm)
 * aqsn vcoul wtilde[p][igp], gpp.cpp:369-371), for the occupied bands only:
 *   asxtemp[iw] = - sum_{n1 < nvband} sum_p conj(aqsm[n1][igp]) aqsn[n1][igp]
 *                 vcoul[igp] wtilde[p][igp]
 *                 sum_ig I_eps[p][ig] wtilde[p][ig] / (wx^2 - wtilde[p][ig]^2)
 * (the delta_GG' bare-exchange part is excluded).  Product form, long double
 * complex division per term; wx[n1 * stride + iw] as in orc_gpp_direct.
 * factored != 0 (stride 0 only): X(p) = sum_n1 of the band factor first,
 * O(P G) -- the full-size form. */
static void sx_term(double wx, const double *wt, const double *ie, ld *qr, ld *qi) {
  const ld wr = wt[0], wi = wt[1];
  /* With the guard on, a pole of the product form within delta of wx
   * (wtilde = wx) or of -wx (wtilde = -wx) drops that pole's partial
   * fraction: I wtilde / (wx^2 - wtilde^2) = (I/2) (1/(wx - wtilde) -
   * 1/(wx + wtilde)). */
  const int gm = guarded((ld)wx - wr, -wi), gp = guarded((ld)wx + wr, wi);
  if (gm || gp) {
    *qr = 0.0L; *qi = 0.0L;
    if (gm && gp) return;
    const ld sgn = gm ? -0.5L : 0.5L;                       /* keep -1/(wx+wt) or +1/(wx-wt) */
    const ld dr = gm ? (ld)wx + wr : (ld)wx - wr, di = gm ? wi : -wi;
    const ld den = dr * dr + di * di;
    const ld cr = sgn * dr / den, ci = -sgn * di / den;     /* sgn / (dr + i di) */
    *qr = cr * (ld)ie[0] - ci * (ld)ie[1];
    *qi = cr * (ld)ie[1] + ci * (ld)ie[0];
    return;
  }
  const ld nr = (ld)ie[0] * wr - (ld)ie[1] * wi, ni = (ld)ie[0] * wi + (ld)ie[1] * wr;  /* I wtilde */
  const ld dr = (ld)wx * (ld)wx - (wr * wr - wi * wi), di = -2.0L * wr * wi;          /* wx^2 - wtilde^2 */
  const ld den = dr * dr + di * di;
  *qr = (nr * dr + ni * di) / den;
  *qi = (ni * dr - nr * di) / den;
}

int orc_gpp_sx(long nb, long nvband, long P, long G, const int *inv_igp_index, const int *indinv,
               long indinv_len, const double *wx, long wx_band_stride, const double *wtilde,
               const double *aqsm, const double *aqsn, const double *I_eps, const double *vcoul,
               double *asxtemp, int factored) {
  if (nb < 0 || nvband < 0 || nvband > nb || P < 0 || G <= 0 || wx_band_stride < 0) return -1;
  if (factored && wx_band_stride != 0) return -1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(P > 0 ? P : 1) * 6, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (long p = 0; p < P; ++p) {
    const long g = igp[p];
    ld acc[6] = {0, 0, 0, 0, 0, 0};
    if (factored) {
      ld xr = 0, xi = 0;  /* X(p) = sum over occupied bands of -2 sch_store1 */
      for (long n1 = 0; n1 < nvband; ++n1) {
        ld sr, si;
        gpp_store1(aqsm + 2 * (n1 * G + g), aqsn + 2 * (n1 * G + g), vcoul[g], wtilde + 2 * (p * G + g), &sr, &si);
        xr -= 2.0L * sr;
        xi -= 2.0L * si;
      }
      for (long ig = 0; ig < G; ++ig)
        for (int iw = 0; iw < 3; ++iw) {
          ld qr, qi;
          sx_term(wx[iw], wtilde + 2 * (p * G + ig), I_eps + 2 * (p * G + ig), &qr, &qi);
          acc[2 * iw] += qr * xr - qi * xi;
          acc[2 * iw + 1] += qr * xi + qi * xr;
        }
    } else {
      for (long n1 = 0; n1 < nvband; ++n1) {
        ld sr, si;
        gpp_store1(aqsm + 2 * (n1 * G + g), aqsn + 2 * (n1 * G + g), vcoul[g], wtilde + 2 * (p * G + g), &sr, &si);
        const ld xr = -2.0L * sr, xi = -2.0L * si;
        for (long ig = 0; ig < G; ++ig)
          for (int iw = 0; iw < 3; ++iw) {
            ld qr, qi;
            sx_term(wx[n1 * wx_band_stride + iw], wtilde + 2 * (p * G + ig), I_eps + 2 * (p * G + ig), &qr, &qi);
            acc[2 * iw] += qr * xr - qi * xi;
            acc[2 * iw + 1] += qr * xi + qi * xr;
          }
      }
    }
    for (int k = 0; k < 6; ++k) part[6 * p + k] = acc[k];
  }
  ld tot[6] = {0, 0, 0, 0, 0, 0};
  for (long p = 0; p < P; ++p)
    for (int k = 0; k < 6; ++k) tot[k] += part[6 * p + k];
  for (int k = 0; k < 6; ++k) asxtemp[k] = (double)tot[k];
  free(igp); free(part);
  return 0;
}

/* Factored evaluation of the same sum for a band-independent wx (the
 * reference's case): nothing inside the ig/iw loop of gpp.cpp:373-390 depends
 * on n1 except sch_store1, so
 *   achtemp[iw] = sum_p S(p) * T(p, iw),
 *   S(p) = sum_n1 sch_store1(n1, p),  T(p, iw) = sum_ig quot(p, ig, iw).
 * This is an exact algebraic identity; only rounding differs, and long double
 * keeps that far below the 1e-12 parity bar.  Cost O(P * G * 3 + nb * P), so
 * it serves as the oracle at the full benchmark sizes. */
int orc_gpp_factored(long nb, long P, long G, const int *inv_igp_index,
                     const int *indinv, long indinv_len, const double *wx,
                     const double *wtilde, const double *aqsm,
                     const double *aqsn, const double *I_eps,
                     const double *vcoul, double *achtemp) {
  if (nb < 0 || P < 0 || G <= 0) return -1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(P > 0 ? P : 1) * 6, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
#pragma omp parallel for schedule(dynamic, 4)
  for (long p = 0; p < P; ++p) {
    long g = igp[p];
    ld Sr = 0, Si = 0;
    for (long n1 = 0; n1 < nb; ++n1) {
      ld sr, si;
      gpp_store1(aqsm + 2 * (n1 * G + g), aqsn + 2 * (n1 * G + g), vcoul[g],
                 wtilde + 2 * (p * G + g), &sr, &si);
      Sr += sr; Si += si;
    }
    ld T[6] = {0, 0, 0, 0, 0, 0};
    for (long ig = 0; ig < G; ++ig) {
      const double *wt = wtilde + 2 * (p * G + ig);
      const double *ie = I_eps + 2 * (p * G + ig);
      for (int iw = 0; iw < 3; ++iw) {
        ld qr, qi;
        gpp_quot(wx[iw], wt, ie, &qr, &qi);
        T[2 * iw] += qr;
        T[2 * iw + 1] += qi;
      }
    }
    for (int iw = 0; iw < 3; ++iw) {
      part[6 * p + 2 * iw] = T[2 * iw] * Sr - T[2 * iw + 1] * Si;
      part[6 * p + 2 * iw + 1] = T[2 * iw] * Si + T[2 * iw + 1] * Sr;
    }
  }
  ld tot[6] = {0, 0, 0, 0, 0, 0};
  for (long p = 0; p < P; ++p)
    for (int k = 0; k < 6; ++k) tot[k] += part[6 * p + k];
  for (int k = 0; k < 6; ++k) achtemp[k] = (double)tot[k];
  free(igp); free(part);
  return 0;
}

/* ------------------------------------------------------------------- FF -- */

/* Last interval j (0 <= j < nFreq-1) with grid[j] < x < grid[j+1], or `init`
 * if none: the linear search of ff.cpp:107-110 (strict inequalities, the
 * last match wins). */
static int last_bracket(double x, int nFreq, const double *grid, int init) {
  int ifreq = init;
  for (int j = 0; j < nFreq - 1; ++j)
    if (x > grid[j] && x < grid[j + 1]) ifreq = j;
  return ifreq;
}

/* compute_fact of ff.cpp:103-152 with its quirks kept bit-for-bit:
 *   loop 1 (SX): a found ifreq == 0 is overwritten with nFreq-2 (:111, :121);
 *   loop 2 (COR), wx > 0: the `ifreq == -1` test can never fire (:133), and
 *     both weights carry a -0.5 factor (:135-138);
 *   loop 2, wx <= 0, occupied: search on -wx, 0 -> nFreq-2 (:146-147);
 *   loop 2, wx <= 0, unoccupied: outputs untouched (ifreq 0, facts 0).
 * *ifreq, *f1, *f2 must hold the caller's initial values (0, 0, 0 in both
 * reference callers, ff.cpp:249-250, 339-340). */
void orc_compute_fact(double wx, int nFreq, const double *g, int loop,
                      int flag_occ, int *ifreq, double *f1, double *f2) {
  if (loop == 1 && wx > 0.0) {
    int i = last_bracket(wx, nFreq, g, *ifreq);
    if (i == 0) i = nFreq - 2;
    *f1 = (g[i + 1] - wx) / (g[i + 1] - g[i]);
    *f2 = (wx - g[i]) / (g[i + 1] - g[i]);
    *ifreq = i;
  } else if (loop == 1) {
    int i = last_bracket(-wx, nFreq, g, *ifreq);
    if (i == 0) i = nFreq - 2;
    *f1 = (g[i + 1] + wx) / (g[i + 1] - g[i]);
    *f2 = (-g[i] - wx) / (g[i + 1] - g[i]);
    *ifreq = i;
  }
  if (loop == 2 && wx > 0.0) {
    int i = last_bracket(wx, nFreq, g, *ifreq);
    if (i == -1) i = nFreq - 2;
    *f1 = -0.5 * (g[i + 1] - wx) / (g[i + 1] - g[i]);
    *f2 = -0.5 * (wx - g[i]) / (g[i + 1] - g[i]);
    *ifreq = i;
  } else if (loop == 2 && flag_occ) {
    double x = -wx;
    int i = last_bracket(x, nFreq, g, 0);
    if (i == 0) i = nFreq - 2;
    *f1 = (g[i + 1] - x) / (g[i + 1] - g[i]);
    *f2 = (x - g[i]) / (g[i + 1] - g[i]);
    *ifreq = i;
  }
}

static int ff_check(long nb, long P, long G, long nFreq) {
  return (nb < 0 || P < 0 || G <= 0 || P > G || nFreq < 2) ? -1 : 0;
}

/* achsDtemp_Kernel, ff.cpp:171-209:
 *   achsDtemp = sum_{n1<nb, p} 0.5 vcoul[igp] *
 *               ( - sum_ig aqsn[n1][ig] conj(aqsm[n1][igp]) I_epsR[1][p][ig] )
 * conj(aqsm[n1][igp]) does not depend on ig and is factored out of the ig sum
 * (exact algebra).  out = 1 complex (2 doubles). */
int orc_ff_achs(long nb, long P, long G, long nFreq, const int *inv_igp_index,
                const int *indinv, long indinv_len, const double *aqsn,
                const double *aqsm, const double *I_epsR, const double *vcoul,
                double *out) {
  if (ff_check(nb, P, G, nFreq)) return -1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(nb > 0 ? nb : 1) * 2, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
  const double *R1 = I_epsR + 2 * (1 * P * G);
#pragma omp parallel for schedule(dynamic, 1)
  for (long n1 = 0; n1 < nb; ++n1) {
    ld accr = 0, acci = 0;
    const double *a = aqsn + 2 * n1 * G;
    for (long p = 0; p < P; ++p) {
      const double *r = R1 + 2 * p * G;
      ld cr = 0, ci = 0;
      for (long ig = 0; ig < G; ++ig) {
        ld ar = a[2 * ig], ai = a[2 * ig + 1];
        ld br = r[2 * ig], bi = r[2 * ig + 1];
        cr += ar * br - ai * bi;
        ci += ar * bi + ai * br;
      }
      long g = igp[p];
      ld mr = aqsm[2 * (n1 * G + g)], mi = -(ld)aqsm[2 * (n1 * G + g) + 1];
      ld sr = cr * mr - ci * mi, si = cr * mi + ci * mr;
      ld v = (ld)vcoul[g] * 0.5L;
      accr += -sr * v;
      acci += -si * v;
    }
    part[2 * n1] = accr;
    part[2 * n1 + 1] = acci;
  }
  ld tr = 0, ti = 0;
  for (long n1 = 0; n1 < nb; ++n1) { tr += part[2 * n1]; ti += part[2 * n1 + 1]; }
  out[0] = (double)tr;
  out[1] = (double)ti;
  free(igp); free(part);
  return 0;
}

/* sum_{p, ig} aqsn[n1][ig] * W(n1, p) * (X[i][p][ig] * c1 + X[i+1][p][ig] * c2)
 * with W(n1, p) = conj(aqsm[n1][igp]) * vcoul[igp] and X = R - A (sub = 1)
 * or X = E (sub = 0, B ignored).  Shared by the SX and COR restatements. */
static void ff_band_sum(long n1, long P, long G, const long *igp,
                        const double *aqsn, const double *aqsm,
                        const double *vcoul, const double *E,
                        const double *B, int sub, int i, ld c1, ld c2,
                        ld *out_r, ld *out_i) {
  const double *a = aqsn + 2 * n1 * G;
  ld accr = 0, acci = 0;
  for (long p = 0; p < P; ++p) {
    const double *x0 = E + 2 * (((long)i * P + p) * G);
    const double *x1 = E + 2 * (((long)(i + 1) * P + p) * G);
    const double *y0 = sub ? B + 2 * (((long)i * P + p) * G) : NULL;
    const double *y1 = sub ? B + 2 * (((long)(i + 1) * P + p) * G) : NULL;
    ld cr = 0, ci = 0;
    for (long ig = 0; ig < G; ++ig) {
      ld u0r = x0[2 * ig], u0i = x0[2 * ig + 1];
      ld u1r = x1[2 * ig], u1i = x1[2 * ig + 1];
      if (sub) {
        u0r -= y0[2 * ig]; u0i -= y0[2 * ig + 1];
        u1r -= y1[2 * ig]; u1i -= y1[2 * ig + 1];
      }
      ld xr = u0r * c1 + u1r * c2, xi = u0i * c1 + u1i * c2;
      ld ar = a[2 * ig], ai = a[2 * ig + 1];
      cr += ar * xr - ai * xi;
      ci += ar * xi + ai * xr;
    }
    long g = igp[p];
    ld mr = aqsm[2 * (n1 * G + g)], mi = -(ld)aqsm[2 * (n1 * G + g) + 1];
    ld v = vcoul[g];
    mr *= v; mi *= v;
    accr += cr * mr - ci * mi;
    acci += cr * mi + ci * mr;
  }
  *out_r = accr;
  *out_i = acci;
}

/* The frequency argument of band n1 at evaluation point iw.  The reference
 * uses wx = freqevalmin - ekq[n1] + freqevalstep for every iw (no iw term,
 * ff.cpp:245, 337); per_iw selects wx = freqevalmin - ekq[n1] +
 * iw * freqevalstep instead (a distinct value per iw; the reference's value is
 * the one at iw = 1). */
static double ff_wx(double freqevalmin, double freqevalstep, double ekq, long iw, int per_iw) {
  return per_iw ? freqevalmin - ekq + (double)iw * freqevalstep : freqevalmin - ekq + freqevalstep;
}

/* asxDtemp_Kernel + ssxDittt_kernel, ff.cpp:154-169, 211-293.  For n1 <
 * nvband: wx (ff_wx), compute_fact(loop 1), X = I_epsR if wx > 0 else
 * I_epsA (:254-261), times occ.  Without per_iw every asxDtemp[iw] receives
 * the same sum; out has nfreqeval complex values. */
static int ff_asx(long nvband, long nfreqeval, long G, long P, long nFreq,
                  double freqevalmin, double freqevalstep, double occ,
                  const double *ekq, const double *dFreqGrid,
                  const int *inv_igp_index, const int *indinv, long indinv_len,
                  const double *aqsm, const double *aqsn, const double *vcoul,
                  const double *I_epsR, const double *I_epsA, double *out, int per_iw) {
  if (ff_check(nvband, P, G, nFreq) || nfreqeval < 0) return -1;
  const long ne = per_iw ? nfreqeval : 1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(nvband > 0 ? nvband : 1) * (size_t)(ne > 0 ? ne : 1) * 2, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (long n1 = 0; n1 < nvband; ++n1)
    for (long e = 0; e < ne; ++e) {
      double wx = ff_wx(freqevalmin, freqevalstep, ekq[n1], e, per_iw);
      int ifreq = 0;
      double f1 = 0, f2 = 0;
      orc_compute_fact(wx, (int)nFreq, dFreqGrid, 1, 0, &ifreq, &f1, &f2);
      ld r, i;
      ff_band_sum(n1, P, G, igp, aqsn, aqsm, vcoul, wx > 0 ? I_epsR : I_epsA,
                  NULL, 0, ifreq, f1, f2, &r, &i);
      part[2 * (n1 * ne + e)] = r * (ld)occ;
      part[2 * (n1 * ne + e) + 1] = i * (ld)occ;
    }
  for (long iw = 0; iw < nfreqeval; ++iw) {
    const long e = per_iw ? iw : 0;
    ld tr = 0, ti = 0;
    for (long n1 = 0; n1 < nvband; ++n1) { tr += part[2 * (n1 * ne + e)]; ti += part[2 * (n1 * ne + e) + 1]; }
    out[2 * iw] = (double)tr;
    out[2 * iw + 1] = (double)ti;
  }
  free(igp); free(part);
  return 0;
}

int orc_ff_asx(long nvband, long nfreqeval, long G, long P, long nFreq,
               double freqevalmin, double freqevalstep, double occ,
               const double *ekq, const double *dFreqGrid,
               const int *inv_igp_index, const int *indinv, long indinv_len,
               const double *aqsm, const double *aqsn, const double *vcoul,
               const double *I_epsR, const double *I_epsA, double *out) {
  return ff_asx(nvband, nfreqeval, G, P, nFreq, freqevalmin, freqevalstep, occ, ekq, dFreqGrid, inv_igp_index,
                indinv, indinv_len, aqsm, aqsn, vcoul, I_epsR, I_epsA, out, 0);
}

/* asxDtemp with wx = freqevalmin - ekq + iw * freqevalstep per iw. */
int orc_ff_asx_iw(long nvband, long nfreqeval, long G, long P, long nFreq,
                  double freqevalmin, double freqevalstep, double occ,
                  const double *ekq, const double *dFreqGrid,
                  const int *inv_igp_index, const int *indinv, long indinv_len,
                  const double *aqsm, const double *aqsn, const double *vcoul,
                  const double *I_epsR, const double *I_epsA, double *out) {
  return ff_asx(nvband, nfreqeval, G, P, nFreq, freqevalmin, freqevalstep, occ, ekq, dFreqGrid, inv_igp_index,
                indinv, indinv_len, aqsm, aqsn, vcoul, I_epsR, I_epsA, out, 1);
}

/* achDtemp_cor_Kernel + schDttt_corKernel1/2, ff.cpp:295-451.  For every
 * band: flag_occ = n1 < nvband (the intended per-iteration value; the
 * reference shares the variable across OpenMP threads, :310), wx (ff_wx),
 * compute_fact(loop 2).  wx > 0 and unoccupied -> Kernel1 with (f1, f2);
 * wx <= 0 and occupied -> Kernel2 with an extra -0.5 (:437-444); otherwise
 * nothing.  X = I_epsR - I_epsA.  Without per_iw every achDtemp_cor[iw]
 * receives the same sum. */
static int ff_cor(long nb, long nvband, long nfreqeval, long G, long P,
                  long nFreq, double freqevalmin, double freqevalstep,
                  const double *ekq, const double *dFreqGrid,
                  const int *inv_igp_index, const int *indinv, long indinv_len,
                  const double *aqsm, const double *aqsn, const double *vcoul,
                  const double *I_epsR, const double *I_epsA, double *out, int per_iw) {
  if (ff_check(nb, P, G, nFreq) || nfreqeval < 0 || nvband < 0) return -1;
  const long ne = per_iw ? nfreqeval : 1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(nb > 0 ? nb : 1) * (size_t)(ne > 0 ? ne : 1) * 2, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (long n1 = 0; n1 < nb; ++n1)
    for (long e = 0; e < ne; ++e) {
      int occ = n1 < nvband;
      double wx = ff_wx(freqevalmin, freqevalstep, ekq[n1], e, per_iw);
      int ifreq = 0;
      double f1 = 0, f2 = 0;
      orc_compute_fact(wx, (int)nFreq, dFreqGrid, 2, occ, &ifreq, &f1, &f2);
      ld r = 0, i = 0;
      if (wx > 0) {
        if (!occ)
          ff_band_sum(n1, P, G, igp, aqsn, aqsm, vcoul, I_epsR, I_epsA, 1,
                      ifreq, f1, f2, &r, &i);
      } else if (occ) {
        ff_band_sum(n1, P, G, igp, aqsn, aqsm, vcoul, I_epsR, I_epsA, 1, ifreq,
                    -0.5L * f1, -0.5L * f2, &r, &i);
      }
      part[2 * (n1 * ne + e)] = r;
      part[2 * (n1 * ne + e) + 1] = i;
    }
  for (long iw = 0; iw < nfreqeval; ++iw) {
    const long e = per_iw ? iw : 0;
    ld tr = 0, ti = 0;
    for (long n1 = 0; n1 < nb; ++n1) { tr += part[2 * (n1 * ne + e)]; ti += part[2 * (n1 * ne + e) + 1]; }
    out[2 * iw] = (double)tr;
    out[2 * iw + 1] = (double)ti;
  }
  free(igp); free(part);
  return 0;
}

int orc_ff_cor(long nb, long nvband, long nfreqeval, long G, long P,
               long nFreq, double freqevalmin, double freqevalstep,
               const double *ekq, const double *dFreqGrid,
               const int *inv_igp_index, const int *indinv, long indinv_len,
               const double *aqsm, const double *aqsn, const double *vcoul,
               const double *I_epsR, const double *I_epsA, double *out) {
  return ff_cor(nb, nvband, nfreqeval, G, P, nFreq, freqevalmin, freqevalstep, ekq, dFreqGrid, inv_igp_index,
                indinv, indinv_len, aqsm, aqsn, vcoul, I_epsR, I_epsA, out, 0);
}

/* achDtemp_cor with wx = freqevalmin - ekq + iw * freqevalstep per iw. */
int orc_ff_cor_iw(long nb, long nvband, long nfreqeval, long G, long P,
                  long nFreq, double freqevalmin, double freqevalstep,
                  const double *ekq, const double *dFreqGrid,
                  const int *inv_igp_index, const int *indinv, long indinv_len,
                  const double *aqsm, const double *aqsn, const double *vcoul,
                  const double *I_epsR, const double *I_epsA, double *out) {
  return ff_cor(nb, nvband, nfreqeval, G, P, nFreq, freqevalmin, freqevalstep, ekq, dFreqGrid, inv_igp_index,
                indinv, indinv_len, aqsm, aqsn, vcoul, I_epsR, I_epsA, out, 1);
}

/* ------------------------------------------------------------ GPP adjoint --
 * Long-double reference gradient of the GPP sum for a band-independent wx.
 * With q = 1/(wx - wtilde) (= conj(wdiff)/|wdiff|^2, gpp.cpp:374-378) the
 * sum is holomorphic in wtilde and I_eps; for cotangents G_iw (gcot: 3
 * complex) the complex gradient of L = sum_iw Re(conj(G_iw) Sigma_iw) is
 * sum_iw G_iw conj(dSigma_iw/dz), with
 *   dSigma/dI_eps[p][ig]  = S(p) q,   dSigma/dwtilde[p][ig] = S(p) I_eps q^2,
 *   plus C(p) T(p) at ig = igp(p) (wtilde[p][igp] inside sch_store1),
 *   dSigma_iw/dwx = - sum S(p) I_eps q^2.
 * grad_wt / grad_ie: [P][G] complex or NULL; domega: 3 complex or NULL. */
int orc_gpp_backward(long nb, long P, long G, const int *inv_igp_index,
                     const int *indinv, long indinv_len, const double *wx,
                     const double *wtilde, const double *aqsm,
                     const double *aqsn, const double *I_eps,
                     const double *vcoul, const double *gcot,
                     double *grad_wt, double *grad_ie, double *domega) {
  if (nb < 0 || P < 0 || G <= 0) return -1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(P > 0 ? P : 1) * 6, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
  /* conj(G_iw) */
  ld cgr[3], cgi[3];
  for (int iw = 0; iw < 3; ++iw) { cgr[iw] = gcot[2 * iw]; cgi[iw] = -(ld)gcot[2 * iw + 1]; }
#pragma omp parallel for schedule(dynamic, 4)
  for (long p = 0; p < P; ++p) {
    long g = igp[p];
    ld Cr = 0, Ci = 0;
    for (long n1 = 0; n1 < nb; ++n1) {
      ld ar = aqsm[2 * (n1 * G + g)], ai = -(ld)aqsm[2 * (n1 * G + g) + 1];
      ld br = aqsn[2 * (n1 * G + g)], bi = aqsn[2 * (n1 * G + g) + 1];
      ld v = 0.5L * (ld)vcoul[g];
      Cr += (ar * br - ai * bi) * v;
      Ci += (ar * bi + ai * br) * v;
    }
    ld wgr = wtilde[2 * (p * G + g)], wgi = wtilde[2 * (p * G + g) + 1];
    ld Sr = Cr * wgr - Ci * wgi, Si = Cr * wgi + Ci * wgr;
    ld Tr[3] = {0, 0, 0}, Ti[3] = {0, 0, 0}, Ur[3] = {0, 0, 0}, Ui[3] = {0, 0, 0};
    for (long ig = 0; ig < G; ++ig) {
      ld wr = wtilde[2 * (p * G + ig)], wi = wtilde[2 * (p * G + ig) + 1];
      ld er = I_eps[2 * (p * G + ig)], ei = I_eps[2 * (p * G + ig) + 1];
      ld hIr = 0, hIi = 0, hWr = 0, hWi = 0;
      for (int iw = 0; iw < 3; ++iw) {
        ld dr = (ld)wx[iw] - wr, di = -wi;          /* d = wx - w        */
        ld den = dr * dr + di * di;
        ld qr = dr / den, qi = -di / den;           /* q = 1/d           */
        ld iqr = er * qr - ei * qi, iqi = er * qi + ei * qr;       /* I q   */
        ld q2r = iqr * qr - iqi * qi, q2i = iqr * qi + iqi * qr;   /* I q^2 */
        Tr[iw] += iqr; Ti[iw] += iqi;
        Ur[iw] += q2r; Ui[iw] += q2i;
        hIr += cgr[iw] * qr - cgi[iw] * qi;  hIi += cgr[iw] * qi + cgi[iw] * qr;
        hWr += cgr[iw] * q2r - cgi[iw] * q2i; hWi += cgr[iw] * q2i + cgi[iw] * q2r;
      }
      if (grad_ie) {  /* conj(S hI) */
        grad_ie[2 * (p * G + ig)] = (double)(Sr * hIr - Si * hIi);
        grad_ie[2 * (p * G + ig) + 1] = (double)(-(Sr * hIi + Si * hIr));
      }
      if (grad_wt) {  /* the (p, igp) entry is redone below with both terms */
        ld xr = Sr * hWr - Si * hWi, xi = Sr * hWi + Si * hWr;
        grad_wt[2 * (p * G + ig)] = (double)xr;
        grad_wt[2 * (p * G + ig) + 1] = (double)(-xi);
      }
    }
    if (grad_wt) {
      /* recompute the (p, igp) entry in long double with both terms */
      ld wr = wgr, wi = wgi;
      ld er = I_eps[2 * (p * G + g)], ei = I_eps[2 * (p * G + g) + 1];
      ld hWr = 0, hWi = 0, hCr = 0, hCi = 0;
      for (int iw = 0; iw < 3; ++iw) {
        ld dr = (ld)wx[iw] - wr, di = -wi;
        ld den = dr * dr + di * di;
        ld qr = dr / den, qi = -di / den;
        ld iqr = er * qr - ei * qi, iqi = er * qi + ei * qr;
        ld q2r = iqr * qr - iqi * qi, q2i = iqr * qi + iqi * qr;
        hWr += cgr[iw] * q2r - cgi[iw] * q2i; hWi += cgr[iw] * q2i + cgi[iw] * q2r;
        hCr += cgr[iw] * Tr[iw] - cgi[iw] * Ti[iw]; hCi += cgr[iw] * Ti[iw] + cgi[iw] * Tr[iw];
      }
      ld xr = (Sr * hWr - Si * hWi) + (Cr * hCr - Ci * hCi);
      ld xi = (Sr * hWi + Si * hWr) + (Cr * hCi + Ci * hCr);
      grad_wt[2 * (p * G + g)] = (double)xr;
      grad_wt[2 * (p * G + g) + 1] = (double)(-xi);
    }
    for (int iw = 0; iw < 3; ++iw) {
      part[6 * p + 2 * iw] = -(Sr * Ur[iw] - Si * Ui[iw]);
      part[6 * p + 2 * iw + 1] = -(Sr * Ui[iw] + Si * Ur[iw]);
    }
  }
  if (domega) {
    ld tot[6] = {0, 0, 0, 0, 0, 0};
    for (long p = 0; p < P; ++p)
      for (int k = 0; k < 6; ++k) tot[k] += part[6 * p + k];
    for (int k = 0; k < 6; ++k) domega[k] = (double)tot[k];
  }
  free(igp); free(part);
  return 0;
}

/* Band-loop form of the same gradient for a band-dependent wx
 * (wx[n1 * wx_band_stride + iw]; stride 0 is the reference's shared triple):
 * nothing is factored over bands.  With s(n1, p) = C(n1, p) wtilde[p][igp],
 * C(n1, p) = conj(aqsm[n1][igp]) aqsn[n1][igp] 0.5 vcoul[igp] and
 * q = 1 / (wx[n1][iw] - wtilde[p][ig]):
 *   dSigma_iw/dI_eps[p][ig]  = A_iw = sum_n1 s q
 *   dSigma_iw/dwtilde[p][ig] = I_eps B_iw,  B_iw = sum_n1 s q^2
 *                              (+ D_iw(p) = sum_ig I_eps sum_n1 C q at ig = igp)
 *   dSigma_iw/domega         = - sum_{p, ig} I_eps B_iw
 * and the gradients follow as in orc_gpp_backward.  Cost O(nb P G 3):
 * small sizes only. */
int orc_gpp_backward_direct(long nb, long P, long G, const int *inv_igp_index,
                            const int *indinv, long indinv_len, const double *wx,
                            long wx_band_stride, const double *wtilde,
                            const double *aqsm, const double *aqsn,
                            const double *I_eps, const double *vcoul,
                            const double *gcot, double *grad_wt, double *grad_ie,
                            double *domega) {
  if (nb < 0 || P < 0 || G <= 0 || wx_band_stride < 0) return -1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(P > 0 ? P : 1) * 6, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
  ld cgr[3], cgi[3];
  for (int iw = 0; iw < 3; ++iw) { cgr[iw] = gcot[2 * iw]; cgi[iw] = -(ld)gcot[2 * iw + 1]; }
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1)
  for (long p = 0; p < P; ++p) {
    const long g = igp[p];
    ld *C = (ld *)malloc(sizeof(ld) * 2 * (size_t)(nb > 0 ? nb : 1));
    if (!C) { bad = 1; continue; }
    for (long n1 = 0; n1 < nb; ++n1) {
      ld ar = aqsm[2 * (n1 * G + g)], ai = -(ld)aqsm[2 * (n1 * G + g) + 1];
      ld br = aqsn[2 * (n1 * G + g)], bi = aqsn[2 * (n1 * G + g) + 1];
      ld v = 0.5L * (ld)vcoul[g];
      C[2 * n1] = (ar * br - ai * bi) * v;
      C[2 * n1 + 1] = (ar * bi + ai * br) * v;
    }
    const ld wgr = wtilde[2 * (p * G + g)], wgi = wtilde[2 * (p * G + g) + 1];
    ld Dr[3] = {0, 0, 0}, Di[3] = {0, 0, 0}, Wr[3] = {0, 0, 0}, Wi[3] = {0, 0, 0};
    ld diag_r = 0, diag_i = 0;  /* conj-free value of the (p, igp) entry */
    for (long ig = 0; ig < G; ++ig) {
      const ld wr = wtilde[2 * (p * G + ig)], wi = wtilde[2 * (p * G + ig) + 1];
      const ld er = I_eps[2 * (p * G + ig)], ei = I_eps[2 * (p * G + ig) + 1];
      ld hIr = 0, hIi = 0, hWr = 0, hWi = 0;
      for (int iw = 0; iw < 3; ++iw) {
        ld Apr = 0, Api = 0, Bpr = 0, Bpi = 0;  /* sum_n1 C q, sum_n1 C q^2 */
        for (long n1 = 0; n1 < nb; ++n1) {
          const ld dr = (ld)wx[n1 * wx_band_stride + iw] - wr, di = -wi;
          const ld den = dr * dr + di * di;
          const ld qr = dr / den, qi = -di / den;
          const ld q2r = qr * qr - qi * qi, q2i = 2.0L * qr * qi;
          const ld cr = C[2 * n1], ci = C[2 * n1 + 1];
          Apr += cr * qr - ci * qi;  Api += cr * qi + ci * qr;
          Bpr += cr * q2r - ci * q2i; Bpi += cr * q2i + ci * q2r;
        }
        /* A = wtilde[p][igp] A', I B = I wtilde[p][igp] B' */
        const ld Ar = wgr * Apr - wgi * Api, Ai = wgr * Api + wgi * Apr;
        const ld Br = wgr * Bpr - wgi * Bpi, Bi = wgr * Bpi + wgi * Bpr;
        const ld ibr = er * Br - ei * Bi, ibi = er * Bi + ei * Br;
        Dr[iw] += er * Apr - ei * Api;  Di[iw] += er * Api + ei * Apr;
        Wr[iw] += ibr; Wi[iw] += ibi;
        hIr += cgr[iw] * Ar - cgi[iw] * Ai;   hIi += cgr[iw] * Ai + cgi[iw] * Ar;
        hWr += cgr[iw] * ibr - cgi[iw] * ibi; hWi += cgr[iw] * ibi + cgi[iw] * ibr;
      }
      if (grad_ie) {
        grad_ie[2 * (p * G + ig)] = (double)hIr;
        grad_ie[2 * (p * G + ig) + 1] = (double)(-hIi);
      }
      if (grad_wt) {
        grad_wt[2 * (p * G + ig)] = (double)hWr;
        grad_wt[2 * (p * G + ig) + 1] = (double)(-hWi);
      }
      if (ig == g) { diag_r = hWr; diag_i = hWi; }
    }
    if (grad_wt) {
      for (int iw = 0; iw < 3; ++iw) {
        diag_r += cgr[iw] * Dr[iw] - cgi[iw] * Di[iw];
        diag_i += cgr[iw] * Di[iw] + cgi[iw] * Dr[iw];
      }
      grad_wt[2 * (p * G + g)] = (double)diag_r;
      grad_wt[2 * (p * G + g) + 1] = (double)(-diag_i);
    }
    for (int iw = 0; iw < 3; ++iw) {
      part[6 * p + 2 * iw] = -Wr[iw];
      part[6 * p + 2 * iw + 1] = -Wi[iw];
    }
    free(C);
  }
  if (!bad && domega) {
    ld tot[6] = {0, 0, 0, 0, 0, 0};
    for (long p = 0; p < P; ++p)
      for (int k = 0; k < 6; ++k) tot[k] += part[6 * p + k];
    for (int k = 0; k < 6; ++k) domega[k] = (double)tot[k];
  }
  free(igp); free(part);
  return bad ? -1 : 0;
}

/* orc_gpp_factored with long-double outputs (6 values), for finite
 * differences whose step is far below double resolution of the sum. */
int orc_gpp_factored_ld(long nb, long P, long G, const int *inv_igp_index,
                        const int *indinv, long indinv_len, const double *wx,
                        const double *wtilde, const double *aqsm,
                        const double *aqsn, const double *I_eps,
                        const double *vcoul, long double *achtemp) {
  if (nb < 0 || P < 0 || G <= 0) return -1;
  long *igp = (long *)malloc(sizeof(long) * (size_t)(P > 0 ? P : 1));
  ld *part = (ld *)calloc((size_t)(P > 0 ? P : 1) * 6, sizeof(ld));
  if (!igp || !part) { free(igp); free(part); return -1; }
  if (resolve_igp(P, G, inv_igp_index, indinv, indinv_len, igp)) {
    free(igp); free(part); return -1;
  }
#pragma omp parallel for schedule(dynamic, 4)
  for (long p = 0; p < P; ++p) {
    long g = igp[p];
    ld Sr = 0, Si = 0;
    for (long n1 = 0; n1 < nb; ++n1) {
      ld sr, si;
      gpp_store1(aqsm + 2 * (n1 * G + g), aqsn + 2 * (n1 * G + g), vcoul[g],
                 wtilde + 2 * (p * G + g), &sr, &si);
      Sr += sr; Si += si;
    }
    ld T[6] = {0, 0, 0, 0, 0, 0};
    for (long ig = 0; ig < G; ++ig) {
      for (int iw = 0; iw < 3; ++iw) {
        ld qr, qi;
        gpp_quot(wx[iw], wtilde + 2 * (p * G + ig), I_eps + 2 * (p * G + ig), &qr, &qi);
        T[2 * iw] += qr;
        T[2 * iw + 1] += qi;
      }
    }
    for (int iw = 0; iw < 3; ++iw) {
      part[6 * p + 2 * iw] = T[2 * iw] * Sr - T[2 * iw + 1] * Si;
      part[6 * p + 2 * iw + 1] = T[2 * iw] * Si + T[2 * iw + 1] * Sr;
    }
  }
  for (int k = 0; k < 6; ++k) achtemp[k] = 0;
  for (long p = 0; p < P; ++p)
    for (int k = 0; k < 6; ++k) achtemp[k] += part[6 * p + k];
  free(igp); free(part);
  return 0;
}
