// ff_plan.cuh -- host-side plan of the FF contractions (ff.cu).
#pragma once

#include <vector>

#include "bgw_internal.cuh"

namespace bgw {

enum { SRC_R = 0, SRC_A = 1, SRC_RA = 2 };
enum { OUT_ACHS = 0, OUT_ASX = 1, OUT_COR = 2, OUT_COUNT = 3 };

struct FFRow {
  int32_t band;
  int32_t pad;
  double coef;
};

// With per-iw outputs a group holds each band once (coef 1) and the terms
// carry the coefficients: output `out` += coef * (row's contraction).
struct FFTerm {
  int32_t row, out;
  double coef;
};

// Output index of (sum, slot): 0 = achsDtemp, 1 + iw = asxDtemp[iw],
// 1 + nE + iw = achDtemp_cor[iw].
inline int ff_out_index(int out, int slot, int64_t nE) {
  return out == OUT_ACHS ? 0 : out == OUT_ASX ? 1 + slot : 1 + (int)nE + slot;
}

struct FFTile {
  int32_t src, f, row_begin, row_count;
  int32_t p_begin, k_begin, k_count, out;
};

// One band group: rows [row_begin, row_begin + row_count) of FFPlan::rows,
// all contracted with the same slice f of source `src`, summed into `out`.
struct FFGroup {
  int32_t out, src, f, row_begin, row_count;
};

struct FFPlan {
  std::vector<FFGroup> groups;
  std::vector<FFRow> rows;
  std::vector<FFTile> tiles;
  int seg[OUT_COUNT + 1] = {0, 0, 0, 0};  // tile range of each output
  double useful_cmacs = 0.0;               // sum over groups rows * P * G
  // Frequency slices read from I_epsR / I_epsA: [lo, hi] (lo > hi: none).
  int r_lo = 1 << 30, r_hi = -1, a_lo = 1 << 30, a_hi = -1;
  std::vector<double> slice_reads;  // distinct [ngpown][ncouls] slices read
  // wx = freqevalmin - ekq + iw * freqevalstep per evaluation point:
  // distinct outputs per iw, rows deduplicated per group, coefficients in
  // `terms` (sorted by output).  Otherwise the reference's single wx and
  // every iw output gets the same value.
  bool per_iw = false;
  std::vector<FFTerm> terms;
};

// Host CSR tables of the per-iw finalize: the partials of each plan row and
// the terms of each output.
struct FFTermTables {
  std::vector<int> row_ptr, part_idx, out_ptr, term_row;
  std::vector<double> term_coef;
};
// row_of[i] = plan row of partial i (-1: none).
void ff_build_term_tables(const FFPlan &plan, const std::vector<int> &row_of, int64_t nE, FFTermTables *tt);
// Uploads the tables into workspace slot `slot` and enqueues the finalize:
// output o = sum over its terms (in order) of coef * (sum of the row's
// partials, in order); writes achs, asx[nE], cor[nE] (null skipped).
int ff_launch_term_finalize(CallEnv *env, int slot, const FFTermTables &tt, const double *partials, int64_t nE,
                            double *achs, double *asx, double *cor);

// Builds the plan of the requested sums from host copies of ekq[0..nb) and
// dFreqGrid; sizes the k split for the device.
int ff_make_plan(CallEnv *env, int64_t nb, int64_t nvband, int64_t P, int64_t G, int64_t nFreq, double fmin,
                 double fstep, double occ, const double *ekq_h, const double *grid_h, bool want_achs,
                 bool want_asx, bool want_cor, bool per_iw, int64_t nE, FFPlan *plan);

// Builds W[n1][p] = conj(aqsm[n1][igp]) vcoul[igp] for n1 < nb_w on `stream`.
int ff_build_w(CallEnv *env, int64_t nb_w, int64_t G, int64_t P, const int32_t *inv, const int32_t *indinv,
               int64_t indinv_len, const double2 *am, const double *vc, double2 **W_out);
// FP64 (DMMA) tiles of the given groups, appended to `tiles` (k split sized
// for `target_ctas` together with `base_tiles` tiles already planned).
void ff_fp64_tiles(const std::vector<FFGroup> &groups, int64_t P, int64_t G, int target_ctas,
                   std::vector<FFTile> *tiles);
// Launches the DMMA contraction over device tiles: one complex partial per
// tile at `partials`, or with `per_row` one per tile row (ntiles x
// ff_fp64_tile_rows(), zero for padding rows).
// n_rows: rows of the plan; nb: rows of aqsn and W (both bound the debug
// build's checks, which report through `status`).  gate (optional, one
// entry per tile): -1 runs the tile; u >= 0 runs it only if unit_flag[u] is
// nonzero, and writes a zero partial otherwise.
int ff_launch_fp64_tiles(cudaStream_t stream, const FFTile *d_tiles, int ntiles, const FFRow *d_rows, int n_rows,
                         int64_t nb, int64_t P, int64_t G, const double2 *an, const double2 *R, int r_f0,
                         const double2 *A, int a_f0, const double2 *W, double *partials, int *status,
                         bool per_row = false, const int *gate = nullptr, const int *unit_flag = nullptr);
int ff_fp64_tile_rows();
int ff_fp64_tile_cols();
// Sums each partial into its output (out_of[i]: 0 achs, 1 asx, 2 cor) in
// index order; writes achs, asx[nE] and cor[nE] (null skipped).  One block.
int ff_enqueue_out_finalize(cudaStream_t stream, const double *partials, const int *out_of, int n, int nE,
                            double *achs, double *asx, double *cor);
// Plan row of every per-row partial of `tiles` (-1 for padding rows),
// appended to `row_of`.
void ff_fp64_row_ids(const std::vector<FFTile> &tiles, std::vector<int> *row_of);
int ff_fp64_per_sm(int *per_sm);
// Mixed precision (integer slices on tcgen05) evaluation of a plan.
int ff_launch_mixed(CallEnv *env, const FFPlan &plan, int64_t nb, int64_t nb_w, int64_t nE, int64_t G, int64_t P,
                    const int32_t *inv, const int32_t *indinv, int64_t indinv_len, const double2 *am,
                    const double2 *an, const double *vc, const double2 *R, int r_f0, const double2 *A, int a_f0,
                    double *achs_dev, double *asx_dev, double *cor_dev);

// Mixed precision with the fused kernel (ff_fused.cu): the FP64 slices are
// cut into integer digits inside the tensor-core kernel.  Groups of fewer
// than `min_rows` rows stay on the FP64 kernel.
int ff_launch_fused(CallEnv *env, const FFPlan &plan, int64_t nb_w, int64_t nE, int64_t G, int64_t P,
                    const int32_t *inv,
                    const int32_t *indinv, int64_t indinv_len, const double2 *am, const double2 *an,
                    const double *vc, const double2 *R, int r_f0, const double2 *A, int a_f0, int min_rows,
                    double *achs_dev, double *asx_dev, double *cor_dev);

// Enqueues a planned FF evaluation.  Device pointers; R / A point at
// frequency slice r_f0 / a_f0.  Outputs are device pointers (nullptr skips).
int ff_launch(CallEnv *env, const FFPlan &plan, int64_t nb_w, int64_t nE, int64_t G, int64_t P,
              const int32_t *inv, const int32_t *indinv, int64_t indinv_len, const double2 *am, const double2 *an,
              const double *vc, const double2 *R, int r_f0, const double2 *A, int a_f0, double *achs_dev,
              double *asx_dev, double *cor_dev);

}  // namespace bgw
