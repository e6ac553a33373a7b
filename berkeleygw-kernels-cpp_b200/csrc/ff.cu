// ff.cu -- full-frequency self-energy sums (FF/ff.cpp:103-451) on sm_100a.
//
// All three FF sums are weighted complex contractions over (band, G', G):
//   sum_{rows r} coef(r) sum_p W(band(r), p) C(r, p),
//   C(r, p)  = sum_ig aqsn[band(r)][ig] * X_f[p][ig],
//   W(n1, p) = conj(aqsm[n1][igp(p)]) * vcoul[igp(p)],
// with X_f one frequency slice of I_epsR (achsDtemp, and asxDtemp when
// wx > 0), of I_epsA (asxDtemp when wx <= 0) or of I_epsR - I_epsA
// (achDtemp_cor).  The reference evaluates (f1 X_i + f2 X_{i+1}) per band
// (ff.cpp:161-164, 396-403, 432-437); by linearity this equals f1 C_i + f2
// C_{i+1}, so a band contributes one row with coefficient f1 to the group of
// slice i and one with f2 to the group of slice i+1.  Grouping bands by slice
// turns every sum into a dense complex GEMM per group (rows x G' x G), which
// runs on the FP64 tensor cores (mma.sync m8n8k4 f64, the only FP64 MMA on
// sm_100a) with a fused epilogue that applies W and coef and reduces to one
// complex partial per tile.  The reference's iw loop recomputes an
// iw-independent value (wx has no iw term, ff.cpp:245, 337); it is computed
// once and written to every iw.
//
// Reductions are deterministic: per-tile partials in a fixed slot, summed in
// tile order by one block.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "bgw_internal.cuh"
#include "ff_plan.cuh"
#include "reduce.cuh"

namespace bgw {

// --------------------------------------------------------------- planning --

// compute_fact (FF/ff.cpp:103-152), quirks included: loop 1 maps a found
// ifreq == 0 to nFreq - 2; loop 2 with wx > 0 keeps ifreq == 0 (its `== -1`
// test never fires) and scales both weights by -0.5; loop 2 with wx <= 0 and
// an occupied band searches -wx and maps 0 to nFreq - 2; otherwise the
// outputs keep their initial values (0, 0, 0).
struct Fact {
  int ifreq = 0;
  double f1 = 0.0, f2 = 0.0;
};

static int bracket_last(double x, int nFreq, const double *g, int init) {
  int r = init;
  for (int j = 0; j + 1 < nFreq; ++j)
    if (x > g[j] && x < g[j + 1]) r = j;
  return r;
}

Fact compute_fact_host(double wx, int nFreq, const double *g, int loop, bool flag_occ) {
  Fact o;
  if (loop == 1) {
    const double x = wx > 0.0 ? wx : -wx;
    int i = bracket_last(x, nFreq, g, 0);
    if (i == 0) i = nFreq - 2;
    const double span = g[i + 1] - g[i];
    if (wx > 0.0) {
      o.f1 = (g[i + 1] - wx) / span;
      o.f2 = (wx - g[i]) / span;
    } else {
      o.f1 = (g[i + 1] + wx) / span;
      o.f2 = (-g[i] - wx) / span;
    }
    o.ifreq = i;
  } else if (wx > 0.0) {
    const int i = bracket_last(wx, nFreq, g, 0);
    const double span = g[i + 1] - g[i];
    o.f1 = -0.5 * (g[i + 1] - wx) / span;
    o.f2 = -0.5 * (wx - g[i]) / span;
    o.ifreq = i;
  } else if (flag_occ) {
    const double x = -wx;
    int i = bracket_last(x, nFreq, g, 0);
    if (i == 0) i = nFreq - 2;
    const double span = g[i + 1] - g[i];
    o.f1 = (g[i + 1] - x) / span;
    o.f2 = (x - g[i]) / span;
    o.ifreq = i;
  }
  return o;
}

namespace {

constexpr int kTM = 32;        // rows (bands) per tile
constexpr int kTN = 64;        // G' columns per tile
constexpr int kBK = 8;         // complex k per pipeline stage
constexpr int kLds = kBK + 4;  // padded row stride (double2): 192 B, conflict-free fragment reads
constexpr int kStages = 2;     // cp.async double buffer (3 CTAs / 12 warps per SM fit)
constexpr int kFFThreads = 128;

struct GroupKey {
  int out, src, f;
  bool operator<(const GroupKey &o) const { return std::tie(out, src, f) < std::tie(o.out, o.src, o.f); }
};

// Builds rows and tiles.  ekq/grid are host copies.
int build_plan(int64_t nb, int64_t nvband, int64_t P, int64_t G, int64_t nFreq, double fmin, double fstep,
               double occ, const double *ekq, const double *grid, bool want_achs, bool want_asx, bool want_cor,
               bool per_iw, int64_t nE, int target_ctas, FFPlan *plan) {
  // Evaluation points with a distinct wx: iw = 0 .. nE - 1 with
  // wx = fmin - ekq + iw fstep, or the reference's single wx = fmin - ekq +
  // fstep (ff.cpp:245, 337).  Rows of every iw that read the same slice
  // share one group (one GEMM over that slice).
  const int64_t n_iw = per_iw ? nE : 1;
  auto wx_of = [&](int64_t n1, int64_t iw) { return fmin - ekq[n1] + (per_iw ? (double)iw : 1.0) * fstep; };
  std::map<GroupKey, std::vector<FFRow>> groups;
  if (want_achs) {
    auto &g = groups[{OUT_ACHS, SRC_R, 1}];
    for (int64_t n1 = 0; n1 < nb; ++n1) g.push_back({(int32_t)n1, 0, -0.5});
  }
  // Per-iw rows (band, iw, coef) of each group, before deduplication.
  struct IwRow {
    int32_t band, iw;
    double coef;
  };
  // Rows are collected in dense (out, src, slice) buckets, then moved into
  // the ordered maps (a map lookup per row costs more than the whole plan).
  const int64_t nkeys = (int64_t)OUT_COUNT * 3 * (nFreq + 1);
  auto kidx = [&](const GroupKey &k) { return ((int64_t)k.out * 3 + k.src) * (nFreq + 1) + k.f; };
  std::vector<std::vector<FFRow>> dense_rows(per_iw ? 0 : nkeys);
  std::vector<std::vector<IwRow>> dense_iw(per_iw ? nkeys : 0);
  auto add = [&](const GroupKey &k, int64_t n1, int64_t iw, double coef) {
    if (per_iw)
      dense_iw[kidx(k)].push_back({(int32_t)n1, (int32_t)iw, coef});
    else
      dense_rows[kidx(k)].push_back({(int32_t)n1, 0, coef});
  };
  if (want_asx) {
    for (int64_t iw = 0; iw < n_iw; ++iw)
    for (int64_t n1 = 0; n1 < nvband; ++n1) {
      const double wx = wx_of(n1, iw);
      const Fact fc = compute_fact_host(wx, (int)nFreq, grid, 1, false);
      const int src = wx > 0 ? SRC_R : SRC_A;
      add({OUT_ASX, src, fc.ifreq}, n1, iw, fc.f1 * occ);
      add({OUT_ASX, src, fc.ifreq + 1}, n1, iw, fc.f2 * occ);
    }
  }
  if (want_cor) {
    for (int64_t iw = 0; iw < n_iw; ++iw)
    for (int64_t n1 = 0; n1 < nb; ++n1) {
      const bool flag_occ = n1 < nvband;
      const double wx = wx_of(n1, iw);
      const Fact fc = compute_fact_host(wx, (int)nFreq, grid, 2, flag_occ);
      double s;
      if (wx > 0) {
        if (flag_occ) continue;  // schDttt_corKernel1 only for unoccupied bands
        s = 1.0;
      } else if (flag_occ) {
        s = -0.5;  // schDttt_corKernel2 (ff.cpp:437-444)
      } else {
        continue;
      }
      add({OUT_COR, SRC_RA, fc.ifreq}, n1, iw, fc.f1 * s);
      add({OUT_COR, SRC_RA, fc.ifreq + 1}, n1, iw, fc.f2 * s);
    }
  }
  std::map<GroupKey, std::vector<IwRow>> iw_rows;
  for (int out = 0; out < OUT_COUNT; ++out)
    for (int src = 0; src < 3; ++src)
      for (int f = 0; f <= (int)nFreq; ++f) {
        const GroupKey k{out, src, f};
        const int64_t i = kidx(k);
        if (per_iw && !dense_iw[i].empty()) iw_rows[k] = std::move(dense_iw[i]);
        if (!per_iw && !dense_rows[i].empty()) groups[k] = std::move(dense_rows[i]);
      }
  // Per-iw: one row per distinct band of a group (coef 1, bands ascending);
  // each (band, iw) becomes a term on output ff_out_index(out, iw).
  if (per_iw) {
    if (want_achs) {
      auto &g = groups[{OUT_ACHS, SRC_R, 1}];
      for (auto &r : g) r.coef = 1.0;
    }
    std::vector<char> used((size_t)std::max<int64_t>(nb, 1));
    for (auto &kv : iw_rows) {
      std::fill(used.begin(), used.end(), 0);
      for (const auto &r : kv.second) used[r.band] = 1;
      auto &g = groups[kv.first];
      for (int64_t b = 0; b < nb; ++b)
        if (used[b]) g.push_back({(int32_t)b, 0, 1.0});
    }
  }
  plan->rows.clear();
  plan->tiles.clear();
  plan->groups.clear();
  plan->useful_cmacs = 0.0;
  plan->per_iw = per_iw;
  plan->terms.clear();
  std::vector<int32_t> row_of_band;
  std::vector<std::vector<FFTerm>> terms_of((size_t)(1 + 2 * std::max<int64_t>(nE, 0)));
  for (auto &kv : groups) {
    const GroupKey &key = kv.first;
    const int32_t rb = (int32_t)plan->rows.size();
    const int64_t nrows = (int64_t)kv.second.size();
    plan->rows.insert(plan->rows.end(), kv.second.begin(), kv.second.end());
    plan->groups.push_back({key.out, key.src, key.f, rb, (int32_t)nrows});
    plan->useful_cmacs += (double)nrows * (double)P * (double)G;
    if (per_iw) {
      if (key.out == OUT_ACHS) {
        for (int64_t r = 0; r < nrows; ++r) terms_of[0].push_back({rb + (int32_t)r, 0, -0.5});
      } else {
        row_of_band.assign((size_t)std::max<int64_t>(nb, 1), -1);
        for (int64_t r = 0; r < nrows; ++r) row_of_band[kv.second[r].band] = rb + (int32_t)r;
        for (const auto &t : iw_rows[key]) {
          const int o = ff_out_index(key.out, t.iw, nE);
          terms_of[o].push_back({row_of_band[t.band], o, t.coef});
        }
      }
    }
  }
  for (auto &v : terms_of) plan->terms.insert(plan->terms.end(), v.begin(), v.end());  // sorted by output
  // Tiles in group (= output) order; seg[o] = first tile of output o.
  ff_fp64_tiles(plan->groups, P, G, target_ctas, &plan->tiles);
  for (int o = 0; o <= OUT_COUNT; ++o) {
    int first = (int)plan->tiles.size();
    for (int i = 0; i < (int)plan->tiles.size(); ++i)
      if (plan->tiles[i].out >= o) {
        first = i;
        break;
      }
    plan->seg[o] = first;
  }
  // Distinct (array, slice) pairs read: 1 per R or A slice, 2 per R - A slice.
  {
    std::map<std::pair<int, int>, int> seen;
    for (auto &kv : groups) {
      if (kv.first.src != SRC_A) seen[{0, kv.first.f}] = 1;
      if (kv.first.src != SRC_R) seen[{1, kv.first.f}] = 1;
    }
    plan->slice_reads.assign(1, (double)seen.size());
  }
  for (auto &kv : groups) {
    const int f = kv.first.f;
    if (kv.first.src == SRC_R || kv.first.src == SRC_RA) {
      plan->r_lo = std::min(plan->r_lo, f);
      plan->r_hi = std::max(plan->r_hi, f);
    }
    if (kv.first.src == SRC_A || kv.first.src == SRC_RA) {
      plan->a_lo = std::min(plan->a_lo, f);
      plan->a_hi = std::max(plan->a_hi, f);
    }
  }
  return BGW_OK;
}

// ------------------------------------------------------------------ prep --
// W[n1][p] = conj(aqsm[n1][igp]) * vcoul[igp], igp = indinv[inv[p]] (checked).
__global__ void ff_w_kernel(int nb, int P, int G, const int *__restrict__ inv, const int *__restrict__ indinv,
                            long long indinv_len, const double2 *__restrict__ am, const double *__restrict__ vc,
                            double2 *__restrict__ W, int *status) {
  const long long total = (long long)nb * P;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int n1 = (int)(idx / P), p = (int)(idx % P);
    const int a = inv[p];
    double2 w = make_double2(0.0, 0.0);
    if (a < 0 || (long long)a >= indinv_len) {
      raise_status(status, BGW_ERR_INDEX, p);
    } else {
      const int g = indinv[a];
      if (g < 0 || g >= G) {
        raise_status(status, BGW_ERR_INDEX, p);
      } else {
        const double2 m = am[(size_t)n1 * G + g];
        const double v = vc[g];
        w = make_double2(m.x * v, -m.y * v);
      }
    }
    W[idx] = w;
  }
}

// ------------------------------------------------------- DMMA contraction --
// Not volatile: the MMA has no side effects, so the compiler may interleave
// independent accumulators to hide the DMMA latency.
__device__ __forceinline__ void dmma_f64(double &c0, double &c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

// cp.async (16-byte, L2-only) global -> shared copies.  `valid` false
// zero-fills the destination without reading the source.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(smem)), "l"(gmem),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

struct FFStage {
  double2 a[kTM * kLds];   // aqsn rows of the tile
  double2 b[kTN * kLds];   // X_f rows (I_epsR or I_epsA)
  double2 b2[kTN * kLds];  // I_epsA rows when the tile needs R - A
};
struct FFSmem {
  FFStage st[kStages];
  double red[(kFFThreads / 32) * 2];
  double row_red[kFFThreads / 32][kTM][2];  // per-row partials of each warp
};

// One CTA per tile.  4 warps; warp w owns G' columns [16w, 16w + 16) of the
// tile and all 32 rows: 4 x 2 m8n8 blocks, each complex block kept as three
// real DMMA accumulators of Gauss's three-multiplication product (3 real
// MMAs per complex k4 step instead of 4):
//   K1 += (Ar + Ai) Br,  K2 += Ar (Bi - Br),  K3 += Ai (Br + Bi),
//   Re = K1 - K3 = sum Ar Br - Ai Bi,  Im = K1 + K2 = sum Ar Bi + Ai Br.
// Operands stream global -> shared through a kStages-deep cp.async pipeline
// (rows gathered by band index, out-of-range rows / k zero-filled); for the
// COR sum the I_epsR and I_epsA rows are staged separately and R - A is
// formed when the B fragments are read.
// MC = 8-row blocks of the tile that hold real rows (1..4): the all-padding
// blocks of a partly filled tile are neither copied nor multiplied.
template <int MC, bool ROWS>
__device__ __forceinline__ void contract_tile(FFSmem &sm, const FFTile &t, const FFRow *__restrict__ rows, int P,
                                              int G, const double2 *__restrict__ aqsn,
                                              const double2 *__restrict__ R, int r_f0,
                                              const double2 *__restrict__ A, int a_f0,
                                              const double2 *__restrict__ W, double *__restrict__ partials,
                                              int nb, int *status) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g8 = lane >> 2, t4 = lane & 3;

  const size_t slice = (size_t)P * G;
  // R / A point at slice r_f0 / a_f0 (host-staged inputs hold only the
  // slices the plan reads).
  const double2 *X0 = (t.src == SRC_A) ? A + (size_t)(t.f - a_f0) * slice : R + (size_t)(t.f - r_f0) * slice;
  const bool sub = (t.src == SRC_RA);
  const double2 *X1 = sub ? A + (size_t)(t.f - a_f0) * slice : X0;

  // Copy assignment: element idx = q * 128 + tid of a [rows][kBK] tile,
  // row idx / kBK, k offset idx % kBK.
  constexpr int kAq = kTM * kBK / kFFThreads, kBq = kTN * kBK / kFFThreads;
  const int kc = tid % kBK;
  const double2 *a_src[kAq];
  bool a_ok[kAq];
#pragma unroll
  for (int q = 0; q < kAq; ++q) {
    const int r = (q * kFFThreads + tid) / kBK;
    a_ok[q] = r < t.row_count && BGW_CHECKED(r >= t.row_count || (unsigned)rows[t.row_begin + r].band < (unsigned)nb,
                                             status, 42);
    a_src[q] = a_ok[q] ? aqsn + (size_t)rows[t.row_begin + r].band * G + t.k_begin + kc : aqsn;
  }
  const double2 *b_src[kBq];
  const double2 *b2_src[kBq];
  bool b_ok[kBq];
#pragma unroll
  for (int q = 0; q < kBq; ++q) {
    const int p = t.p_begin + (q * kFFThreads + tid) / kBK;
    b_ok[q] = p < P;
    b_src[q] = b_ok[q] ? X0 + (size_t)p * G + t.k_begin + kc : X0;
    b2_src[q] = b_ok[q] ? X1 + (size_t)p * G + t.k_begin + kc : X1;
  }

  const int nk = (t.k_count + kBK - 1) / kBK;
  auto issue = [&](int kb, int buf) {
    FFStage &s = sm.st[buf];
    const bool kin = kb * kBK + kc < t.k_count;
    const size_t off = (size_t)kb * kBK;
#pragma unroll
    for (int q = 0; q < kAq; ++q) {
      if (q * (kFFThreads / kBK) >= MC * 8) continue;  // rows of this copy are all padding
      const int idx = q * kFFThreads + tid;
      const bool v = kin && a_ok[q];
      cp_async16(&s.a[(idx / kBK) * kLds + kc], v ? a_src[q] + off : aqsn, v);
    }
#pragma unroll
    for (int q = 0; q < kBq; ++q) {
      const int idx = q * kFFThreads + tid;
      const bool v = kin && b_ok[q];
      cp_async16(&s.b[(idx / kBK) * kLds + kc], v ? b_src[q] + off : X0, v);
      if (sub) cp_async16(&s.b2[(idx / kBK) * kLds + kc], v ? b2_src[q] + off : X1, v);
    }
  };

  double k1[4][2][2], k2[4][2][2], k3[4][2][2];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 2; ++n)
#pragma unroll
      for (int j = 0; j < 2; ++j) k1[m][n][j] = k2[m][n][j] = k3[m][n][j] = 0.0;

#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) issue(s, s);
    cp_async_commit();
  }
  for (int kb = 0; kb < nk; ++kb) {
    cp_async_wait<kStages - 2>();
    __syncthreads();  // stage kb landed for every thread; stage kb-1 fully consumed
    const int nxt = kb + kStages - 1;
    if (nxt < nk) issue(nxt, nxt % kStages);
    cp_async_commit();
    const FFStage &s = sm.st[kb % kStages];
    const double2 *sa = s.a;
    const double2 *sb = s.b + (warp * 16) * kLds;
    const double2 *sb2 = s.b2 + (warp * 16) * kLds;
#pragma unroll
    for (int ks = 0; ks < kBK / 4; ++ks) {
      double ar[4], ai[4], as[4], br[2], bd[2], bs[2];
#pragma unroll
      for (int m = 0; m < MC; ++m) {
        const double2 v = sa[(m * 8 + g8) * kLds + ks * 4 + t4];
        ar[m] = v.x;
        ai[m] = v.y;
        as[m] = v.x + v.y;
      }
#pragma unroll
      for (int n = 0; n < 2; ++n) {
        double2 v = sb[(n * 8 + g8) * kLds + ks * 4 + t4];
        if (sub) {
          const double2 y = sb2[(n * 8 + g8) * kLds + ks * 4 + t4];
          v.x -= y.x;
          v.y -= y.y;
        }
        br[n] = v.x;
        bd[n] = v.y - v.x;
        bs[n] = v.x + v.y;
      }
      // Three sweeps, one per Gauss product: each accumulator receives one
      // MMA per k4 step, 2 MC MMAs after the previous one into it.
#pragma unroll
      for (int m = 0; m < MC; ++m)
#pragma unroll
        for (int n = 0; n < 2; ++n) dmma_f64(k1[m][n][0], k1[m][n][1], as[m], br[n]);
#pragma unroll
      for (int m = 0; m < MC; ++m)
#pragma unroll
        for (int n = 0; n < 2; ++n) dmma_f64(k2[m][n][0], k2[m][n][1], ar[m], bd[n]);
#pragma unroll
      for (int m = 0; m < MC; ++m)
#pragma unroll
        for (int n = 0; n < 2; ++n) dmma_f64(k3[m][n][0], k3[m][n][1], ai[m], bs[n]);
    }
  }
  cp_async_wait<0>();

  // Epilogue: sum_r coef(r) sum_p W(band(r), p) C(r, p) over this thread's
  // accumulator entries (row m*8+g8, column warp*16 + n*8 + 2*t4 + j).
  // ROWS: one partial per tile row instead (rows of one tile may feed
  // different outputs), reduced over the 4 lanes and 4 warps sharing a row.
  double vr = 0.0, vi = 0.0;
  double rv[MC][2];
#pragma unroll
  for (int m = 0; m < MC; ++m) {
    rv[m][0] = rv[m][1] = 0.0;
    const int r = m * 8 + g8;
    if (r >= t.row_count) continue;
    const FFRow row = rows[t.row_begin + r];
#pragma unroll
    for (int n = 0; n < 2; ++n)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int p = t.p_begin + warp * 16 + n * 8 + 2 * t4 + j;
        if (p >= P) continue;
        const double2 w = W[(size_t)row.band * P + p];
        const double xr = k1[m][n][j] - k3[m][n][j], xi = k1[m][n][j] + k2[m][n][j];
        if (ROWS) {
          rv[m][0] = fma(row.coef, xr * w.x - xi * w.y, rv[m][0]);
          rv[m][1] = fma(row.coef, xr * w.y + xi * w.x, rv[m][1]);
        } else {
          vr = fma(row.coef, xr * w.x - xi * w.y, vr);
          vi = fma(row.coef, xr * w.y + xi * w.x, vi);
        }
      }
  }
  if (ROWS) {
#pragma unroll
    for (int m = 0; m < MC; ++m)
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        rv[m][k] += __shfl_xor_sync(0xffffffffu, rv[m][k], 1);
        rv[m][k] += __shfl_xor_sync(0xffffffffu, rv[m][k], 2);
      }
    if (t4 == 0)
#pragma unroll
      for (int m = 0; m < MC; ++m) {
        sm.row_red[warp][m * 8 + g8][0] = rv[m][0];
        sm.row_red[warp][m * 8 + g8][1] = rv[m][1];
      }
    __syncthreads();
    if (tid < kTM) {
      double pr = 0.0, pi = 0.0;
      if (tid < MC * 8)
        for (int w = 0; w < kFFThreads / 32; ++w) {
          pr += sm.row_red[w][tid][0];
          pi += sm.row_red[w][tid][1];
        }
      partials[((size_t)blockIdx.x * kTM + tid) * 2 + 0] = pr;
      partials[((size_t)blockIdx.x * kTM + tid) * 2 + 1] = pi;
    }
    return;
  }
  double v[2] = {vr, vi};
  block_sum<2, kFFThreads>(v, sm.red);
  if (tid == 0) {
    partials[(size_t)blockIdx.x * 2 + 0] = v[0];
    partials[(size_t)blockIdx.x * 2 + 1] = v[1];
  }
}

__global__ void __launch_bounds__(kFFThreads, 3)
    ff_contract_kernel(const FFTile *__restrict__ tiles, const FFRow *__restrict__ rows, int P, int G,
                       const double2 *__restrict__ aqsn, const double2 *__restrict__ R, int r_f0,
                       const double2 *__restrict__ A, int a_f0, const double2 *__restrict__ W,
                       double *__restrict__ partials, int per_row, int nb, int n_rows, int *status,
                       const int *__restrict__ gate, const int *__restrict__ unit_flag) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  FFSmem &sm = *reinterpret_cast<FFSmem *>(smem_raw);
  // A gated tile (FP64 recomputation of an integer-slice unit) runs only
  // when that unit flagged a value outside its digit range; otherwise its
  // partial is zero.
  if (gate) {
    const int u = gate[blockIdx.x];
    if (u >= 0 && unit_flag[u] == 0) {
      const int n = per_row ? 2 * kTM : 2;
      for (int i = threadIdx.x; i < n; i += blockDim.x) partials[(size_t)blockIdx.x * n + i] = 0.0;
      return;
    }
  }
  FFTile t = tiles[blockIdx.x];
  // Debug build: the tile's rows, columns and k range lie inside the plan
  // and the arrays (a failing tile contributes zero).
  if (!BGW_CHECKED(t.row_count >= 0 && t.row_count <= kTM && t.row_begin >= 0 && t.row_begin + t.row_count <= n_rows &&
                       t.p_begin >= 0 && t.p_begin < P && t.k_begin >= 0 && t.k_count >= 0 &&
                       t.k_begin + t.k_count <= G,
                   status, 41)) {
    t.row_count = 0;
    t.k_count = 0;
  }
  const int mc = min(4, (t.row_count + 7) >> 3);  // uniform per CTA
  if (per_row) {
    switch (mc) {
      case 1: contract_tile<1, true>(sm, t, rows, P, G, aqsn, R, r_f0, A, a_f0, W, partials, nb, status); break;
      case 2: contract_tile<2, true>(sm, t, rows, P, G, aqsn, R, r_f0, A, a_f0, W, partials, nb, status); break;
      case 3: contract_tile<3, true>(sm, t, rows, P, G, aqsn, R, r_f0, A, a_f0, W, partials, nb, status); break;
      default: contract_tile<4, true>(sm, t, rows, P, G, aqsn, R, r_f0, A, a_f0, W, partials, nb, status); break;
    }
    return;
  }
  switch (mc) {
    case 1: contract_tile<1, false>(sm, t, rows, P, G, aqsn, R, r_f0, A, a_f0, W, partials, nb, status); break;
    case 2: contract_tile<2, false>(sm, t, rows, P, G, aqsn, R, r_f0, A, a_f0, W, partials, nb, status); break;
    case 3: contract_tile<3, false>(sm, t, rows, P, G, aqsn, R, r_f0, A, a_f0, W, partials, nb, status); break;
    default: contract_tile<4, false>(sm, t, rows, P, G, aqsn, R, r_f0, A, a_f0, W, partials, nb, status); break;
  }
}

// Sums the partials of each output segment in tile order and writes
// achs (1 complex), asx (nE complex) and cor (nE complex).  One block.
__global__ void __launch_bounds__(256)
    ff_finalize_kernel(const double *__restrict__ partials, int s0, int s1, int s2, int s3, int nE,
                       double *__restrict__ achs, double *__restrict__ asx, double *__restrict__ cor) {
  __shared__ double red[8 * 2];
  __shared__ double res[OUT_COUNT][2];
  const int seg[4] = {s0, s1, s2, s3};
  for (int o = 0; o < OUT_COUNT; ++o) {
    double v[2] = {0.0, 0.0};
    for (int i = seg[o] + threadIdx.x; i < seg[o + 1]; i += 256) {
      v[0] += partials[(size_t)i * 2];
      v[1] += partials[(size_t)i * 2 + 1];
    }
    block_sum<2, 256>(v, red);
    if (threadIdx.x == 0) {
      res[o][0] = v[0];
      res[o][1] = v[1];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && achs) {
    achs[0] = res[OUT_ACHS][0];
    achs[1] = res[OUT_ACHS][1];
  }
  for (int i = threadIdx.x; i < nE; i += 256) {
    if (asx) {
      asx[2 * i] = res[OUT_ASX][0];
      asx[2 * i + 1] = res[OUT_ASX][1];
    }
    if (cor) {
      cor[2 * i] = res[OUT_COR][0];
      cor[2 * i + 1] = res[OUT_COR][1];
    }
  }
}

// Output o (0 = achsDtemp, 1 + iw = asxDtemp[iw], 1 + nE + iw =
// achDtemp_cor[iw]) = sum over its terms t (thread-strided in order, then
// block_sum) of coef_t * (sum of the partials of row_t, in order): bitwise
// reproducible.
__global__ void __launch_bounds__(256)
    ff_term_finalize_kernel(const double *__restrict__ partials, const int *__restrict__ row_ptr,
                            const int *__restrict__ part_idx, const int *__restrict__ out_ptr,
                            const int *__restrict__ term_row, const double *__restrict__ term_coef, int nE,
                            double *__restrict__ achs, double *__restrict__ asx, double *__restrict__ cor) {
  __shared__ double red[8 * 2];
  const int o = blockIdx.x;
  double v[2] = {0.0, 0.0};
  for (int t = out_ptr[o] + threadIdx.x; t < out_ptr[o + 1]; t += 256) {
    const int r = term_row[t];
    double sr = 0.0, si = 0.0;
    for (int j = row_ptr[r]; j < row_ptr[r + 1]; ++j) {
      const int i = part_idx[j];
      sr += partials[(size_t)i * 2];
      si += partials[(size_t)i * 2 + 1];
    }
    v[0] = fma(term_coef[t], sr, v[0]);
    v[1] = fma(term_coef[t], si, v[1]);
  }
  block_sum<2, 256>(v, red);
  if (threadIdx.x != 0) return;
  double *dst = o == 0 ? achs : o <= nE ? (asx ? asx + 2 * (o - 1) : nullptr) : (cor ? cor + 2 * (o - 1 - nE) : nullptr);
  if (dst) {
    dst[0] = v[0];
    dst[1] = v[1];
  }
}

}  // namespace

// Builds the plan of the requested sums (host copies of ekq[0..nb) and
// dFreqGrid); sizes the k split for the device.
int ff_make_plan(CallEnv *env, int64_t nb, int64_t nvband, int64_t P, int64_t G, int64_t nFreq, double fmin,
                 double fstep, double occ, const double *ekq_h, const double *grid_h, bool want_achs,
                 bool want_asx, bool want_cor, bool per_iw, int64_t nE, FFPlan *plan) {
  const size_t smem = sizeof(FFSmem);
  BGW_CUDA_TRY(cudaFuncSetAttribute(ff_contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  BGW_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ff_contract_kernel, kFFThreads, smem));
  return build_plan(nb, nvband, P, G, nFreq, fmin, fstep, occ, ekq_h, grid_h, want_achs, want_asx, want_cor,
                    per_iw, nE, 2 * env->ws->sm_count * std::max(per_sm, 1), plan);
}

int ff_build_w(CallEnv *env, int64_t nb_w, int64_t G, int64_t P, const int32_t *inv, const int32_t *indinv,
               int64_t indinv_len, const double2 *am, const double *vc, double2 **W_out) {
  void *W = nullptr;
  BGW_TRY(ws_reserve(env->ws, SLOT_TABLE2, sizeof(double2) * (size_t)std::max<int64_t>(nb_w * P, 1), &W));
  if (nb_w * P > 0) {
    int g = (int)std::min<long long>((nb_w * P + 255) / 256, (long long)env->ws->sm_count * 8);
    ff_w_kernel<<<g, 256, 0, env->stream>>>((int)nb_w, (int)P, (int)G, inv, indinv, indinv_len, am, vc,
                                            (double2 *)W, env->d_status);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
  }
  *W_out = static_cast<double2 *>(W);
  return BGW_OK;
}

void ff_fp64_tiles(const std::vector<FFGroup> &groups, int64_t P, int64_t G, int target_ctas,
                   std::vector<FFTile> *tiles) {
  const int64_t ptiles = (P + kTN - 1) / kTN;
  int64_t base = 0;
  for (const auto &g : groups) base += ((int64_t)g.row_count + kTM - 1) / kTM * ptiles;
  const int64_t kblocks = (G + kBK - 1) / kBK;
  int64_t ksplit = base > 0 ? (target_ctas + base - 1) / base : 1;
  ksplit = std::max<int64_t>(1, std::min<int64_t>(ksplit, std::max<int64_t>(1, kblocks / 8)));
  const int64_t kb_per = (kblocks + ksplit - 1) / ksplit;
  ksplit = (kblocks + kb_per - 1) / kb_per;
  // Row tiles innermost: the tiles that read the same X block (p0, k range)
  // are launched next to each other and share it through L2.
  for (const auto &g : groups)
    for (int64_t p0 = 0; p0 < P; p0 += kTN)
      for (int64_t ks = 0; ks < ksplit; ++ks)
        for (int64_t r0 = 0; r0 < g.row_count; r0 += kTM) {
          FFTile t;
          t.src = g.src;
          t.f = g.f;
          t.row_begin = g.row_begin + (int32_t)r0;
          t.row_count = (int32_t)std::min<int64_t>(kTM, g.row_count - r0);
          t.p_begin = (int32_t)p0;
          t.k_begin = (int32_t)(ks * kb_per * kBK);
          const int64_t kend = std::min<int64_t>(G, (ks + 1) * kb_per * kBK);
          t.k_count = (int32_t)std::max<int64_t>(0, kend - t.k_begin);
          t.out = g.out;
          tiles->push_back(t);
        }
}

int ff_fp64_per_sm(int *per_sm) {
  const size_t smem = sizeof(FFSmem);
  BGW_CUDA_TRY(cudaFuncSetAttribute(ff_contract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  BGW_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, ff_contract_kernel, kFFThreads, smem));
  return BGW_OK;
}

int ff_launch_fp64_tiles(cudaStream_t stream, const FFTile *d_tiles, int ntiles, const FFRow *d_rows, int n_rows,
                         int64_t nb, int64_t P, int64_t G, const double2 *an, const double2 *R, int r_f0,
                         const double2 *A, int a_f0, const double2 *W, double *partials, int *status, bool per_row,
                         const int *gate, const int *unit_flag) {
  if (ntiles <= 0) return BGW_OK;
  int per_sm = 0;
  BGW_TRY(ff_fp64_per_sm(&per_sm));
  ff_contract_kernel<<<ntiles, kFFThreads, sizeof(FFSmem), stream>>>(d_tiles, d_rows, (int)P, (int)G, an, R, r_f0,
                                                                      A, a_f0, W, partials, per_row ? 1 : 0, (int)nb,
                                                                      n_rows, status, gate, unit_flag);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

int ff_fp64_tile_rows() { return kTM; }
int ff_fp64_tile_cols() { return kTN; }

void ff_fp64_row_ids(const std::vector<FFTile> &tiles, std::vector<int> *row_of) {
  for (const auto &t : tiles)
    for (int r = 0; r < kTM; ++r) row_of->push_back(r < t.row_count ? t.row_begin + r : -1);
}

void ff_build_term_tables(const FFPlan &plan, const std::vector<int> &row_of, int64_t nE, FFTermTables *tt) {
  const int nrows = (int)plan.rows.size(), n_out = 1 + 2 * (int)nE;
  tt->row_ptr.assign(nrows + 1, 0);
  for (int r : row_of)
    if (r >= 0) ++tt->row_ptr[r + 1];
  for (int r = 0; r < nrows; ++r) tt->row_ptr[r + 1] += tt->row_ptr[r];
  tt->part_idx.assign(tt->row_ptr[nrows], 0);
  std::vector<int> fill(tt->row_ptr.begin(), tt->row_ptr.end() - 1);
  for (int i = 0; i < (int)row_of.size(); ++i)
    if (row_of[i] >= 0) tt->part_idx[fill[row_of[i]]++] = i;  // partials of a row in index order
  tt->out_ptr.assign(n_out + 1, 0);
  tt->term_row.clear();
  tt->term_coef.clear();
  for (const auto &t : plan.terms) {  // sorted by output
    ++tt->out_ptr[t.out + 1];
    tt->term_row.push_back(t.row);
    tt->term_coef.push_back(t.coef);
  }
  for (int o = 0; o < n_out; ++o) tt->out_ptr[o + 1] += tt->out_ptr[o];
}

int ff_launch_term_finalize(CallEnv *env, int slot, const FFTermTables &tt, const double *partials, int64_t nE,
                            double *achs, double *asx, double *cor) {
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_rp = 0, o_pi = o_rp + al(sizeof(int) * tt.row_ptr.size());
  const size_t o_op = o_pi + al(sizeof(int) * std::max<size_t>(tt.part_idx.size(), 1));
  const size_t o_tr = o_op + al(sizeof(int) * tt.out_ptr.size());
  const size_t o_tc = o_tr + al(sizeof(int) * std::max<size_t>(tt.term_row.size(), 1));
  const size_t total = o_tc + al(sizeof(double) * std::max<size_t>(tt.term_coef.size(), 1));
  std::vector<unsigned char> host(total, 0);
  auto put = [&](size_t o, const void *src, size_t bytes) {
    if (bytes) std::memcpy(host.data() + o, src, bytes);
  };
  put(o_rp, tt.row_ptr.data(), sizeof(int) * tt.row_ptr.size());
  put(o_pi, tt.part_idx.data(), sizeof(int) * tt.part_idx.size());
  put(o_op, tt.out_ptr.data(), sizeof(int) * tt.out_ptr.size());
  put(o_tr, tt.term_row.data(), sizeof(int) * tt.term_row.size());
  put(o_tc, tt.term_coef.data(), sizeof(double) * tt.term_coef.size());
  void *d = nullptr;
  BGW_TRY(ws_reserve(env->ws, slot, total, &d));
  BGW_CUDA_TRY(cudaMemcpyAsync(d, host.data(), total, cudaMemcpyHostToDevice, env->stream));
  const unsigned char *b = static_cast<const unsigned char *>(d);
  const int n_out = 1 + 2 * (int)nE;
  ff_term_finalize_kernel<<<n_out, 256, 0, env->stream>>>(
      partials, (const int *)(b + o_rp), (const int *)(b + o_pi), (const int *)(b + o_op), (const int *)(b + o_tr),
      (const double *)(b + o_tc), (int)nE, achs, asx, cor);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

// Enqueues a planned FF evaluation.  Device pointers; R / A point at
// frequency slice r_f0 / a_f0.  Outputs are device pointers (nullptr skips).
int ff_launch(CallEnv *env, const FFPlan &plan, int64_t nb_w, int64_t nE, int64_t G, int64_t P,
              const int32_t *inv, const int32_t *indinv, int64_t indinv_len, const double2 *am, const double2 *an,
              const double *vc, const double2 *R, int r_f0, const double2 *A, int a_f0, double *achs_dev,
              double *asx_dev, double *cor_dev) {
  Workspace *ws = env->ws;
  cudaStream_t stream = env->stream;
  const size_t smem = sizeof(FFSmem);

  // Plan upload: rows then tiles, one copy.
  const size_t rows_bytes = sizeof(FFRow) * plan.rows.size();
  const size_t tiles_off = (rows_bytes + 255) & ~size_t(255);
  const size_t plan_bytes = tiles_off + sizeof(FFTile) * plan.tiles.size();
  std::vector<unsigned char> host_plan(std::max<size_t>(plan_bytes, 1));
  if (rows_bytes) std::memcpy(host_plan.data(), plan.rows.data(), rows_bytes);
  if (!plan.tiles.empty())
    std::memcpy(host_plan.data() + tiles_off, plan.tiles.data(), sizeof(FFTile) * plan.tiles.size());
  void *d_plan = nullptr, *W = nullptr, *partials = nullptr;
  BGW_TRY(ws_reserve(ws, SLOT_PLAN, host_plan.size(), &d_plan));
  BGW_CUDA_TRY(cudaMemcpyAsync(d_plan, host_plan.data(), host_plan.size(), cudaMemcpyHostToDevice, stream));
  const FFRow *d_rows = reinterpret_cast<const FFRow *>(d_plan);
  const FFTile *d_tiles = reinterpret_cast<const FFTile *>(static_cast<unsigned char *>(d_plan) + tiles_off);

  BGW_TRY(ws_reserve(ws, SLOT_TABLE2, sizeof(double2) * (size_t)std::max<int64_t>(nb_w * P, 1), &W));
  if (nb_w * P > 0) {
    int g = (int)std::min<long long>((nb_w * P + 255) / 256, (long long)ws->sm_count * 8);
    ff_w_kernel<<<g, 256, 0, stream>>>((int)nb_w, (int)P, (int)G, inv, indinv, indinv_len, am, vc, (double2 *)W,
                                       env->d_status);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
  }
  const int ntiles = (int)plan.tiles.size();
  // Distinct outputs per iw: one partial per tile row, combined by the terms.
  const bool per_row = plan.per_iw;
  std::vector<int> row_of;
  if (per_row) ff_fp64_row_ids(plan.tiles, &row_of);
  const size_t n_part = per_row ? row_of.size() : (size_t)ntiles;
  BGW_TRY(ws_reserve(ws, SLOT_PARTIALS, sizeof(double) * 2 * std::max<size_t>(n_part, 1), &partials));
  BGW_TRY(prof_mark(env, 1));
  if (ntiles > 0) {
    ff_contract_kernel<<<ntiles, kFFThreads, smem, stream>>>(d_tiles, d_rows, (int)P, (int)G, an, R, r_f0, A, a_f0,
                                                             (const double2 *)W, (double *)partials,
                                                             per_row ? 1 : 0, (int)nb_w, (int)plan.rows.size(),
                                                             env->d_status, nullptr, nullptr);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
  }
  BGW_TRY(prof_mark(env, 2));
  {
    // Compulsory bytes of the contraction: every frequency slice it reads
    // (R, A or both) once, plus the aqsn rows and the W table.
    double slices = 0.0;
    for (const auto &b : plan.slice_reads) slices += b;
    env->prof.flops = 8.0 * plan.useful_cmacs;
    env->prof.main_bytes = slices * 16.0 * (double)P * (double)G + 16.0 * (double)nb_w * (double)G +
                           16.0 * (double)nb_w * (double)P;
    env->prof.main_launches = ntiles > 0 ? 1 : 0;
    std::snprintf(env->prof.main_kernel, sizeof(env->prof.main_kernel), "ff_contract_kernel");
  }
  if (per_row) {
    FFTermTables tt;
    ff_build_term_tables(plan, row_of, nE, &tt);
    BGW_TRY(ff_launch_term_finalize(env, SLOT_TABLE1, tt, (const double *)partials, nE, achs_dev, asx_dev,
                                    cor_dev));
  } else {
    ff_finalize_kernel<<<1, 256, 0, stream>>>((const double *)partials, plan.seg[0], plan.seg[1], plan.seg[2],
                                              plan.seg[3], (int)nE, achs_dev, asx_dev, cor_dev);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
  }
  // The pageable plan buffer must outlive its (staged) upload.
  BGW_CUDA_TRY(cudaStreamSynchronize(stream));
  return BGW_OK;
}

}  // namespace bgw
