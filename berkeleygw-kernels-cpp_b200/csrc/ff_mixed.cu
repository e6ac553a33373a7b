// ff_mixed.cu -- mixed-precision FF sums: integer-slice (Ozaki) products on
// the sm_100a tensor cores (tcgen05.mma kind::i8), FP64 recombination.
//
// Split.  Each operand row (an aqsn band row on the A side, a G' row of the
// frequency slice X_f on the B side) is scaled by 2^-e (e from frexp of the
// row's largest |re| / |im|, so every scaled entry lies in (-1, 1)) and cut
// into kS signed digits of 7 bits: x 2^-e = sum_s d_s 128^-s + r,
// |d_s| <= 127, |r| < 128^-kS.  The digits are exact in int8, every digit
// product is exact in int32, so C = A X^T is recovered as
//   C(r, p) = 2^(eA(r) + eB(p)) sum_L 128^-L C_L(r, p),
//   C_L = sum_{s + t = L} A_s X_t^T   (L = 2 .. kS + 1; the digit pairs of
//                                       higher levels are dropped),
// following the integer Ozaki scheme of H. Ootomo, K. Ozaki and R. Yokota,
// "DGEMM on integer matrix multiplication unit" (IJHPCA 2024).  Complex
// products use four real products per digit pair: Re += A_r X_r + (-A_i) X_i,
// Im += A_r X_i + A_i X_r (the -A_i digits are stored: kind::i8 MMAs have no
// operand negation).
//
// Kernels.  ff_slice_kernel writes the digits straight into the tcgen05
// canonical K-major layout (core matrices of 8 rows x 16 bytes), one packed
// tile per (plane, digit, row tile, 64-k block), so a pipeline stage is one
// 1-D bulk copy per plane.  ff_mix_gemm_kernel is persistent, one CTA per
// SM: the (tile, k block) units of all groups are split evenly over the CTAs
// as segments; warp 0 stages digit tiles with bulk copies (5 stages), warp 1
// issues the MMAs (M = 128 rows, N = 128 columns, K = 32 per instruction)
// into two int32 TMEM accumulators (Re, Im) per level, double-buffered in the
// 512 columns so that a level drains while the next one multiplies;
// warps 2-9 drain each finished level (tcgen05.ld), convert to FP64 and fold
// W(band, p) 2^eB(p) 128^-L into a per-row sum; the row factor coef 2^eA and
// a fixed-order reduction give one partial per segment.  Every mbarrier wait
// is bounded.  Groups of at most 16 rows (the SX sum's) go to the FP64 DMMA
// kernel instead: a 128-row integer tile would be mostly padding.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "bgw_internal.cuh"
#include "ff_plan.cuh"
#include "reduce.cuh"
#include "tcgen05.cuh"

namespace bgw {
namespace {

constexpr int kS = 6;                        // digits per operand
constexpr int kLevels = kS;                  // levels L = 2 .. kS + 1
constexpr int kM = 128;                      // A rows per tile (MMA M)
constexpr int kN = 128;                      // X rows per tile (MMA N)
constexpr int kBK = 64;                      // k per packed tile / pipeline stage
constexpr int kATile = kM * kBK;             // 8 KB
constexpr int kXTile = kN * kBK;             // 16 KB
constexpr int kALbo = kM * 16;               // bytes between 16-k column groups
constexpr int kXLbo = kN * 16;
constexpr int kAPlanes = 3;                  // Re, Im, -Im
constexpr int kXPlanes = 2;                  // Re, Im
constexpr int kStages = 5;
constexpr int kAccBufs = 512 / (2 * kN);     // TMEM accumulator sets (Re + Im)
constexpr int kEpiWarps = 8;                 // two per TMEM lane quarter (column halves)
constexpr int kMixThreads = 64 + 32 * kEpiWarps;  // warp 0 copies, warp 1 MMAs, warps 2.. epilogue
constexpr int kMixMinRows = 128;             // default: smaller groups use the FP64 kernel
constexpr int kMixMinRowsAll = 17;           // with BGW_FLAG_FF_SLICE_ALL
constexpr int kMaxSegBlocks = 128;           // 8192 k: every int32 accumulator stays below 2^31
constexpr int kWinBlocks = 32;               // k blocks sharing one row scale (2048 k)
constexpr int kSliceThreads = 256;
constexpr int kSliceK = kWinBlocks * kBK / kSliceThreads;  // consecutive k per slicing thread
constexpr uint32_t kStageBytes = kAPlanes * kATile + kXPlanes * kXTile;
static_assert(kAccBufs >= 1, "TMEM holds at least one Re/Im accumulator pair");
static_assert(kBK % 32 == 0 && kBK % 16 == 0, "k block is a whole number of MMA k steps");
static_assert(kSliceK == 8, "a slicing thread writes one 8-byte word pair per (plane, digit)");
static_assert(kS == 6, "digit extraction splits 7 kS = 42 bits into two exact 21-bit halves");
static_assert(kMaxSegBlocks % kWinBlocks == 0, "segments never straddle a scale window");

struct MixGroup {       // one integer-slice band group
  long long a_off;      // byte offset of its packed A digits
  int xid, out;         // X slice id, output id
  int prow0;            // first packed A row
  int row_tiles;        // kM-row tiles
};
struct MixRow {         // packed A row
  int band, g;
  int plan_row, pad;    // row of the plan (-1 for padding rows)
  double coef;          // 0 for padding rows
};
struct MixX {           // one distinct X = slice f of R, A or R - A
  long long b_off;      // byte offset of its packed digits
  const double2 *x0;    // slice rows
  const double2 *x1;    // subtrahend (R - A) or null
  int sb_off;           // offset of its row scales 2^eB(p)
  int pad;
};
struct MixSeg {         // k blocks [kb0, kb1) of tile (g, rt, pt), inside scale window w
  int g, rt, pt, kb0, kb1, out, w, pad;
};

// Byte offset of (row, k) inside a packed tile of `rows` rows x kBK k.
__host__ __device__ __forceinline__ int tile_off(int r, int k, int rows) {
  return (k >> 4) * (rows * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 15);
}

// One CTA per (packed row, k window of kWinBlocks blocks), 256 threads,
// 8 consecutive k per thread.  MODE 0: A rows (aqsn band rows of the integer
// groups, planes Re / Im / -Im); MODE 1 / 2: X rows (G' rows of each distinct
// slice, or of the difference of two slices; planes Re / Im).  The window is
// read once: its largest |re| / |im| gives the scale 2^e (stored to
// sA[w][row] / sB[x][w][p]), then each value becomes
// T = trunc(|x| 2^(7 kS - e)) < 2^(7 kS), whose base-128 digits with the sign
// of x are exactly the truncated 7-bit digits of x 2^-e.  Padding rows and
// k >= G are written as zero digits, so the packed buffers need no clearing.
template <int MODE>
__global__ void __launch_bounds__(kSliceThreads)
    ff_slice_kernel(const MixGroup *__restrict__ groups, const MixRow *__restrict__ arows,
                    const MixX *__restrict__ xs, int n_arows, int x_rows_padded, int P, int G, int KB, int NW,
                    const double2 *__restrict__ aqsn, int8_t *__restrict__ pack, double *__restrict__ sA,
                    double *__restrict__ sB, long long pack_bytes, int *status) {
  constexpr bool kA = MODE == 0, kSub = MODE == 2;
  __shared__ double2 stage[kSliceThreads * (kSliceK + 1)];
  __shared__ double red[kSliceThreads / 32];
  const int w = (int)(blockIdx.x % NW);
  const long long R = blockIdx.x / NW;
  const double2 *src0 = nullptr, *src1 = nullptr;
  long long plane_stride, base;
  int r_in_tile, rows;
  bool valid;
  double *scale_out;
  if (kA) {
    const MixRow row = arows[R];
    const MixGroup Gp = groups[row.g];
    const int r = (int)(R - Gp.prow0);
    valid = row.coef != 0.0;
    src0 = aqsn + (size_t)row.band * G;
    rows = kM;
    plane_stride = (long long)Gp.row_tiles * KB * kATile;
    base = Gp.a_off + (long long)(r / kM) * KB * kATile;
    r_in_tile = r % kM;
    scale_out = sA + (size_t)w * n_arows + R;
  } else {
    const int x = (int)(R / x_rows_padded);
    const int p = (int)(R % x_rows_padded);
    const MixX X = xs[x];
    valid = p < P;
    src0 = X.x0 + (size_t)(valid ? p : 0) * G;
    src1 = kSub ? X.x1 + (size_t)(valid ? p : 0) * G : nullptr;
    rows = kN;
    plane_stride = (long long)(x_rows_padded / kN) * KB * kXTile;
    base = X.b_off + (long long)(p / kN) * KB * kXTile;
    r_in_tile = p % kN;
    scale_out = valid ? sB + X.sb_off + (size_t)w * x_rows_padded + p : nullptr;
  }
  const int tile_bytes = rows * kBK;
  const int kw = w * kWinBlocks * kBK;  // first k of the window
  // Coalesced loads of the window (thread t: k = kw + 256 j + t) into shared
  // memory, padded by one double2 per 8 so that the per-thread reads of 8
  // consecutive k below hit distinct banks.
  // The loads are unconditional (index clamped into the row, value zeroed
  // after), so all of them are in flight at once.
  double2 xv[kSliceK], yv[kSliceK];
#pragma unroll
  for (int j = 0; j < kSliceK; ++j) {
    const int k = min(kw + j * kSliceThreads + (int)threadIdx.x, G - 1);
    xv[j] = src0[k];
    if (kSub) yv[j] = src1[k];
  }
  double m = 0.0;
#pragma unroll
  for (int j = 0; j < kSliceK; ++j) {
    const int kk = j * kSliceThreads + (int)threadIdx.x;
    double2 x = xv[j];
    if (kSub) {
      x.x -= yv[j].x;
      x.y -= yv[j].y;
    }
    if (!valid || kw + kk >= G) x = make_double2(0.0, 0.0);
    m = fmax(m, fmax(fabs(x.x), fabs(x.y)));
    stage[kk + (kk >> 3)] = x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  m = red[0];
#pragma unroll
  for (int i = 1; i < kSliceThreads / 32; ++i) m = fmax(m, red[i]);
  const int k0 = kw + (int)threadIdx.x * kSliceK;
  double2 v[kSliceK];
#pragma unroll
  for (int j = 0; j < kSliceK; ++j) v[j] = stage[threadIdx.x * (kSliceK + 1) + j];
  int e = 0;
  if (m > 0.0) (void)frexp(m, &e);
  if (threadIdx.x == 0 && scale_out) *scale_out = ldexp(1.0, e);
  // |x| 2^(21 - e) in [0, 2^21): its integer part holds digits 0-2, the
  // next 21 fraction bits digits 3-5 (both exact), so T = hi 2^21 + lo.
  const double mult = ldexp(1.0, 21 - e);
  if (k0 >= KB * kBK) return;  // past the packed k range (last window)

  int hr[kSliceK], lr[kSliceK], hi_[kSliceK], li_[kSliceK];
  uint32_t mr[2] = {0u, 0u}, mi[2] = {0u, 0u};  // 0xff bytes: negative entries
#pragma unroll
  for (int j = 0; j < kSliceK; ++j) {
    const double ar = fabs(v[j].x) * mult, ai = fabs(v[j].y) * mult;
    const double tr = trunc(ar), ti = trunc(ai);
    hr[j] = (int)tr;
    hi_[j] = (int)ti;
    lr[j] = (int)((ar - tr) * 2097152.0);
    li_[j] = (int)((ai - ti) * 2097152.0);
    mr[j >> 2] |= (v[j].x < 0.0 ? 0xffu : 0u) << (8 * (j & 3));
    mi[j >> 2] |= (v[j].y < 0.0 ? 0xffu : 0u) << (8 * (j & 3));
  }
  const long long off = base + (long long)(k0 / kBK) * tile_bytes + tile_off(r_in_tile, k0 % kBK, rows);
  // Debug build: every digit plane this thread writes lies in the packed buffer.
  if (!BGW_CHECKED(off >= 0 && off + ((kA ? 3LL : 2LL) * kS - 1) * plane_stride + 8 <= pack_bytes, status, 51)) return;
#pragma unroll
  for (int s = 0; s < kS; ++s) {
    const int sh = 7 * (2 - s % 3);
    uint32_t ur[2] = {0u, 0u}, ui[2] = {0u, 0u};
#pragma unroll
    for (int j = 0; j < kSliceK; ++j) {
      const uint32_t dr = ((uint32_t)(s < 3 ? hr[j] : lr[j]) >> sh) & 127u;
      const uint32_t di = ((uint32_t)(s < 3 ? hi_[j] : li_[j]) >> sh) & 127u;
      ur[j >> 2] |= dr << (8 * (j & 3));
      ui[j >> 2] |= di << (8 * (j & 3));
    }
    // Signed digits: per-byte negation where the entry is negative.
    uint32_t wr[2], wi[2], wn[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const uint32_t nr = __vneg4(ur[q]), ni = __vneg4(ui[q]);
      wr[q] = (nr & mr[q]) | (ur[q] & ~mr[q]);
      wi[q] = (ni & mi[q]) | (ui[q] & ~mi[q]);
      wn[q] = (ui[q] & mi[q]) | (ni & ~mi[q]);
    }
    *reinterpret_cast<uint2 *>(pack + off + (0LL * kS + s) * plane_stride) = make_uint2(wr[0], wr[1]);
    *reinterpret_cast<uint2 *>(pack + off + (1LL * kS + s) * plane_stride) = make_uint2(wi[0], wi[1]);
    if (kA)
      *reinterpret_cast<uint2 *>(pack + off + (2LL * kS + s) * plane_stride) = make_uint2(wn[0], wn[1]);
  }
}

struct __align__(128) MixSmem {
  int8_t a[kStages][kAPlanes][kATile];
  int8_t x[kStages][kXPlanes][kXTile];
  uint64_t full[kStages], empty[kStages], acc_full[kAccBufs], acc_empty[kAccBufs], done;
  uint32_t tmem;
  double red[kEpiWarps][2];
};

__device__ __forceinline__ bool wait_or_flag(uint64_t *bar, uint32_t parity, int *status) {
  if (mbar_wait_bounded(bar, parity, kWaitCycles)) return true;
  raise_status(status, BGW_ERR_TIMEOUT, (int)blockIdx.x);
  return false;
}

// Digit pairs (s, t), 0-based, of level L = s + t + 2, in a fixed order.
__device__ __forceinline__ int pair_lo(int L) { return max(0, L - 2 - (kS - 1)); }
__device__ __forceinline__ int pair_hi(int L) { return min(kS - 1, L - 2); }

// ROWS: one partial per (segment, column half, row) instead of one per
// segment (rows of one tile may feed different outputs).
template <bool ROWS>
__global__ void __launch_bounds__(kMixThreads, 1)
    ff_mix_gemm_kernel(const MixSeg *__restrict__ segs, const int *__restrict__ cta_seg,
                       const MixGroup *__restrict__ groups, const MixRow *__restrict__ arows,
                       const MixX *__restrict__ xs, const int8_t *__restrict__ pack, const double *__restrict__ sA,
                       const double *__restrict__ sB, int n_arows, int x_rows_padded, const double2 *__restrict__ W,
                       int P, int KB, int PT, double *__restrict__ partials, int *status, long long pack_bytes,
                       int nb_w) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  MixSmem &sm = *reinterpret_cast<MixSmem *>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int seg0 = cta_seg[blockIdx.x], seg1 = cta_seg[blockIdx.x + 1];

  if (threadIdx.x == 0) {
    for (int i = 0; i < kStages; ++i) {
      mbar_init(&sm.full[i], 1);
      mbar_init(&sm.empty[i], 1);
    }
    for (int i = 0; i < kAccBufs; ++i) {
      mbar_init(&sm.acc_full[i], 1);
      mbar_init(&sm.acc_empty[i], kEpiWarps);
    }
    mbar_init(&sm.done, 1);
    fence_mbar_init();
  }
  __syncwarp();
  if (warp == 0) {
    tc::alloc(&sm.tmem, 512);
    tc::relinquish();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = sm.tmem;

  if (warp == 0) {
    // ---- producer: digit tiles in (segment, level, pair, k block) order.
    if (lane == 0) {
      int step = 0, st = 0;
      uint32_t ph = 0;  // phase of the current pass over the stages
      bool ok = true;
      for (int sg = seg0; sg < seg1 && ok; ++sg) {
        const MixSeg S = segs[sg];
        const MixGroup Gp = groups[S.g];
        const MixX X = xs[Gp.xid];
        const long long a_plane = (long long)Gp.row_tiles * KB * kATile;
        const long long x_plane = (long long)PT * KB * kXTile;
        const int8_t *a_base = pack + Gp.a_off + ((long long)S.rt * KB + S.kb0) * kATile;
        const int8_t *x_base = pack + X.b_off + ((long long)S.pt * KB + S.kb0) * kXTile;
        for (int li = 0; li < kLevels && ok; ++li) {
          const int L = li + 2;
          for (int s = pair_lo(L); s <= pair_hi(L) && ok; ++s) {
            const int8_t *ap = a_base + s * a_plane;
            const int8_t *xp = x_base + (L - 2 - s) * x_plane;
            for (int kb = S.kb0; kb < S.kb1; ++kb) {
              // Debug build: the stage's digit tiles lie in the packed buffer.
              if (!BGW_CHECKED(ap >= pack && ap + (kAPlanes - 1) * kS * a_plane + kATile <= pack + pack_bytes &&
                                   xp >= pack && xp + (kXPlanes - 1) * kS * x_plane + kXTile <= pack + pack_bytes,
                               status, 52)) {
                ok = false;
                break;
              }
              if (step >= kStages && !wait_or_flag(&sm.empty[st], ph ^ 1u, status)) {
                ok = false;
                break;
              }
              mbar_expect_tx(&sm.full[st], kStageBytes);
#pragma unroll
              for (int pl = 0; pl < kAPlanes; ++pl)
                bulk_g2s(sm.a[st][pl], ap + pl * kS * a_plane, kATile, &sm.full[st]);
#pragma unroll
              for (int pl = 0; pl < kXPlanes; ++pl)
                bulk_g2s(sm.x[st][pl], xp + pl * kS * x_plane, kXTile, &sm.full[st]);
              ap += kATile;
              xp += kXTile;
              ++step;
              if (++st == kStages) {
                st = 0;
                ph ^= 1u;
              }
            }
          }
        }
      }
      // Copies still in flight (error paths only) land before the CTA exits:
      // wait for the last phase issued on every stage.
      for (int t = 0; t < kStages; ++t) {
        if (step <= t) continue;
        const int last = (step - 1) - ((step - 1 - t) % kStages);
        (void)wait_or_flag(&sm.full[t], (last / kStages) & 1, status);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---- MMA issuer (one thread).  Shared-memory descriptors are built
    // once; a stage / k step only adds its 16-byte-unit offset to the start
    // address field (addresses stay below 2^18, so the field never carries).
    if (lane == 0) {
      constexpr uint32_t idesc = tc::idesc_i8(kM, kN);
      const uint64_t dA = tc::smem_desc(smem_u32(&sm.a[0][0][0]), kALbo, 128);
      const uint64_t dX = tc::smem_desc(smem_u32(&sm.x[0][0][0]), kXLbo, 128);
      int st = 0, lvl = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int sg = seg0; sg < seg1 && ok; ++sg) {
        const MixSeg S = segs[sg];
        for (int li = 0; li < kLevels && ok; ++li, ++lvl) {
          const int L = li + 2, buf = lvl % kAccBufs;
          if (lvl >= kAccBufs && !wait_or_flag(&sm.acc_empty[buf], ((lvl / kAccBufs) - 1) & 1, status)) {
            ok = false;
            break;
          }
          tc::fence_after();
          const uint32_t d_re = tmem + (uint32_t)(buf * 2 * kN), d_im = d_re + kN;
          bool first = true;
          for (int s = pair_lo(L); s <= pair_hi(L) && ok; ++s) {
            for (int kb = S.kb0; kb < S.kb1; ++kb) {
              if (!wait_or_flag(&sm.full[st], ph, status)) {
                ok = false;
                break;
              }
              tc::fence_after();
              const uint64_t a_st = dA + (uint64_t)(st * (kAPlanes * kATile / 16));
              const uint64_t x_st = dX + (uint64_t)(st * (kXPlanes * kXTile / 16));
#pragma unroll
              for (int j = 0; j < kBK / 32; ++j) {  // 16-k column groups 2j, 2j + 1
                const uint64_t ar = a_st + (0 * kATile + j * 2 * kALbo) / 16;
                const uint64_t ai = a_st + (1 * kATile + j * 2 * kALbo) / 16;
                const uint64_t an = a_st + (2 * kATile + j * 2 * kALbo) / 16;
                const uint64_t xr = x_st + (0 * kXTile + j * 2 * kXLbo) / 16;
                const uint64_t xi = x_st + (1 * kXTile + j * 2 * kXLbo) / 16;
                tc::mma_i8(d_re, ar, xr, idesc, !first);
                tc::mma_i8(d_re, an, xi, idesc, true);
                tc::mma_i8(d_im, ar, xi, idesc, !first);
                tc::mma_i8(d_im, ai, xr, idesc, true);
                first = false;
              }
              tc::commit(&sm.empty[st]);  // stage reusable once these MMAs have read it
              if (++st == kStages) {
                st = 0;
                ph ^= 1u;
              }
            }
          }
          tc::commit(&sm.acc_full[buf]);  // level complete
        }
      }
      tc::commit(&sm.done);
    }
    __syncwarp();
  } else {
    // ---- epilogue: warps 2..9; warp w reads TMEM lane quarter w % 4 and
    // column half (w - 2) / 4.  The W row values of a 16-column chunk are
    // loaded before the chunk's tensor-memory loads so both latencies overlap.
    const int e = warp - 2, q = warp & 3, half = e >> 2;
    const int row = q * 32 + lane;
    int lvl = 0;
    bool ok = true;
    for (int sg = seg0; sg < seg1; ++sg) {
      const MixSeg S = segs[sg];
      const MixGroup Gp = groups[S.g];
      const MixX X = xs[Gp.xid];
      long long prow = (long long)Gp.prow0 + (long long)S.rt * kM + row;
      if (!BGW_CHECKED(prow >= 0 && prow < n_arows, status, 53)) prow = 0;
      MixRow ar = arows[prow];
      if (!BGW_CHECKED((unsigned)ar.band < (unsigned)nb_w, status, 54)) ar.band = 0;
      const double2 *wrow = W + (size_t)ar.band * P;
      const double *sb = sB + X.sb_off + (size_t)S.w * x_rows_padded;
      const int c0 = half * (kN / 2);  // first tile column of this warp
      const int p0 = S.pt * kN + c0;
      double tr = 0.0, ti = 0.0;
      for (int li = 0; li < kLevels; ++li, ++lvl) {
        const int buf = lvl % kAccBufs;
        if (ok && !wait_or_flag(&sm.acc_full[buf], (lvl / kAccBufs) & 1, status)) ok = false;
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) continue;
        tc::fence_after();
        double vr = 0.0, vi = 0.0;
        const uint32_t tb = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * 2 * kN + c0);
        for (int cc = 0; cc < kN / 32; ++cc) {
          double2 w[16];
          double sc[16];
#pragma unroll
          for (int c = 0; c < 16; ++c) {
            const int p = min(p0 + cc * 16 + c, P - 1);
            w[c] = wrow[p];
            sc[c] = sb[p];
          }
          int32_t re[16], im[16];
          tc::ld16(tb + cc * 16, re);
          tc::ld16(tb + kN + cc * 16, im);
          tc::wait_ld();
#pragma unroll
          for (int c = 0; c < 16; ++c) {
            if (p0 + cc * 16 + c < P) {
              const double wr = w[c].x * sc[c], wi = w[c].y * sc[c];
              const double cr = (double)re[c], ci = (double)im[c];
              vr = fma(wr, cr, fma(-wi, ci, vr));
              vi = fma(wr, ci, fma(wi, cr, vi));
            }
          }
        }
        tc::fence_before();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&sm.acc_empty[buf]);
        const double lv = ldexp(1.0, -7 * (li + 2));
        tr = fma(vr, lv, tr);
        ti = fma(vi, lv, ti);
      }
      const double f = ar.coef * sA[(size_t)S.w * n_arows + prow];
      tr *= f;
      ti *= f;
      if (ROWS) {
        partials[(((size_t)sg * 2 + half) * kM + row) * 2 + 0] = tr;
        partials[(((size_t)sg * 2 + half) * kM + row) * 2 + 1] = ti;
        continue;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        tr += __shfl_xor_sync(0xffffffffu, tr, o);
        ti += __shfl_xor_sync(0xffffffffu, ti, o);
      }
      if (lane == 0) {
        sm.red[e][0] = tr;
        sm.red[e][1] = ti;
      }
      asm volatile("bar.sync 1, %0;" ::"n"(kEpiWarps * 32) : "memory");  // epilogue warps only
      if (e == 0 && lane == 0) {
        double pr = 0.0, pi = 0.0;
        for (int k = 0; k < kEpiWarps; ++k) {
          pr += sm.red[k][0];
          pi += sm.red[k][1];
        }
        partials[(size_t)sg * 2 + 0] = pr;
        partials[(size_t)sg * 2 + 1] = pi;
      }
      asm volatile("bar.sync 1, %0;" ::"n"(kEpiWarps * 32) : "memory");
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    // Every MMA has completed before the columns are released.
    if (lane == 0) (void)wait_or_flag(&sm.done, 0, status);
    __syncwarp();
    tc::fence_after();
    tc::dealloc(tmem, 512);
  }
}

// Sums every partial into its output in index order; writes achs, asx (nE)
// and cor (nE).  One block.
__global__ void __launch_bounds__(256)
    ff_mix_finalize_kernel(const double *__restrict__ partials, const int *__restrict__ out_of, int n, int nE,
                           double *__restrict__ achs, double *__restrict__ asx, double *__restrict__ cor) {
  __shared__ double red[8 * 6];
  __shared__ double res[6];
  double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int i = threadIdx.x; i < n; i += 256) {
    const int o = out_of[i];
    const double pr = partials[(size_t)i * 2], pi = partials[(size_t)i * 2 + 1];
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (o == k) {
        v[2 * k] += pr;
        v[2 * k + 1] += pi;
      }
  }
  block_sum<6, 256>(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) res[k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0 && achs) {
    achs[0] = res[0];
    achs[1] = res[1];
  }
  for (int i = threadIdx.x; i < nE; i += 256) {
    if (asx) {
      asx[2 * i] = res[2];
      asx[2 * i + 1] = res[3];
    }
    if (cor) {
      cor[2 * i] = res[4];
      cor[2 * i + 1] = res[5];
    }
  }
}

// Work split of the integer groups.  CTAs form teams of PT (one per
// kN-column tile); a team takes a contiguous, equal share of the (group,
// row tile, k block) units, cut into segments that never cross a row tile, a
// scale window or kMaxSegBlocks, and every member runs the same segments on
// its own column tile.  The members stream the same A digit tiles at the
// same time, so one of them reads them from DRAM and the others from L2.
void mix_segments(const std::vector<MixGroup> &mg, int PT, int KB, int sm_count, std::vector<MixSeg> *segs,
                  std::vector<int> *cta_seg) {
  long long units = 0;
  for (const auto &m : mg) units += (long long)m.row_tiles * KB;
  const int nteams = (int)std::max<long long>(1, std::min<long long>(std::max(1, sm_count / PT), units));
  const long long per = (units + nteams - 1) / nteams;
  std::vector<std::vector<MixSeg>> team(nteams);
  long long u = 0;  // first unit of the current row tile
  for (int g = 0; g < (int)mg.size(); ++g)
    for (int rt = 0; rt < mg[g].row_tiles; ++rt) {
      int kb = 0;
      while (kb < KB) {
        const long long t = std::min<long long>((u + kb) / per, nteams - 1);
        const long long team_end = (t + 1) * per;
        const int take = (int)std::min<long long>(
            {(long long)(KB - kb), std::max<long long>(1, team_end - (u + kb)),
             (long long)(kWinBlocks - kb % kWinBlocks), (long long)kMaxSegBlocks});
        MixSeg s;
        s.g = g;
        s.rt = rt;
        s.pt = 0;
        s.kb0 = kb;
        s.kb1 = kb + take;
        s.out = mg[g].out;
        s.w = kb / kWinBlocks;
        s.pad = 0;
        team[t].push_back(s);
        kb += take;
      }
      u += KB;
    }
  cta_seg->assign(1, 0);
  for (int t = 0; t < nteams; ++t) {
    if (team[t].empty()) continue;
    for (int pt = 0; pt < PT; ++pt) {
      for (MixSeg s : team[t]) {
        s.pt = pt;
        segs->push_back(s);
      }
      cta_seg->push_back((int)segs->size());
    }
  }
}

}  // namespace

int ff_enqueue_out_finalize(cudaStream_t stream, const double *partials, const int *out_of, int n, int nE,
                            double *achs, double *asx, double *cor) {
  ff_mix_finalize_kernel<<<1, 256, 0, stream>>>(partials, out_of, n, nE, achs, asx, cor);
  count_launch();
  BGW_CUDA_TRY(cudaGetLastError());
  return BGW_OK;
}

int ff_launch_mixed(CallEnv *env, const FFPlan &plan, int64_t nb, int64_t nb_w, int64_t nE, int64_t G, int64_t P,
                    const int32_t *inv, const int32_t *indinv, int64_t indinv_len, const double2 *am,
                    const double2 *an, const double *vc, const double2 *R, int r_f0, const double2 *A, int a_f0,
                    double *achs_dev, double *asx_dev, double *cor_dev) {
  (void)nb;
  Workspace *ws = env->ws;
  cudaStream_t stream = env->stream;
  double2 *W = nullptr;
  BGW_TRY(ff_build_w(env, nb_w, G, P, inv, indinv, indinv_len, am, vc, &W));

  // Integer slices for the big band groups; the small ones stay on the
  // FP64 tensor cores (per X element an integer group moves about 42 bytes
  // of digits, which pays off only when many rows share it).
  const int min_rows = (env->opt.flags & BGW_FLAG_FF_SLICE_ALL) ? kMixMinRowsAll : kMixMinRows;
  std::vector<FFGroup> small, big;
  for (const auto &g : plan.groups) (g.row_count < min_rows ? small : big).push_back(g);
  const int KB = (int)((G + kBK - 1) / kBK);
  const int NW = (KB + kWinBlocks - 1) / kWinBlocks;
  const int PT = (int)((P + kN - 1) / kN);
  const int x_rows_padded = PT * kN;

  // Distinct X slices, then packed layouts: X digits first, A digits after.
  std::map<std::pair<int, int>, int> xid_of;
  std::vector<MixX> xs;
  const size_t slice_elems = (size_t)P * (size_t)G;
  // Plain slices first, then the R - A differences (one slicing launch each).
  for (int pass = 0; pass < 2; ++pass)
    for (const auto &g : big) {
      if ((g.src == SRC_RA) != (pass == 1)) continue;
      const auto key = std::make_pair(g.src, g.f);
      if (xid_of.count(key)) continue;
      MixX x;
      x.b_off = 0;
      x.x0 = (g.src == SRC_A) ? A + (size_t)(g.f - a_f0) * slice_elems : R + (size_t)(g.f - r_f0) * slice_elems;
      x.x1 = (g.src == SRC_RA) ? A + (size_t)(g.f - a_f0) * slice_elems : nullptr;
      x.sb_off = (int)xs.size() * NW * x_rows_padded;
      x.pad = 0;
      xid_of[key] = (int)xs.size();
      xs.push_back(x);
    }
  long long off = 0;
  for (auto &x : xs) {
    x.b_off = off;
    off += (long long)kXPlanes * kS * PT * KB * kXTile;
  }
  std::vector<MixGroup> mg;
  std::vector<MixRow> arows;
  int prow = 0;
  for (const auto &g : big) {
    MixGroup m;
    m.xid = xid_of[std::make_pair(g.src, g.f)];
    m.out = g.out;
    m.prow0 = prow;
    m.row_tiles = (g.row_count + kM - 1) / kM;
    m.a_off = off;
    off += (long long)kAPlanes * kS * m.row_tiles * KB * kATile;
    for (int r = 0; r < m.row_tiles * kM; ++r) {
      MixRow mr;
      mr.g = (int)mg.size();
      mr.pad = 0;
      if (r < g.row_count) {
        const FFRow &fr = plan.rows[g.row_begin + r];
        mr.band = fr.band;
        mr.plan_row = g.row_begin + r;
        mr.coef = fr.coef;
      } else {
        mr.band = 0;
        mr.plan_row = -1;
        mr.coef = 0.0;
      }
      arows.push_back(mr);
    }
    prow += m.row_tiles * kM;
    mg.push_back(m);
  }

  // Segments of the integer groups, then FP64 tiles of the small groups.
  std::vector<MixSeg> segs;
  std::vector<int> cta_seg;
  if (!mg.empty()) mix_segments(mg, PT, KB, ws->sm_count, &segs, &cta_seg);
  const int nctas = segs.empty() ? 0 : (int)cta_seg.size() - 1;
  std::vector<FFTile> ft;
  if (!small.empty()) {
    int per_sm = 1;
    BGW_TRY(ff_fp64_per_sm(&per_sm));
    ff_fp64_tiles(small, P, G, 2 * ws->sm_count * std::max(per_sm, 1), &ft);
  }
  const int nft = (int)ft.size(), nseg = (int)segs.size();
  // Partials: one per FP64 tile then one per segment; with distinct outputs
  // per iw, one per FP64 tile row then one per (segment, column half, row).
  const bool per_row = plan.per_iw;
  std::vector<int> out_of;  // per_row: plan row of each partial, else its output
  if (per_row) {
    ff_fp64_row_ids(ft, &out_of);
    for (int i = 0; i < nseg; ++i)
      for (int h = 0; h < 2; ++h)
        for (int r = 0; r < kM; ++r)
          out_of.push_back(arows[(size_t)mg[segs[i].g].prow0 + (size_t)segs[i].rt * kM + r].plan_row);
  } else {
    out_of.resize(nft + nseg);
    for (int i = 0; i < nft; ++i) out_of[i] = ft[i].out;
    for (int i = 0; i < nseg; ++i) out_of[nft + i] = segs[i].out;
  }
  const size_t n_part = out_of.size();
  const size_t seg_part0 = per_row ? (size_t)nft * ff_fp64_tile_rows() : (size_t)nft;  // first segment partial

  // Device buffers: packed digits (TABLE0); plan arrays and row scales in
  // one upload (PLAN).
  void *pack = nullptr, *small_buf = nullptr, *partials = nullptr;
  BGW_TRY(ws_reserve(ws, SLOT_TABLE0, (size_t)std::max<long long>(off, 256), &pack));
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_rows = 0;
  const size_t o_mg = o_rows + al(sizeof(FFRow) * std::max<size_t>(plan.rows.size(), 1));
  const size_t o_ft = o_mg + al(sizeof(MixGroup) * std::max<size_t>(mg.size(), 1));
  const size_t o_seg = o_ft + al(sizeof(FFTile) * std::max(nft, 1));
  const size_t o_cta = o_seg + al(sizeof(MixSeg) * std::max(nseg, 1));
  const size_t o_xs = o_cta + al(sizeof(int) * std::max<size_t>(cta_seg.size(), 1));
  const size_t o_ar = o_xs + al(sizeof(MixX) * std::max<size_t>(xs.size(), 1));
  const size_t o_out = o_ar + al(sizeof(MixRow) * std::max<size_t>(arows.size(), 1));
  const size_t o_sa = o_out + al(sizeof(int) * std::max<size_t>(n_part, 1));
  const size_t o_sb = o_sa + al(sizeof(double) * std::max<size_t>(arows.size() * (size_t)NW, 1));
  const size_t total = o_sb + al(sizeof(double) * std::max<size_t>(xs.size() * (size_t)NW * x_rows_padded, 1));
  std::vector<unsigned char> host(total, 0);
  auto put = [&](size_t o, const void *src, size_t bytes) {
    if (bytes) std::memcpy(host.data() + o, src, bytes);
  };
  put(o_rows, plan.rows.data(), sizeof(FFRow) * plan.rows.size());
  put(o_mg, mg.data(), sizeof(MixGroup) * mg.size());
  put(o_ft, ft.data(), sizeof(FFTile) * nft);
  put(o_seg, segs.data(), sizeof(MixSeg) * nseg);
  put(o_cta, cta_seg.data(), sizeof(int) * cta_seg.size());
  put(o_xs, xs.data(), sizeof(MixX) * xs.size());
  put(o_ar, arows.data(), sizeof(MixRow) * arows.size());
  put(o_out, out_of.data(), sizeof(int) * n_part);
  BGW_TRY(ws_reserve(ws, SLOT_PLAN, total, &small_buf));
  BGW_CUDA_TRY(cudaMemcpyAsync(small_buf, host.data(), total, cudaMemcpyHostToDevice, stream));
  unsigned char *sb = static_cast<unsigned char *>(small_buf);
  BGW_TRY(ws_reserve(ws, SLOT_PARTIALS, sizeof(double) * 2 * std::max<size_t>(n_part, 1), &partials));
  double *part = static_cast<double *>(partials);

  BGW_TRY(prof_mark(env, 1));
  const uint64_t launches_before = g_launches.load();
  if (nctas > 0) {
    const MixGroup *d_mg = (const MixGroup *)(sb + o_mg);
    const MixRow *d_ar = (const MixRow *)(sb + o_ar);
    const MixX *d_xs = (const MixX *)(sb + o_xs);
    double *d_sa = (double *)(sb + o_sa), *d_sb = (double *)(sb + o_sb);
    const int na = (int)arows.size();
    ff_slice_kernel<0><<<(unsigned)((size_t)na * NW), kSliceThreads, 0, stream>>>(
        d_mg, d_ar, d_xs, na, x_rows_padded, (int)P, (int)G, KB, NW, an, (int8_t *)pack, d_sa, d_sb, off,
        env->d_status);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
    // X slices: xs holds the plain ones first, then the differences.
    int n_plain = 0;
    while (n_plain < (int)xs.size() && xs[n_plain].x1 == nullptr) ++n_plain;
    for (int sub = 0; sub < 2; ++sub) {
      const int x0 = sub ? n_plain : 0, x1 = sub ? (int)xs.size() : n_plain;
      if (x1 <= x0) continue;
      const unsigned grid = (unsigned)((size_t)(x1 - x0) * x_rows_padded * NW);
      const MixX *d_x = d_xs + x0;
      if (sub)
        ff_slice_kernel<2><<<grid, kSliceThreads, 0, stream>>>(d_mg, d_ar, d_x, na, x_rows_padded, (int)P, (int)G,
                                                              KB, NW, an, (int8_t *)pack, d_sa, d_sb, off,
                                                              env->d_status);
      else
        ff_slice_kernel<1><<<grid, kSliceThreads, 0, stream>>>(d_mg, d_ar, d_x, na, x_rows_padded, (int)P, (int)G,
                                                              KB, NW, an, (int8_t *)pack, d_sa, d_sb, off,
                                                              env->d_status);
      count_launch();
      BGW_CUDA_TRY(cudaGetLastError());
    }
    const int smem = (int)sizeof(MixSmem);
    auto gemm = per_row ? ff_mix_gemm_kernel<true> : ff_mix_gemm_kernel<false>;
    BGW_CUDA_TRY(cudaFuncSetAttribute(gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    gemm<<<nctas, kMixThreads, smem, stream>>>(
        (const MixSeg *)(sb + o_seg), (const int *)(sb + o_cta), d_mg, d_ar, d_xs, (const int8_t *)pack, d_sa, d_sb,
        na, x_rows_padded, W, (int)P, KB, PT, part + 2 * seg_part0, env->d_status, off, (int)nb_w);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
  }
  BGW_TRY(ff_launch_fp64_tiles(stream, (const FFTile *)(sb + o_ft), nft, (const FFRow *)(sb + o_rows),
                               (int)plan.rows.size(), nb_w, P, G, an, R, r_f0, A, a_f0, W, part, env->d_status,
                               per_row));
  BGW_TRY(prof_mark(env, 2));
  if (per_row) {
    FFTermTables tt;
    ff_build_term_tables(plan, out_of, nE, &tt);
    BGW_TRY(ff_launch_term_finalize(env, SLOT_TABLE1, tt, part, nE, achs_dev, asx_dev, cor_dev));
  } else {
    ff_mix_finalize_kernel<<<1, 256, 0, stream>>>(part, (const int *)(sb + o_out), (int)n_part, (int)nE, achs_dev,
                                                  asx_dev, cor_dev);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
  }
  {
    // Useful work as in the FP64 path; bytes = the packed digits written
    // once and the operands read once.
    double slices = 0.0;
    for (const auto &b : plan.slice_reads) slices += b;
    env->prof.flops = 8.0 * plan.useful_cmacs;
    env->prof.main_bytes = slices * 16.0 * (double)P * (double)G + 16.0 * (double)nb_w * (double)G + (double)off;
    env->prof.main_launches = (int)(g_launches.load() - launches_before);
    std::snprintf(env->prof.main_kernel, sizeof(env->prof.main_kernel), "ff_mix_gemm_kernel");
  }
  // The pageable plan buffer must outlive its (staged) upload.
  BGW_CUDA_TRY(cudaStreamSynchronize(stream));
  return BGW_OK;
}

}  // namespace bgw
