// ff_fused.cu -- mixed-precision FF sums with the digit split fused into the
// tensor-core kernel (tcgen05.mma kind::i8, integer Ozaki scheme, FP64
// recombination; ff_mixed.cu holds the staged form, which cuts both
// operands into digit buffers first).
//
// Roles.  A unit of work is (band-row chunk, 128 G' columns p, k range of
// one 4096-k window).  The MMA's M side is the frequency slice tile X[p][k]
// (I_epsR, I_epsA or their difference, 128 rows), its N side the chunk's
// band rows a = aqsn[band][k] with real and imaginary parts stacked:
//   D = Xr [ar; ai]^T + Xi [-ai; ar]^T  =  [Re(X a^T) | Im(X a^T)],
// two real products per digit pair, N0 = 2 * rows columns per level.  A
// chunk holds at most 48 rows, so the five level accumulators (L = 2..6,
// 15 digit pairs) take 5 N0 <= 480 of the 512 tensor-memory columns and
// stay resident for the whole unit.  The band digits of a stage are stored
// as two stacks over the digit index t, Sr = [ar_t; ai_t]_t and
// Si = [-ai_t; ar_t]_t, and the accumulator of level s + t + 2 sits at
// columns (s + t) N0, so X digit s meets every band digit t <= 4 - s in one
// MMA over (5 - s) N0 columns (split at 256): 16 MMAs per 32-k stage.
//
// Digits.  A value x with |x| < 2^E becomes T = floor(x 2^(38 - E)),
// |T| < 2^38, written as five balanced signed bytes d_0..d_4 (most
// significant first), T = sum_s d_s 256^(4 - s), d_s in [-128, 127]: one
// FP64 add rounded toward zero, r = (1.5 2^52 + C) + x 2^(38 - E) with
// C = 0x80808080, leaves u = T + C in the low 40 bits of r; the low four
// bytes of u minus 128 (byte ^ 0x80) are d_4..d_1 and its signed top byte
// is d_0.  So x = 2^(E + 2) sum_s d_s 256^-(s + 1) up to 2^(E - 38), and a
// product of digit levels s + t + 2 = L carries the weight 256^-L.  Every
// digit product is exact in int32 (|C_L| <= 5 pairs x 2 x 4096 x 2^14).
//
// Split.  The band rows are cut by ff_bslice_kernel (exact per-window row
// scale, the two stacks in the canonical K-major layout, one contiguous
// block per (chunk, 32-k stage)).  The X tile is cut inside the
// kernel: its FP64 values are read once from HBM by the converter warps,
// scaled per row p by 2^-E(p) and written as 10 digit planes (Re, Im x 5)
// straight into the stage buffer.  E(p) comes from the unit's first 32-k
// block (largest |re|, |im|, one bit of headroom), so the tile is read in a
// single pass.  A later value at or above 2^E(p) (or a nonzero value in a
// row whose first block is zero, or a NaN) does not fit the digits: the
// unit then reports itself in unit_flag, writes a zero partial, and gated
// FP64 tiles of ff.cu recompute exactly that unit (they write zero for
// every unit that did not flag).  The result is complete either way and
// reductions are in fixed orders (bitwise reproducible).
//
// k order.  Inside each 32-k stage both operands store the digit of stage
// position k at byte 4 (k mod 8) + k / 8 of the stage's K extent (the sum
// over k does not depend on its order): a converter lane then loads
// k = q + 8 e (e < 4), so every 16-byte load instruction of a warp covers
// four whole 128-byte lines, and still writes its four digits as one word.
//
// Warps: 0 is the producer (band-row digit blocks by 1-D bulk copies into a
// 3-stage ring; in a 2-CTA pair also this CTA's converted half to the
// peer), 1 issues the MMAs, 2-17 convert X; after the last stage warps 2-9
// read the accumulators (tcgen05.ld), fold W(band, p) and the scales, and
// reduce one partial per unit (or per row slot).  Every mbarrier wait is
// bounded.  The grid is made of 2-CTA clusters (kFPair, see ff_fuse_kernel).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "bgw_internal.cuh"
#include "ff_plan.cuh"
#include "tcgen05.cuh"

namespace bgw {
namespace {

constexpr int kFS = 5;                                 // digits per operand (8 bits each)
constexpr int kFM = 128;                               // G' columns per unit (MMA M)
constexpr int kFK = 32;                                // k per stage (one kind::i8 MMA)
constexpr int kFStages = 3;
constexpr int kFMaxRows = 48;                          // band rows per chunk (N = 2 rows)
constexpr int kFWin = 4096;                            // k per unit; band-row scale window
constexpr int kFConvWarps = 16;                        // per stage: 1 task (4 rows x 32 k) each in a pair
constexpr int kFEpiWarps = 8;                          // two per TMEM lane quarter
constexpr int kFConv = 32 * kFConvWarps;               // converter threads
constexpr int kFThreads = 64 + kFConv;
// One digit plane of the X tile: two 16-k column groups of 128 rows x 16
// bytes, the second kFXLbo bytes after the first (2048 + 64: the two groups
// fall on different shared-memory banks, so a warp's stores of 4 rows x 32
// k do not conflict).
constexpr int kFXLbo = kFM * 16 + 64;
constexpr int kFXPlane = kFXLbo + kFM * 16;
constexpr int kFXStage = 2 * kFS * kFXPlane;           // Re digits 0-4, Im digits 0-4
constexpr int kFBStageMax = 2 * kFS * 2 * kFMaxRows * kFK;  // stacks Sr, Si x digits x 2 rows x k
constexpr int kFHeadroom = 1;                          // bits above the first block's largest value
constexpr int kFBThreads = 256;                        // band-row slicing
constexpr int kFuseMinRows = 8;                        // default: smaller groups stay FP64
// 2-CTA clusters share the slice conversion (false: each CTA converts its
// whole tile, 2 tasks per converter warp; the measured default is true).
constexpr bool kFPair = true;
static_assert(kFBThreads == 256, "band-row slicing: 8 warps, one per row slot of a group");
static_assert((kFM / 4) % (2 * kFConvWarps) == 0, "every converter warp takes the same tasks per stage");
constexpr int kFTasks = (kFM / 4) / kFConvWarps;  // tasks (4 rows x 32 k) per converter warp and stage
static_assert(kFS * 2 * kFMaxRows <= 512, "the level accumulators fit in tensor memory");
static_assert(kFMaxRows % 8 == 0, "chunks are whole 8-row core-matrix groups");
static_assert(kFWin % kFK == 0, "a unit is a whole number of stages");
// |C_L| <= (pairs per level) x 2 products x kFWin x 128^2 < 2^31.
static_assert((long long)kFS * 2 * kFWin * 128 * 128 < (1LL << 31), "int32 accumulators cannot overflow");
constexpr double kFMagic = 6755399441055744.0 + 2155905152.0;  // 1.5 2^52 + 0x80808080

struct FuseChunk {        // up to kFMaxRows rows of one band group
  long long b_off;        // byte offset of its packed band-row digits
  const double2 *x0;      // frequency slice [P][G]
  const double2 *x1;      // subtrahend (R - A) or null
  int slot0;              // first row slot
  int nrp;                // row slots (multiple of 8)
  int out, pad;
};
struct FuseRow {          // row slot
  int band, chunk;
  double coef;            // 0 for padding slots
};
struct FuseUnit {         // columns [kFM pt, kFM pt + kFM) x k [k0, k1) of a chunk
  int chunk, pt, k0, k1;
  int phantom;            // pair member without rows: converts its half of the tile only
  int pad;
};

struct __align__(128) FuseSmem {
  int8_t x[kFStages][kFXStage];
  int8_t b[kFStages][kFBStageMax];
  uint64_t bfull[kFStages], xfull[kFStages], empty[kFStages], done;
  uint64_t xlocal[kFStages];  // a pair: this CTA's half of the stage is written
  uint64_t never;             // stall injection: nothing arrives on it
  uint32_t tmem;
  int ovf;                // a value of this CTA's rows did not fit
  int ovf_peer;           // ... of the peer's rows (written by the peer)
  int nrecv;              // stages whose half the peer sent (written by the peer)
  double mult[kFM];       // 2^(38 - E(p))
  double lim[kFM];        // values with |x| >= lim do not fit the digits
  int ex[kFM];            // E(p)
  double rmax[kFM];       // first block: largest |re|, |im| per row
  double red[4][kFMaxRows][2];
};

// mbarrier wait that lets the hardware suspend the thread (up to the hint)
// instead of spinning, so waiting threads leave the issue slots to the
// converters.  Bounded: BGW_ERR_TIMEOUT after kWaitCycles.
constexpr uint32_t kSuspendNs = 10000;
// (Acquire at cluster scope: in 2-CTA pairs the peer's copies and MMA
// commits complete these phases.)
__device__ __forceinline__ bool try_wait_sleep(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool fwait(uint64_t *bar, uint32_t parity, int *status,
                                      long long budget = kWaitCycles) {
  if (try_wait_sleep(bar, parity)) return true;
  const long long t0 = clock64();
  while (!try_wait_sleep(bar, parity)) {
    if (clock64() - t0 > budget) {
      raise_status(status, BGW_ERR_TIMEOUT, (int)blockIdx.x);
      return false;
    }
  }
  return true;
}
// L2 prefetch of the 128-byte line holding p (no register cost).
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
constexpr int kFPrefetch = 3;  // stages the L2 prefetch runs ahead of the conversion
// 2-CTA clusters: rank, peer shared-memory addresses, cluster barrier,
// shared -> peer shared bulk copies completing on the peer's mbarrier, and
// the MMA commit that arrives on the same mbarrier in both CTAs.
__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t peer_addr(const void *p, uint32_t rank) {
  uint32_t a;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
  return a;
}
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void bulk_s2peer(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst),
               "r"(smem_u32(src)), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void st_peer(uint32_t addr, int v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}
__device__ __forceinline__ void commit_pair(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
          smem_u32(bar)),
      "h"((uint16_t)3)
      : "memory");
}
// Non-coherent 16-byte global load kept where it is written (asm volatile),
// so loads issued a stage ahead stay a stage ahead.
__device__ __forceinline__ double2 ld_nc(const double2 *p) {
  double2 v;
  asm volatile("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}
__device__ __forceinline__ void conv_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kFConv) : "memory"); }


// The kFS digits of four values c_e (see the file comment), mult = 2^(38 -
// E): word s holds value e's digit s in byte e.  Values with |c| >= lim (or
// NaN) set `ovf` (their digits are meaningless; the unit is recomputed).
__device__ __forceinline__ void digits4(const double (&c)[4], double mult, double lim, bool &ovf,
                                        uint32_t (&w)[kFS]) {
  uint32_t lo[4], hi[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    ovf |= !(fabs(c[e]) < lim);
    const double r = __dadd_rz(c[e] * mult, kFMagic);
    lo[e] = (uint32_t)__double2loint(r);
    hi[e] = (uint32_t)__double2hiint(r);
  }
  // 4 x 4 byte transpose of the low words; digit 0 from byte 0 of the high words.
  const uint32_t a01l = __byte_perm(lo[0], lo[1], 0x5140), a01h = __byte_perm(lo[0], lo[1], 0x7362);
  const uint32_t a23l = __byte_perm(lo[2], lo[3], 0x5140), a23h = __byte_perm(lo[2], lo[3], 0x7362);
  w[4] = __byte_perm(a01l, a23l, 0x5410) ^ 0x80808080u;
  w[3] = __byte_perm(a01l, a23l, 0x7632) ^ 0x80808080u;
  w[2] = __byte_perm(a01h, a23h, 0x5410) ^ 0x80808080u;
  w[1] = __byte_perm(a01h, a23h, 0x7632) ^ 0x80808080u;
  w[0] = __byte_perm(__byte_perm(hi[0], hi[1], 0x0040), __byte_perm(hi[2], hi[3], 0x0040), 0x5410);
}

// One CTA per (chunk, kFWin-k window, group of 8 row slots), 8 warps.
// Pass 1: warp r reads row slot r's window of aqsn[band] (coalesced) and its
// largest |re| / |im| m < 2^e gives the digit scale (2^(e + 2) to
// sB[slot][w]; NaN when the window holds a non-finite value).  Pass 2 (the
// window again, from L2): warp w takes the stages w, w + 8, ...; lane ->
// (row r = lane / 4, u = lane % 4) writes stage positions [8u, 8u + 8)
// (position 4 q + e holds stage k = q + 8 e, so byte 4 hq + e of its 8
// takes k = 2u + hq + 8 e) of its row in every digit plane: stack Sr (row
// 2 nrp t + slot: ar digit t; row 2 nrp t + nrp + slot: ai digit t), then
// stack Si (-ai, ar), each 10 nrp rows x 32 k in the canonical K-major
// layout (core matrices of 8 rows x 16 bytes; 16-k column groups 10 nrp x
// 16 bytes apart).  A warp's 8-byte stores of one plane cover two whole
// 128-byte lines.  Padding slots and k >= G are written as zero digits.
struct BSliceTask {  // (chunk, group of 8 row slots)
  int chunk, group;
};
__global__ void __launch_bounds__(kFBThreads)
    ff_bslice_kernel(const BSliceTask *__restrict__ tasks, const FuseRow *__restrict__ frows,
                     const FuseChunk *__restrict__ chunks, int NW, int G, int KB, const double2 *__restrict__ aqsn,
                     int nb, int8_t *__restrict__ pack, long long pack_bytes, double *__restrict__ sB, int *status) {
  __shared__ double s_mult[8];
  __shared__ int s_bad[8];
  const int w = (int)(blockIdx.x % NW);
  const BSliceTask T = tasks[blockIdx.x / NW];
  const FuseChunk C = chunks[T.chunk];
  const int nrp = C.nrp, warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
  const int kw = w * kFWin, kend = min(G, kw + kFWin);
  // ---- pass 1: row slot 8 group + warp.
  {
    const int slot = C.slot0 + 8 * T.group + warp;
    const FuseRow fr = frows[slot];
    bool valid = fr.coef != 0.0;
    if (!BGW_CHECKED(!valid || (unsigned)fr.band < (unsigned)nb, status, 63)) valid = false;
    double m = 0.0;
    int nonfinite = 0;
    if (valid) {
      const double2 *src = aqsn + (size_t)fr.band * (size_t)G;
      for (int k = kw + lane; k < kend; k += 32) {
        const double2 x = src[k];
        const double a = fmax(fabs(x.x), fabs(x.y));
        nonfinite |= !(a <= DBL_MAX);
        m = fmax(m, a);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      nonfinite |= __shfl_xor_sync(0xffffffffu, nonfinite, o);
    }
    int e = 0;
    if (m > 0.0 && !nonfinite) (void)frexp(m, &e);
    e = max(e, -960);  // keeps 2^(38 - e) finite; values below 2^-960 lose precision
    if (lane == 0) {
      sB[(size_t)slot * NW + w] = nonfinite ? __longlong_as_double(0x7ff8000000000000LL) : ldexp(1.0, e + 2);
      s_mult[warp] = ldexp(1.0, 38 - e);
      s_bad[warp] = (!valid || nonfinite) ? 1 : 0;
    }
  }
  __syncthreads();
  // ---- pass 2.
  const int r = lane >> 2, u = lane & 3;
  const int rs = 8 * T.group + r;  // row slot within the chunk
  const FuseRow fr = frows[C.slot0 + rs];
  const bool zero = s_bad[r] != 0;
  const double mult = s_mult[r];
  const double2 *src = aqsn + (size_t)(zero ? 0 : fr.band) * (size_t)G;
  const int srows = kFS * 2 * nrp;
  const long long stack = (long long)srows * kFK;  // bytes of one stack
  const int nstages = (kend - kw + kFK - 1) / kFK;
  for (int sl = warp; sl < nstages; sl += kFBThreads / 32) {
    const int kb = kw / kFK + sl;
    if (kb >= KB) break;
    const int k0 = kb * kFK;
    uint32_t wr[kFS][2], wi[kFS][2], wn[kFS][2];
    bool ovf = false;
#pragma unroll
    for (int hq = 0; hq < 2; ++hq) {
      double cr[4], ci[4], cn[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + 2 * u + hq + 8 * j;
        double2 v = make_double2(0.0, 0.0);
        if (!zero && k < G) v = src[k];
        cr[j] = v.x;
        ci[j] = v.y;
        cn[j] = -v.y;
      }
      uint32_t a[kFS], b[kFS], c[kFS];
      digits4(cr, mult, INFINITY, ovf, a);
      digits4(ci, mult, INFINITY, ovf, b);
      digits4(cn, mult, INFINITY, ovf, c);
#pragma unroll
      for (int t = 0; t < kFS; ++t) {
        wr[t][hq] = a[t];
        wi[t][hq] = b[t];
        wn[t][hq] = c[t];
      }
    }
    const int kk = 8 * u;  // stage position of this lane's first byte
    const long long base = C.b_off + (long long)kb * 2 * stack;
    auto off = [&](int row) {
      return (long long)((kk >> 4) * (srows * 16) + (row >> 3) * 128 + (row & 7) * 16 + (kk & 15));
    };
    // Debug build: the stage's block lies in the packed buffer.
    if (!BGW_CHECKED(base >= 0 && base + 2 * stack <= pack_bytes, status, 64)) break;
    int8_t *sr = pack + base, *si = pack + base + stack;
#pragma unroll
    for (int t = 0; t < kFS; ++t) {
      const int r0 = 2 * nrp * t + rs, r1 = r0 + nrp;
      *reinterpret_cast<uint2 *>(sr + off(r0)) = make_uint2(wr[t][0], wr[t][1]);
      *reinterpret_cast<uint2 *>(sr + off(r1)) = make_uint2(wi[t][0], wi[t][1]);
      *reinterpret_cast<uint2 *>(si + off(r0)) = make_uint2(wn[t][0], wn[t][1]);
      *reinterpret_cast<uint2 *>(si + off(r1)) = make_uint2(wr[t][0], wr[t][1]);
    }
  }
}

// PAIR: the grid is made of 2-CTA clusters; the two CTAs hold two chunks
// (or one chunk and a phantom) of the same X tile and k range.  Each
// converts half of the tile's 128 rows (CTA rank r: rows [64 r, 64 r + 64))
// into its own stage buffer; once the half is written (xlocal), the
// producer thread sends it to the peer's buffer with 20 bulk copies (one
// per plane and 16-k column group) that complete on the peer's xfull
// barrier, whose phase also waits for the peer's own half.  Each CTA's MMA
// commit arrives on the empty barrier of both, so neither overwrites a
// stage the other still reads.
template <bool PAIR>
__global__ void __launch_bounds__(kFThreads, 1)
    ff_fuse_kernel(const FuseUnit *__restrict__ units, const FuseChunk *__restrict__ chunks,
                   const FuseRow *__restrict__ frows, int n_slots, const int8_t *__restrict__ pack,
                   long long pack_bytes, const double *__restrict__ sB, int NW, const double2 *__restrict__ W, int P,
                   int G, int nb_w, double *__restrict__ partials, int *__restrict__ unit_flag, int per_row,
                   int *status, long long stall) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  FuseSmem &sm = *reinterpret_cast<FuseSmem *>(smem_raw);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t rank = PAIR ? cluster_rank() : 0u, peer = rank ^ 1u;
  const FuseUnit U = units[blockIdx.x];
  const FuseChunk C = chunks[U.chunk];
  const bool phantom = PAIR && U.phantom != 0;
  const int nrp = phantom ? 0 : C.nrp;
  // Debug build: the chunk's shape and the unit's k range (a failing unit
  // does no work and contributes zero).
  const bool good = BGW_CHECKED((phantom || (nrp >= 8 && nrp <= kFMaxRows && nrp % 8 == 0)) && U.k0 >= 0 &&
                                    U.k1 > U.k0 && U.k1 <= G && U.k1 - U.k0 <= kFWin && U.k0 % kFWin == 0 &&
                                    C.slot0 >= 0 && C.slot0 + nrp <= n_slots && U.pt >= 0 && U.pt * kFM < P,
                                status, 61);
  const int N = 2 * nrp;
  const int ns = good ? (U.k1 - U.k0 + kFK - 1) / kFK : 0;  // stages
  const int kb0 = U.k0 / kFK;
  const uint32_t bbytes = (uint32_t)(2 * kFS * N * kFK);  // stacks Sr and Si
  constexpr int kT = PAIR ? kFTasks / 2 : kFTasks;         // conversion tasks per warp and stage
  // Stall injection (bgw_debug_inject_stall): at CTA-local stage `stall` the
  // MMA thread waits on `never` and gives up; every other wait then has the
  // short budget, so the timeout reaches the rest of the CTA (and of its
  // pair) within milliseconds, along the same path as a real timeout.
  const long long budget = stall >= 0 ? kStallCycles : kWaitCycles;
  constexpr uint32_t kHalf = 2 * kFS * 2 * (kFM / 2) * 16;  // bytes of half the rows of a stage

  if (threadIdx.x == 0) {
    for (int i = 0; i < kFStages; ++i) {
      mbar_init(&sm.bfull[i], 1);
      mbar_init(&sm.xfull[i], PAIR ? 1 : kFConv);
      mbar_init(&sm.xlocal[i], kFConv);
      mbar_init(&sm.empty[i], PAIR ? 2 : 1);
    }
    mbar_init(&sm.done, 1);
    mbar_init(&sm.never, 1);
    sm.ovf = 0;
    sm.ovf_peer = 0;
    sm.nrecv = 0;
    fence_mbar_init();
  }
  __syncwarp();
  if (warp == 0) {
    tc::alloc(&sm.tmem, 512);
    tc::relinquish();
  }
  tc::fence_before();
  __syncthreads();
  if (PAIR) cluster_sync();  // both CTAs' barriers exist before any remote arrive or copy
  tc::fence_after();
  const uint32_t tmem = sm.tmem;

  if (warp == 0) {
    // ---- producer: the band-row digits (one bulk copy per stage, lane 0)
    // and, in a pair, this CTA's half of each converted stage to the peer
    // (20 copies, one per lane: issued one after the other they took longer
    // than the stage's MMAs).
    int issued = 0, nsent = 0;
    for (int j = 0; j < ns; ++j) {
      const int st = j % kFStages;
      int ok = 1;
      if (lane == 0) {
        if (j >= kFStages && !fwait(&sm.empty[st], ((j / kFStages) - 1) & 1, status, budget)) {
          ok = 0;
        } else if (!phantom) {
          const int8_t *src = pack + C.b_off + (long long)(kb0 + j) * bbytes;
          // Debug build: the block lies in the packed buffer.
          if (!BGW_CHECKED(src >= pack && src + bbytes <= pack + pack_bytes, status, 62)) {
            ok = 0;
          } else {
            mbar_expect_tx(&sm.bfull[st], bbytes);
            bulk_g2s(sm.b[st], src, bbytes, &sm.bfull[st]);
            issued = j + 1;
          }
        }
      }
      if (PAIR) {
        // Every lane sees this CTA's half written (acquire) before its copy.
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (ok && !fwait(&sm.xlocal[st], (j / kFStages) & 1, status, budget)) ok = 0;
        ok = __all_sync(0xffffffffu, ok);
        if (!ok) break;
        // This CTA's arrival on xfull, expecting the peer's half as bytes.
        if (lane == 0) mbar_expect_tx(&sm.xfull[st], kHalf);
        if (lane < 2 * 2 * kFS) {
          const int pl = lane >> 1, kg = lane & 1;
          const int8_t *hs = &sm.x[st][pl * kFXPlane + kg * kFXLbo + rank * (kFM / 2) * 16];
          bulk_s2peer(peer_addr(hs, peer), hs, (kFM / 2) * 16, peer_addr(&sm.xfull[st], peer));
        }
        nsent = j + 1;
      } else {
        ok = __shfl_sync(0xffffffffu, ok, 0);
        if (!ok) break;
      }
    }
    if (lane == 0) {
      // Copies still in flight (error paths only) land before the CTA exits.
      for (int t = 0; t < kFStages; ++t) {
        if (issued <= t) continue;
        const int last = (issued - 1) - ((issued - 1 - t) % kFStages);
        (void)fwait(&sm.bfull[t], (last / kFStages) & 1, status, budget);
      }
      // The peer drains the stages sent to it before it exits.
      if (PAIR) st_peer(peer_addr(&sm.nrecv, peer), nsent);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---- MMA issuer: per stage and X digit s, the digits t <= kFS - 1 - s
    // of both stacks in MMAs of at most 256 columns into the resident level
    // accumulators (level s + t + 2 at columns (s + t) N).  At stage 0 the
    // s = 0 products, which cover every column, start the accumulators.
    if (lane == 0) {
      const uint32_t xbase = smem_u32(&sm.x[0][0]), bbase = smem_u32(&sm.b[0][0]);
      const uint32_t srows = (uint32_t)(kFS * N), slbo = srows * 16, sbytes = srows * kFK;
      for (int j = 0; j < ns; ++j) {
        const int st = j % kFStages;
        const uint32_t par = (uint32_t)((j / kFStages) & 1);
        if (j == stall && !fwait(&sm.never, 0, status, kStallCycles)) break;
        if ((!phantom && !fwait(&sm.bfull[st], par, status, budget)) || !fwait(&sm.xfull[st], par, status, budget)) break;
        tc::fence_after();
        if (!phantom) {
          const uint32_t xs = xbase + (uint32_t)(st * kFXStage), bs = bbase + (uint32_t)(st * kFBStageMax);
#pragma unroll 1
          for (int s = 0; s < kFS; ++s) {
            const uint64_t xr = tc::smem_desc(xs + (uint32_t)(s * kFXPlane), kFXLbo, 128);
            const uint64_t xi = tc::smem_desc(xs + (uint32_t)((kFS + s) * kFXPlane), kFXLbo, 128);
            const uint32_t ncol = (uint32_t)((kFS - s) * N);
            for (uint32_t c0 = 0; c0 < ncol; c0 += 256) {
              const uint32_t n = min(256u, ncol - c0);
              const uint32_t idesc = tc::idesc_i8(kFM, (int)n);
              const uint32_t d = tmem + (uint32_t)(s * N) + c0;
              const uint64_t br = tc::smem_desc(bs + (c0 / 8) * 128, slbo, 128);
              const uint64_t bi = tc::smem_desc(bs + sbytes + (c0 / 8) * 128, slbo, 128);
              tc::mma_i8(d, xr, br, idesc, j > 0 || s > 0);
              tc::mma_i8(d, xi, bi, idesc, true);
            }
          }
        }
        // Stage reusable once these MMAs (and, in a pair, the peer's) have read it.
        if (PAIR)
          commit_pair(&sm.empty[st]);
        else
          tc::commit(&sm.empty[st]);
      }
      tc::commit(&sm.done);
    }
    __syncwarp();
  } else {
    // ---- converters.  Conversion task (4 rows x 32 k): lane -> row
    // base + lane / 8 and stage k q8 + 8 e (q8 = lane % 8, e < 4), digit
    // word at stage position 4 q8.
    const int cw = warp - 2, ct = (int)threadIdx.x - 64;
    const int q8 = lane & 7, r4 = lane >> 3;
    const double2 *x0 = C.x0, *x1 = C.x1;
    const int p_base = U.pt * kFM;
    // Rows of this CTA's task i (a pair's CTA converts its half of the tile).
    auto task_row = [&](int i) { return (int)(PAIR ? rank * (kFM / 2) : 0) + (cw + kFConvWarps * i) * 4 + r4; };
    // Stages whose k range lies inside [k0, k1) of a column tile inside
    // [0, P) take the fast path (no clamping, no zeroing); the edges load
    // from clamped addresses and zero the values outside.
    const bool rows_inside = p_base + kFM <= P;
    auto inside = [&](int j) { return rows_inside && U.k0 + (j + 1) * kFK <= U.k1; };
    auto issue = [&](double2 (&a)[4], double2 (&b)[4], int j, int row) {
      const int k = U.k0 + j * kFK + q8;
      if (inside(j)) {
        const size_t o = (size_t)(p_base + row) * (size_t)G + (size_t)k;
#pragma unroll
        for (int e = 0; e < 4; ++e) a[e] = ld_nc(x0 + o + 8 * e);
        if (x1)
#pragma unroll
          for (int e = 0; e < 4; ++e) b[e] = ld_nc(x1 + o + 8 * e);
        return;
      }
      const int p = min(p_base + row, P - 1);
      const double2 *pa = x0 + (size_t)p * (size_t)G;
#pragma unroll
      for (int e = 0; e < 4; ++e) a[e] = ld_nc(pa + min(k + 8 * e, U.k1 - 1));
      if (x1) {
        const double2 *pb = x1 + (size_t)p * (size_t)G;
#pragma unroll
        for (int e = 0; e < 4; ++e) b[e] = ld_nc(pb + min(k + 8 * e, U.k1 - 1));
      }
    };
    // L2 prefetch of a task's 4 rows x 512 bytes of each slice, one
    // 128-byte line per lane (lanes 0-3 of a row: x0, lanes 4-7: x1).
    auto prefetch = [&](int j, int row) {
      const double2 *x = (q8 < 4) ? x0 : x1;
      if (!x) return;
      const int p = min(p_base + row, P - 1);
      const int k = min(U.k0 + j * kFK + 8 * (q8 & 3), U.k1 - 1);
      prefetch_l2(x + (size_t)p * (size_t)G + k);
    };
    auto value = [&](const double2 (&a)[4], const double2 (&b)[4], int j, int row, double (&cr)[4],
                     double (&ci)[4]) {
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        double2 x = a[e];
        if (x1) {
          x.x -= b[e].x;
          x.y -= b[e].y;
        }
        cr[e] = x.x;
        ci[e] = x.y;
      }
      if (inside(j)) return;
      const bool rv = p_base + row < P;
      const int k = U.k0 + j * kFK + q8;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const bool ok = rv && k + 8 * e < U.k1;
        cr[e] = ok ? cr[e] : 0.0;
        ci[e] = ok ? ci[e] : 0.0;
      }
    };
    // Row scales of all 128 rows from stage 0 (the unit's first kFK k):
    // largest |re|, |im| (both CTAs of a pair compute the same values).
    if (ns > 0) {
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int row = (cw + kFConvWarps * i) * 4 + r4;
        double2 a[4], b[4];
        issue(a, b, 0, row);
        double cr[4], ci[4];
        value(a, b, 0, row, cr, ci);
        double m = 0.0;
#pragma unroll
        for (int e = 0; e < 4; ++e) m = fmax(m, fmax(fabs(cr[e]), fabs(ci[e])));
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 1));
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 2));
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 4));
        if (q8 == 0) sm.rmax[row] = m;
      }
    }
    // Loads run one task ahead of the conversion, L2 prefetches kFPrefetch
    // stages ahead (so the loads are L2 hits).
    for (int j = 1; j <= kFPrefetch && j < ns; ++j)
#pragma unroll
      for (int i = 0; i < kT; ++i) prefetch(j, task_row(i));
    double2 ca[4], cb[4];
    if (ns > 0) issue(ca, cb, 0, task_row(0));
    conv_sync();
    if (ct < kFM) {
      const double m = sm.rmax[ct];
      int e = 0;
      if (m > 0.0 && m <= DBL_MAX) (void)frexp(m, &e);
      const int E = e + kFHeadroom;
      if (m > 0.0 && m <= DBL_MAX && 38 - E <= 1000) {
        sm.mult[ct] = ldexp(1.0, 38 - E);
        sm.lim[ct] = ldexp(1.0, E);
        sm.ex[ct] = E + 2;  // x = 2^(E + 2) sum_s d_s 256^-(s + 1)
      } else {
        // No usable scale (zero, tiny or non-finite first block): every
        // nonzero value of the row is out of range.
        sm.mult[ct] = 1.0;
        sm.lim[ct] = m > 0.0 ? 0.0 : 4.9406564584124654e-324;
        sm.ex[ct] = 0;
      }
    }
    conv_sync();

    bool ovf = false;
    for (int j = 0; j < ns; ++j) {
      const int st = j % kFStages;
      if (j >= kFStages && !fwait(&sm.empty[st], ((j / kFStages) - 1) & 1, status, budget)) break;
#pragma unroll
      for (int i = 0; i < kT; ++i) {
        const int row = task_row(i);
        if (j + kFPrefetch < ns) prefetch(j + kFPrefetch, row);
        double cr[4], ci[4];
        value(ca, cb, j, row, cr, ci);
        if (i + 1 < kT)
          issue(ca, cb, j, task_row(i + 1));
        else if (j + 1 < ns)
          issue(ca, cb, j + 1, task_row(0));
        const double mult = sm.mult[row], lim = sm.lim[row];
        uint32_t wr[kFS], wi[kFS];
        digits4(cr, mult, lim, ovf, wr);
        digits4(ci, mult, lim, ovf, wi);
        // Stage positions [4 q8, 4 q8 + 4): 16-k column group q8 / 4, word q8 % 4.
        static_assert(kFXPlane % 16 == 0 && kFXLbo % 16 == 0, "descriptor addresses are 16-byte units");
        uint32_t *dst = reinterpret_cast<uint32_t *>(
            &sm.x[st][(q8 >> 2) * kFXLbo + (row >> 3) * 128 + (row & 7) * 16 + (q8 & 3) * 4]);
#pragma unroll
        for (int s2 = 0; s2 < kFS; ++s2) {
          dst[(s2 * kFXPlane) / 4] = wr[s2];
          dst[((kFS + s2) * kFXPlane) / 4] = wi[s2];
        }
      }
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(PAIR ? &sm.xlocal[st] : &sm.xfull[st]);
    }
    if (ovf) sm.ovf = 1;
    conv_sync();
    // A pair: the peer learns whether a value of this CTA's rows did not fit.
    if (PAIR && ct == 0 && sm.ovf) st_peer(peer_addr(&sm.ovf_peer, peer), 1);
  }
  // ---- all roles have issued their work; wait for the MMAs.
  bool dn = true;
  if (lane == 0 && warp != 1) dn = fwait(&sm.done, 0, status, budget);
  dn = __shfl_sync(0xffffffffu, (int)dn, 0) != 0;
  if (PAIR) {
    cluster_sync();  // the peer's nrecv / ovf_peer are visible, and it issues nothing more
    // Copies the peer sent into this CTA land before it exits (they have
    // already, unless a wait ran out).
    if (threadIdx.x == 64) {
      const int n = sm.nrecv;
      for (int t = 0; t < kFStages; ++t) {
        if (n <= t) continue;
        const int last = (n - 1) - ((n - 1 - t) % kFStages);
        (void)fwait(&sm.xfull[t], (last / kFStages) & 1, status, budget);
      }
    }
  } else {
    __syncthreads();
  }
  tc::fence_after();
  if (warp >= 2) {
    // ---- epilogue.  Warps cw < kFEpiWarps: lane quarter q = warp % 4 (TMEM
    // lanes = G' columns [32 q, 32 q + 32)), half hh = cw / 4 of the rows.
    const int cw = warp - 2, ct = (int)threadIdx.x - 64;
    const int p_base = U.pt * kFM;
    const bool flagged = (sm.ovf | sm.ovf_peer) != 0;
    if (cw < kFEpiWarps) {
      const int q = warp & 3, hh = cw >> 2;
      const int nh = nrp >> 1, j0 = hh * nh;
      const int pl = q * 32 + lane, pg = p_base + pl;
      const double sc = ldexp(1.0, sm.ex[pl]);
      const uint32_t tq = tmem + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
      for (int c = 0; c < nh; c += 4) {
        // The 4 rows' W(band, p) first (their latency overlaps the TMEM loads).
        double2 w[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const FuseRow fr = frows[C.slot0 + j0 + c + e];
          const bool use = pg < P && fr.coef != 0.0 && BGW_CHECKED((unsigned)fr.band < (unsigned)nb_w, status, 65);
          w[e] = use ? W[(size_t)fr.band * P + pg] : make_double2(0.0, 0.0);
        }
        double vr[4] = {0.0, 0.0, 0.0, 0.0}, vi[4] = {0.0, 0.0, 0.0, 0.0};
        if (dn && !flagged) {
          int32_t re[kFS][4], im[kFS][4];
#pragma unroll
          for (int li = 0; li < kFS; ++li) {
            tc::ld4(tq + (uint32_t)(li * N + j0 + c), re[li]);
            tc::ld4(tq + (uint32_t)(li * N + nrp + j0 + c), im[li]);
          }
          tc::wait_ld();
#pragma unroll
          for (int li = 0; li < kFS; ++li) {
            const double wl = ldexp(1.0, -8 * (li + 2));
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              vr[e] = fma((double)re[li][e], wl, vr[e]);
              vi[e] = fma((double)im[li][e], wl, vi[e]);
            }
          }
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const double dr = vr[e] * sc, di = vi[e] * sc;
          double cr = dr * w[e].x - di * w[e].y, ci = dr * w[e].y + di * w[e].x;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            cr += __shfl_xor_sync(0xffffffffu, cr, o);
            ci += __shfl_xor_sync(0xffffffffu, ci, o);
          }
          if (lane == 0) {
            sm.red[q][j0 + c + e][0] = cr;
            sm.red[q][j0 + c + e][1] = ci;
          }
        }
      }
    }
    conv_sync();
    if (per_row) {
      // One partial per row slot (distinct outputs per iw: the plan's terms
      // combine them); zero for padding slots and flagged units.
      if (ct < kFMaxRows) {
        double pr = 0.0, pi = 0.0;
        if (!flagged && ct < nrp) {
          const FuseRow fr = frows[C.slot0 + ct];
          const double f = fr.coef * sB[(size_t)(C.slot0 + ct) * NW + U.k0 / kFWin];
          pr = f * (((sm.red[0][ct][0] + sm.red[1][ct][0]) + sm.red[2][ct][0]) + sm.red[3][ct][0]);
          pi = f * (((sm.red[0][ct][1] + sm.red[1][ct][1]) + sm.red[2][ct][1]) + sm.red[3][ct][1]);
        }
        partials[((size_t)blockIdx.x * kFMaxRows + ct) * 2 + 0] = pr;
        partials[((size_t)blockIdx.x * kFMaxRows + ct) * 2 + 1] = pi;
      }
      if (ct == 0) unit_flag[blockIdx.x] = (flagged && !phantom) ? 1 : 0;
    } else if (ct == 0) {
      double pr = 0.0, pi = 0.0;
      if (!flagged) {
        const int w = U.k0 / kFWin;
        for (int j = 0; j < nrp; ++j) {
          const FuseRow fr = frows[C.slot0 + j];
          if (fr.coef == 0.0) continue;
          const double f = fr.coef * sB[(size_t)(C.slot0 + j) * NW + w];
          const double vr = ((sm.red[0][j][0] + sm.red[1][j][0]) + sm.red[2][j][0]) + sm.red[3][j][0];
          const double vi = ((sm.red[0][j][1] + sm.red[1][j][1]) + sm.red[2][j][1]) + sm.red[3][j][1];
          pr = fma(f, vr, pr);
          pi = fma(f, vi, pi);
        }
      }
      partials[2 * (size_t)blockIdx.x] = pr;
      partials[2 * (size_t)blockIdx.x + 1] = pi;
      unit_flag[blockIdx.x] = (flagged && !phantom) ? 1 : 0;
    }
  }
  tc::fence_before();
  if (PAIR)
    cluster_sync();  // no remote access targets a CTA that has exited
  else
    __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    tc::dealloc(tmem, 512);
  }
}

}  // namespace

int ff_launch_fused(CallEnv *env, const FFPlan &plan, int64_t nb_w, int64_t nE, int64_t G, int64_t P, const int32_t *inv,
                    const int32_t *indinv, int64_t indinv_len, const double2 *am, const double2 *an,
                    const double *vc, const double2 *R, int r_f0, const double2 *A, int a_f0, int min_rows,
                    double *achs_dev, double *asx_dev, double *cor_dev) {
  Workspace *ws = env->ws;
  cudaStream_t stream = env->stream;
  double2 *W = nullptr;
  BGW_TRY(ff_build_w(env, nb_w, G, P, inv, indinv, indinv_len, am, vc, &W));
  if (min_rows <= 0) min_rows = kFuseMinRows;

  std::vector<FFGroup> small, big;
  for (const auto &g : plan.groups) (g.row_count >= min_rows ? big : small).push_back(g);
  const size_t slice = (size_t)P * (size_t)G;
  const int KB = (int)((G + kFK - 1) / kFK);
  const int NW = (int)((G + kFWin - 1) / kFWin);
  const int PT = (int)((P + kFM - 1) / kFM);

  // Chunks: each big group split into ceil(rows / kFMaxRows) chunks of
  // nearly equal size, padded to whole 8-row groups.
  std::vector<FuseChunk> chunks;
  std::vector<FuseRow> frows;
  std::vector<int> chunk_row0, chunk_nr, chunk_group, group_chunk0;
  long long off = 0;
  for (int gi = 0; gi < (int)big.size(); ++gi) {
    const FFGroup &g = big[gi];
    const int n = g.row_count, nch = (n + kFMaxRows - 1) / kFMaxRows;
    group_chunk0.push_back((int)chunks.size());
    int r0 = 0;
    for (int c = 0; c < nch; ++c) {
      const int nr = n / nch + (c < n % nch ? 1 : 0);
      FuseChunk ch;
      ch.b_off = off;
      ch.x0 = (g.src == SRC_A) ? A + (size_t)(g.f - a_f0) * slice : R + (size_t)(g.f - r_f0) * slice;
      ch.x1 = (g.src == SRC_RA) ? A + (size_t)(g.f - a_f0) * slice : nullptr;
      ch.slot0 = (int)frows.size();
      ch.nrp = (nr + 7) / 8 * 8;
      ch.out = g.out;
      ch.pad = 0;
      for (int r = 0; r < ch.nrp; ++r) {
        FuseRow fr;
        fr.chunk = (int)chunks.size();
        if (r < nr) {
          fr.band = plan.rows[g.row_begin + r0 + r].band;
          fr.coef = plan.rows[g.row_begin + r0 + r].coef;
        } else {
          fr.band = 0;
          fr.coef = 0.0;
        }
        frows.push_back(fr);
      }
      chunk_row0.push_back(g.row_begin + r0);
      chunk_nr.push_back(nr);
      chunk_group.push_back(gi);
      off += (long long)KB * 2 * kFS * 2 * ch.nrp * kFK;
      chunks.push_back(ch);
      r0 += nr;
    }
  }
  group_chunk0.push_back((int)chunks.size());
  // Units in (group, window, column tile, chunk) order: the chunks of one
  // X tile run side by side (the tile comes from DRAM once, then L2), and
  // so do the column tiles reading one chunk's digits.  With kFPair the
  // chunks of an X tile go in twos to 2-CTA clusters (an odd chunk count
  // leaves a phantom partner that only converts its half of the tile).
  std::vector<FuseUnit> units;
  for (int gi = 0; gi < (int)big.size(); ++gi)
    for (int w = 0; w < NW; ++w)
      for (int pt = 0; pt < PT; ++pt)
        for (int c = group_chunk0[gi]; c < group_chunk0[gi + 1]; c += kFPair ? 2 : 1)
          for (int m = 0; m < (kFPair ? 2 : 1); ++m) {
            FuseUnit u;
            u.phantom = c + m >= group_chunk0[gi + 1] ? 1 : 0;
            u.chunk = u.phantom ? c : c + m;
            u.pt = pt;
            u.k0 = w * kFWin;
            u.k1 = (int)std::min<int64_t>(G, (int64_t)(w + 1) * kFWin);
            u.pad = 0;
            units.push_back(u);
          }

  // FP64 tiles: the small groups (always run), then the recomputation tiles
  // of every unit (gated on its flag).
  std::vector<FFTile> ft;
  std::vector<int> gate;
  if (!small.empty()) {
    int per_sm = 1;
    BGW_TRY(ff_fp64_per_sm(&per_sm));
    ff_fp64_tiles(small, P, G, 2 * ws->sm_count * std::max(per_sm, 1), &ft);
    gate.assign(ft.size(), -1);
  }
  const int tr = ff_fp64_tile_rows(), tcn = ff_fp64_tile_cols();
  for (int u = 0; u < (int)units.size(); ++u) {
    const FuseUnit &U = units[u];
    if (U.phantom) continue;
    const FFGroup &g = big[chunk_group[U.chunk]];
    for (int r0 = 0; r0 < chunk_nr[U.chunk]; r0 += tr)
      for (int64_t p0 = (int64_t)U.pt * kFM; p0 < std::min<int64_t>(P, (int64_t)(U.pt + 1) * kFM); p0 += tcn) {
        FFTile t;
        t.src = g.src;
        t.f = g.f;
        t.row_begin = chunk_row0[U.chunk] + r0;
        t.row_count = std::min(tr, chunk_nr[U.chunk] - r0);
        t.p_begin = (int32_t)p0;
        t.k_begin = U.k0;
        t.k_count = U.k1 - U.k0;
        t.out = g.out;
        ft.push_back(t);
        gate.push_back(u);
      }
  }
  std::vector<BSliceTask> btasks;  // band-row slicing: (chunk, group of 8 row slots)
  for (int c = 0; c < (int)chunks.size(); ++c)
    for (int gr = 0; gr < chunks[c].nrp / 8; ++gr) btasks.push_back({c, gr});
  const int nbt = (int)btasks.size();
  const int nft = (int)ft.size(), nu = (int)units.size(), ns = (int)frows.size();
  // Partials: FP64 tiles first, then the units'.  One per tile / unit, or
  // with distinct outputs per iw one per tile row / row slot, combined by the
  // plan's terms (out_of then holds the plan row of each partial, -1: none).
  const bool per_row = plan.per_iw;
  std::vector<int> out_of;
  if (per_row) {
    ff_fp64_row_ids(ft, &out_of);
    for (int i = 0; i < nu; ++i)
      for (int j = 0; j < kFMaxRows; ++j)
        out_of.push_back(!units[i].phantom && j < chunk_nr[units[i].chunk] ? chunk_row0[units[i].chunk] + j : -1);
  } else {
    out_of.resize(nft + nu);
    for (int i = 0; i < nft; ++i) out_of[i] = ft[i].out;
    for (int i = 0; i < nu; ++i) out_of[nft + i] = chunks[units[i].chunk].out;
  }
  const size_t n_part = out_of.size();
  const size_t unit_part0 = per_row ? (size_t)nft * ff_fp64_tile_rows() : (size_t)nft;  // first unit partial

  // Device buffers: packed band-row digits (TABLE0); plan tables, scales
  // and unit flags in one buffer (PLAN).
  void *pack = nullptr, *plan_buf = nullptr, *partials = nullptr;
  BGW_TRY(ws_reserve(ws, SLOT_TABLE0, (size_t)std::max<long long>(off, 256), &pack));
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t o_rows = 0;
  const size_t o_ft = o_rows + al(sizeof(FFRow) * std::max<size_t>(plan.rows.size(), 1));
  const size_t o_gate = o_ft + al(sizeof(FFTile) * std::max(nft, 1));
  const size_t o_ch = o_gate + al(sizeof(int) * std::max(nft, 1));
  const size_t o_fr = o_ch + al(sizeof(FuseChunk) * std::max<size_t>(chunks.size(), 1));
  const size_t o_un = o_fr + al(sizeof(FuseRow) * std::max(ns, 1));
  const size_t o_out = o_un + al(sizeof(FuseUnit) * std::max(nu, 1));
  const size_t o_bt = o_out + al(sizeof(int) * std::max<size_t>(n_part, 1));
  const size_t o_sb = o_bt + al(sizeof(BSliceTask) * std::max(nbt, 1));
  const size_t o_flag = o_sb + al(sizeof(double) * std::max<size_t>((size_t)ns * NW, 1));
  const size_t total = o_flag + al(sizeof(int) * std::max(nu, 1));
  std::vector<unsigned char> host(o_sb, 0);  // the device-written tail is not uploaded
  auto put = [&](size_t o, const void *src, size_t bytes) {
    if (bytes) std::memcpy(host.data() + o, src, bytes);
  };
  put(o_rows, plan.rows.data(), sizeof(FFRow) * plan.rows.size());
  put(o_ft, ft.data(), sizeof(FFTile) * nft);
  put(o_gate, gate.data(), sizeof(int) * nft);
  put(o_ch, chunks.data(), sizeof(FuseChunk) * chunks.size());
  put(o_fr, frows.data(), sizeof(FuseRow) * ns);
  put(o_un, units.data(), sizeof(FuseUnit) * nu);
  put(o_out, out_of.data(), sizeof(int) * n_part);
  put(o_bt, btasks.data(), sizeof(BSliceTask) * nbt);
  BGW_TRY(ws_reserve(ws, SLOT_PLAN, total, &plan_buf));
  BGW_CUDA_TRY(cudaMemcpyAsync(plan_buf, host.data(), o_sb, cudaMemcpyHostToDevice, stream));
  unsigned char *pb = static_cast<unsigned char *>(plan_buf);
  BGW_TRY(ws_reserve(ws, SLOT_PARTIALS, sizeof(double) * 2 * std::max<size_t>(n_part, 1), &partials));
  double *part = static_cast<double *>(partials);
  int *d_flag = (int *)(pb + o_flag);

  BGW_TRY(prof_mark(env, 1));
  const uint64_t launches_before = g_launches.load();
  if (nu > 0) {
    const FuseChunk *d_ch = (const FuseChunk *)(pb + o_ch);
    const FuseRow *d_fr = (const FuseRow *)(pb + o_fr);
    double *d_sb = (double *)(pb + o_sb);
    ff_bslice_kernel<<<(unsigned)((size_t)nbt * NW), kFBThreads, 0, stream>>>(
        (const BSliceTask *)(pb + o_bt), d_fr, d_ch, NW, (int)G, KB, an, (int)nb_w, (int8_t *)pack, off, d_sb,
        env->d_status);
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
    const int smem = (int)sizeof(FuseSmem);
    auto kern = ff_fuse_kernel<kFPair>;
    BGW_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)nu);
    cfg.blockDim = dim3(kFThreads);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kFPair ? 2 : 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BGW_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, (const FuseUnit *)(pb + o_un), d_ch, d_fr, ns,
                                    (const int8_t *)pack, off, (const double *)d_sb, NW, (const double2 *)W, (int)P,
                                    (int)G, (int)nb_w, part + 2 * unit_part0, d_flag, per_row ? 1 : 0,
                                    env->d_status, stall_step()));
    count_launch();
    BGW_CUDA_TRY(cudaGetLastError());
  }
  BGW_TRY(ff_launch_fp64_tiles(stream, (const FFTile *)(pb + o_ft), nft, (const FFRow *)(pb + o_rows),
                               (int)plan.rows.size(), nb_w, P, G, an, R, r_f0, A, a_f0, W, part, env->d_status,
                               per_row, (const int *)(pb + o_gate), d_flag));
  BGW_TRY(prof_mark(env, 2));
  if (per_row) {
    FFTermTables tt;
    ff_build_term_tables(plan, out_of, nE, &tt);
    BGW_TRY(ff_launch_term_finalize(env, SLOT_TABLE1, tt, part, nE, achs_dev, asx_dev, cor_dev));
  } else {
    BGW_TRY(ff_enqueue_out_finalize(stream, part, (const int *)(pb + o_out), (int)n_part, (int)nE, achs_dev, asx_dev,
                                    cor_dev));
  }
  {
    double slices = 0.0;
    for (const auto &b : plan.slice_reads) slices += b;
    env->prof.flops = 8.0 * plan.useful_cmacs;
    env->prof.main_bytes = slices * 16.0 * (double)P * (double)G + 16.0 * (double)nb_w * (double)G + (double)off;
    env->prof.main_launches = (int)(g_launches.load() - launches_before);
    std::snprintf(env->prof.main_kernel, sizeof(env->prof.main_kernel), "ff_fuse_kernel");
  }
  // The pageable plan buffer must outlive its (staged) upload.
  BGW_CUDA_TRY(cudaStreamSynchronize(stream));
  return BGW_OK;
}

}  // namespace bgw
