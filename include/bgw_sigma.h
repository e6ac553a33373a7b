/*
 * bgw_sigma.h -- C ABI of libbgwsigma.so, the B200 (sm_100a) implementation
 * of the BerkeleyGW GPP and full-frequency (FF) self-energy summations.
 *
 * Every entry point takes plain pointers and sizes, returns a bgw_status
 * (0 = success, negative = error), never exits the process and never falls
 * back to a CPU path: with no usable CUDA device it returns
 * BGW_ERR_NO_DEVICE.
 *
 * Array conventions (identical to the reference's ArrayMD storage,
 * arrayMD/arrayMD.h:156-184, with ComplexType = std::complex<double>,
 * common/Defines.h:21-25):
 *   - complex arrays are interleaved (re, im) doubles, row-major, last index
 *     fastest; a complex [n][m] array is 2*n*m doubles;
 *   - index arrays are int32.
 * Pointers live in host memory (BGW_MEMORY_HOST, the default: the call copies
 * what it reads to the GPU and the results back) or in device memory of the
 * selected GPU (BGW_MEMORY_DEVICE).  Outputs are overwritten, never
 * accumulated into, as in the reference (GPP/gpp.cpp:399-401,
 * FF/ff.cpp:288-289, 374-375).
 *
 * Reductions are deterministic: no floating-point atomics, fixed-order
 * combination, so a rerun on the same inputs and device is bitwise
 * identical.
 */
#ifndef BGW_SIGMA_H
#define BGW_SIGMA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: bgw_options gained pole_guard; 3: bgw_options gained mixed_order
 * (bgw_options_init writes the whole current struct, so it must be given a
 * struct of this header's size). */
#define BGW_SIGMA_ABI_VERSION 3

typedef enum bgw_status {
  BGW_OK = 0,
  BGW_ERR_INVALID_ARG = -1, /* bad size, null pointer or option          */
  BGW_ERR_INDEX = -2,       /* inv_igp_index / indinv entry out of range */
  BGW_ERR_CUDA = -3,        /* a CUDA runtime call failed                */
  BGW_ERR_ALLOC = -4,       /* device or pinned allocation failed        */
  BGW_ERR_NO_DEVICE = -5,   /* no usable CUDA device                     */
  BGW_ERR_TIMEOUT = -6,     /* a bounded device-side wait ran out        */
  BGW_ERR_UNSUPPORTED = -7, /* option combination not implemented        */
  BGW_ERR_CHECK = -8        /* a bounds check of the debug build failed
                               (libbgwsigma_check.so, built with
                               -DBGW_CHECK; never raised otherwise)      */
} bgw_status;

enum { BGW_MEMORY_HOST = 0, BGW_MEMORY_DEVICE = 1 };
enum { BGW_PRECISION_FP64 = 0, BGW_PRECISION_MIXED = 1 };
/* GPP evaluation strategy:
 *   BANDLOOP  evaluates every (band, G', G, frequency) quotient, as the
 *             reference loop nest does (GPP/gpp.cpp:343-390); supports a
 *             band-dependent wx (wx_band_stride != 0).  FP64-pipe bound.
 *   FACTORED  uses sum_n1 sch_store1(n1, p) once per G' column; valid only
 *             for a band-independent wx (wx_band_stride == 0, the
 *             reference's case) and bound by HBM bandwidth.
 *   AUTO      (default) FACTORED when wx_band_stride == 0, else BANDLOOP. */
enum { BGW_GPP_BANDLOOP = 0, BGW_GPP_FACTORED = 1, BGW_GPP_AUTO = 2 };
/* flags */
enum {
  BGW_FLAG_ASYNC = 1,  /* device memory only: enqueue on `stream` and return
                          without synchronising; the device-side status is
                          written to options->device_status (required).   */
  BGW_FLAG_PROFILE = 2, /* time the call's dominant kernel and all its device
                          work with CUDA events on `stream`; read back with
                          bgw_last_profile() (synchronous calls only).     */
  BGW_FLAG_FF_SLICE_ALL = 4, /* FF with BGW_PRECISION_MIXED: integer-slice
                          tensor-core products for every band group (staged
                          path: every group of more than 16 rows).
                          Default: groups of at least 8 rows (staged path:
                          128 rows); smaller groups stay FP64.             */
  BGW_FLAG_FF_WX_PER_IW = 8, /* FF asxDtemp / achDtemp_cor: evaluate every
                          point iw at wx = freqevalmin - ekq[n1] +
                          iw * freqevalstep, giving nfreqeval distinct
                          outputs.  Default (as FF/ff.cpp:245, 337): one
                          wx = freqevalmin - ekq[n1] + freqevalstep for all
                          iw, every output entry equal (the value at iw = 1
                          of this option).                                 */
  BGW_FLAG_FF_STAGED = 16 /* FF with BGW_PRECISION_MIXED: cut both operands
                          into digit buffers in HBM before the integer
                          products.  Default: the frequency slices are cut
                          inside the tensor-core kernel, read once.        */
};

typedef struct bgw_options {
  int32_t struct_size;     /* sizeof(bgw_options) (forward compatibility)   */
  int32_t memory;          /* BGW_MEMORY_HOST / BGW_MEMORY_DEVICE           */
  int32_t precision;       /* BGW_PRECISION_FP64 / BGW_PRECISION_MIXED      */
  int32_t gpp_algorithm;   /* BGW_GPP_AUTO / BGW_GPP_BANDLOOP / _FACTORED   */
  int64_t wx_band_stride;  /* doubles between bands' wx triples; 0 = shared */
  int32_t device;          /* CUDA ordinal; -1 = the calling thread's one   */
  int32_t flags;           /* BGW_FLAG_*                                    */
  void *stream;            /* cudaStream_t; NULL = legacy default stream    */
  int32_t *device_status;  /* device int written with BGW_FLAG_ASYNC        */
  double pole_guard;       /* GPP near-pole guard delta >= 0; 0 = off       */
  int32_t mixed_order;     /* GPP band loop, BGW_PRECISION_MIXED: Taylor
                              terms K (0..3) hoisted into FP64; default 3  */
} bgw_options;
/* mixed_order (GPP band loop with BGW_PRECISION_MIXED; not in the
 * reference): each step's quotients q = I / (x - w) are expanded about the
 * centre c of the step's band-chunk frequencies, t = (x - c) / (c - w):
 *   q = Q0 (1 - t + ... + (-t)^(K-1)) + (-t)^K Q0 / (1 + t),  Q0 = I / (c - w).
 * The K leading terms are summed over bands exactly, in FP64, through band
 * moments; the remainder, |t|^K of the term, is a per-term complex quotient
 * evaluated in FP32, so its rounding costs about 1e-7 |t|^K of the term.
 * K = 0 is a plain FP32 quotient (~1e-7 relative).  Elements with
 * |t| > 1/8 for some term (near a pole) are summed in FP64.  The cost per
 * term does not depend on K. */
/* pole_guard (GPP sums only; not in the reference, which has no guard and
 * only clamps wx >= 1e-6, GPP/gpp.cpp:273-274): with delta > 0 every
 * (band, G', G, frequency) term whose |wdiff|^2 = |wx - wtilde|^2 is below
 * delta^2 contributes zero -- the term's pole is excluded from the sum
 * (principal-value cut-off) instead of growing like 1/|wdiff|.  The test is
 * made on |wdiff|^2 in FP64 (with BGW_PRECISION_MIXED, every element a cut
 * could reach is summed in FP64).  In bgw_gpp_sigma's asxtemp the cut applies to each
 * of the two partial fractions 1/(wx - wtilde) and 1/(-wx - wtilde).
 * Supported by bgw_noflagOCC_solver and bgw_gpp_sigma; the adjoint and the
 * batched calls return BGW_ERR_UNSUPPORTED for delta > 0; the FF calls
 * ignore it.  An entry point given an older, shorter bgw_options (a smaller
 * struct_size, filled by the caller) reads only that many bytes and uses the
 * defaults (delta = 0, mixed_order = 3) for the fields it lacks;
 * bgw_options_init itself always writes the current layout. */

/* Fills *opt with the defaults (host memory, FP64, AUTO, stride 0,
 * current device, default stream, synchronous, no pole guard, mixed_order
 * 3). */
void bgw_options_init(bgw_options *opt);

/* ------------------------------------------------------------------ GPP --
 * Replaces noflagOCC_solver (GPP/gpp.cpp:307-402; prototype
 * common/Defines.h:50-62).  Same argument order and meaning:
 *   inv_igp_index [ngpown], indinv [indinv_len] (the reference allocates
 *   ncouls + 1, GPP/gpp.cpp:235), wx_array [3] (or [number_bands][stride]
 *   with opt->wx_band_stride), wtilde_array / I_eps_array complex
 *   [ngpown][ncouls], aqsmtemp / aqsntemp complex [number_bands][ncouls],
 *   vcoul [ncouls]; output achtemp complex [3].
 * achtemp[iw] = sum_{n1, my_igp, ig} sch_store1(n1, my_igp) *
 *               conj(wdiff) / |wdiff|^2 * I_eps[my_igp][ig],
 *   wdiff = wx[iw] - wtilde[my_igp][ig],  igp = indinv[inv_igp_index[my_igp]],
 *   sch_store1 = conj(aqsm[n1][igp]) aqsn[n1][igp] 0.5 vcoul[igp]
 *                wtilde[my_igp][igp].
 * Precision FP64: within 1e-12 relative of the reference's OpenMP build.
 * Precision MIXED: per-term quotients in FP32, compensated FP64
 * accumulation. */
int bgw_noflagOCC_solver(int64_t number_bands, int64_t ngpown, int64_t ncouls,
                         const int32_t *inv_igp_index, const int32_t *indinv,
                         int64_t indinv_len, const double *wx_array,
                         const double *wtilde_array, const double *aqsmtemp,
                         const double *aqsntemp, const double *I_eps_array,
                         const double *vcoul, double *achtemp,
                         const bgw_options *opt);

/* ---------------------------------------------------------- GPP adjoint --
 * Analytic adjoint of bgw_noflagOCC_solver (no counterpart in the
 * reference, whose quasiparticle renormalisation uses the three-point finite
 * difference over wx_array, GPP/gpp.cpp:271-275).  With q = 1/(wx - wtilde)
 * Sigma is holomorphic in wtilde and I_eps; for cotangents
 *   grad_achtemp[iw] = dL/dRe achtemp[iw] + i dL/dIm achtemp[iw]  (3 complex)
 * it returns the complex gradients dL/dRe z + i dL/dIm z:
 *   grad_wtilde [ngpown][ncouls] complex (includes wtilde[p][igp] inside
 *                                         sch_store1), may be NULL
 *   grad_I_eps  [ngpown][ncouls] complex, may be NULL
 *   dachtemp_domega [3] complex: d achtemp[iw] / d omega for a common
 *                   shift omega of wx[.][iw] (every band's), may be NULL
 * Quotients are recomputed, nothing of size bands x G' x G is stored.
 * Band-independent wx (wx_band_stride 0) with gpp_algorithm AUTO or
 * FACTORED: the factored form, HBM-bound.  A band-dependent wx
 * (wx_band_stride >= 3, wx_array [number_bands][stride]) or BANDLOOP: the
 * band-loop form, which walks every band per element (FP64-pipe bound).
 * FP64 only; pole_guard > 0 returns BGW_ERR_UNSUPPORTED.  Same arguments as
 * the forward otherwise. */
int bgw_noflagOCC_solver_backward(int64_t number_bands, int64_t ngpown,
                                  int64_t ncouls, const int32_t *inv_igp_index,
                                  const int32_t *indinv, int64_t indinv_len,
                                  const double *wx_array,
                                  const double *wtilde_array,
                                  const double *aqsmtemp,
                                  const double *aqsntemp,
                                  const double *I_eps_array,
                                  const double *vcoul,
                                  const double *grad_achtemp,
                                  double *grad_wtilde, double *grad_I_eps,
                                  double *dachtemp_domega,
                                  const bgw_options *opt);

/* ---------------------------------------------------------- GPP batched --
 * No counterpart in the reference (one instance per process).  Many GPP
 * instances -- q-points of uneven ncouls and number_bands -- evaluated by one
 * persistent launch: the work list of all instances is cut into equal-cost
 * ranges, one per CTA, and the prep / sum / finalize kernels are captured
 * once into a CUDA graph that bgw_gpp_batch_execute replays.  The elements
 * per thread (tile width and occupancy) are chosen at creation by timing the
 * candidate kernels on a sample of the work list (cached per batch shape).
 * Algorithm / precision as bgw_noflagOCC_solver (opt->gpp_algorithm,
 * opt->precision); FACTORED needs every wx_band_stride == 0.  All pointers
 * are device memory of the selected device and must stay valid while the
 * batch exists; the results go to each instance's achtemp. */
typedef struct bgw_gpp_instance {
  int64_t number_bands, ngpown, ncouls;
  const int32_t *inv_igp_index; /* [ngpown]                          */
  const int32_t *indinv;        /* [indinv_len]                      */
  int64_t indinv_len;
  const double *wx_array;       /* [3] or [number_bands][stride]     */
  int64_t wx_band_stride;
  const double *wtilde_array;   /* complex [ngpown][ncouls]          */
  const double *aqsmtemp;       /* complex [number_bands][ncouls]    */
  const double *aqsntemp;
  const double *I_eps_array;    /* complex [ngpown][ncouls]          */
  const double *vcoul;          /* [ncouls]                          */
  double *achtemp;              /* output, complex [3]               */
} bgw_gpp_instance;

typedef struct bgw_gpp_batch bgw_gpp_batch;
/* opt->memory must be BGW_MEMORY_DEVICE; opt->stream is used for tuning. */
int bgw_gpp_batch_create(const bgw_gpp_instance *instances, int64_t n,
                         const bgw_options *opt, bgw_gpp_batch **batch);
/* Replays the graph on opt->stream (NULL options: default stream,
 * synchronous).  With BGW_FLAG_ASYNC the status goes to
 * opt->device_status; with BGW_FLAG_PROFILE the replay is timed. */
int bgw_gpp_batch_execute(bgw_gpp_batch *batch, const bgw_options *opt);
int bgw_gpp_batch_info(const bgw_gpp_batch *batch, int32_t *elems_per_thread,
                       int32_t *grid, int64_t *total_items);
int bgw_gpp_batch_destroy(bgw_gpp_batch *batch);

/* ------------------------------------------ GPP, Coulomb hole + exchange --
 * No counterpart in the reference, whose GPP solver (GPP/gpp.cpp:307-402)
 * has no flagOCC branch and no asxtemp output; the screened-exchange part
 * is specified from the GPP model and its parity is therefore unpinned.
 *   achtemp (may be NULL): the Coulomb-hole sum of bgw_noflagOCC_solver over
 *            all number_bands bands (bitwise equal to a device-memory
 *            bgw_noflagOCC_solver call; host inputs are staged whole here);
 *   asxtemp (may be NULL): screened exchange of the occupied bands n1 <
 *            nvband, eps^-1 - 1 = Omega^2 / (w^2 - wtilde^2) with Omega^2 /
 *            wtilde = I_eps[p][ig] wtilde[p][igp]:
 *     asxtemp[iw] = - sum_{n1<nvband, p, ig} conj(aqsm[n1][igp]) aqsn[n1][igp]
 *                   vcoul[igp] wtilde[p][igp] I_eps[p][ig] wtilde[p][ig]
 *                   / (wx^2 - wtilde[p][ig]^2)
 *            (bare exchange excluded), evaluated as minus the Coulomb-hole sum
 *            of the occupied bands at +wx plus the same at -wx (partial
 *            fractions).  3 complex each.
 * Inputs as bgw_noflagOCC_solver (memory, precision, algorithm and wx_band_stride
 * options apply to both sums); 0 <= nvband <= number_bands. */
int bgw_gpp_sigma(int64_t number_bands, int64_t nvband, int64_t ngpown, int64_t ncouls,
                  const int32_t *inv_igp_index, const int32_t *indinv, int64_t indinv_len,
                  const double *wx_array, const double *wtilde_array, const double *aqsmtemp,
                  const double *aqsntemp, const double *I_eps_array, const double *vcoul,
                  double *achtemp, double *asxtemp, const bgw_options *opt);

/* --------------------------------------------------- GPP, no allocation --
 * No counterpart in the reference.  A variant of bgw_noflagOCC_solver for
 * callers that cannot allocate GPU memory: code whose device memory is all
 * owned by another runtime or a preallocated pool (so a cudaMalloc outside
 * it would fail or break the budget), and latency-critical loops that must
 * never enter the CUDA allocator, because cudaMalloc/cudaFree can
 * synchronise the whole device.  The regular entry points cannot serve them:
 * they grow a cached workspace with cudaMalloc on first use.
 *
 * This variant allocates nothing.  Its scratch (status words, the per-column
 * sums of sch_store1 over bands and per-CTA partials) is one static device
 * array of BGW_NOALLOC_SCRATCH_BYTES (1.1 MiB) compiled into the library;
 * every GPU that loads the library holds that array until the process exits.
 * It evaluates the factored GPP sum (exact algebra for the reference's
 * band-independent wx_array[3]; within 1e-12 of bgw_noflagOCC_solver).
 *   - Every pointer must be device memory of `device` (-1: current device);
 *     complex arrays 16-byte aligned.  achtemp: 3 complex (6 doubles).
 *   - ngpown must not exceed BGW_NOALLOC_MAX_NGPOWN: larger sizes return
 *     BGW_ERR_INVALID_ARG before any device work.
 *   - The call enqueues on `stream` (cudaStream_t, NULL = default stream)
 *     and synchronises it to read the status.
 *   - A device's first call fetches the array's device address
 *     (cudaGetSymbolAddress) for that device and keeps it for the life of
 *     the process; make that first call before any stream capture.  The
 *     kept address belongs to the device's primary context: do not use
 *     this entry point on a device after cudaDeviceReset has destroyed
 *     that context.
 *   - All calls on a device share the array, which keeps the last call's
 *     contents; the call clears the status words itself.  Calls that overlap
 *     on the GPU (other threads or streams) race on the scratch: serialise
 *     them. */
#define BGW_NOALLOC_MAX_NGPOWN 65536
#define BGW_NOALLOC_SCRATCH_BYTES 1147136
int bgw_noflagOCC_solver_noalloc(int64_t number_bands, int64_t ngpown,
                                 int64_t ncouls, const int32_t *inv_igp_index,
                                 const int32_t *indinv, int64_t indinv_len,
                                 const double *wx_array,
                                 const double *wtilde_array,
                                 const double *aqsmtemp,
                                 const double *aqsntemp,
                                 const double *I_eps_array,
                                 const double *vcoul, double *achtemp,
                                 int32_t device, void *stream);

/* ------------------------------------------------------------------- FF --
 * Replaces achsDtemp_Kernel (FF/ff.cpp:171-209).  Note the reference order
 * aqsntemp before aqsmtemp.  I_epsR_array complex [nFreq][ngpown][ncouls]
 * (only frequency 1 is read, ff.cpp:200); indinv [indinv_len] (ncouls in
 * the FF driver, ff.cpp:552); achsDtemp: 1 complex. */
int bgw_achsDtemp_Kernel(int64_t number_bands, int64_t ngpown, int64_t ncouls,
                         const int32_t *inv_igp_index, const int32_t *indinv,
                         int64_t indinv_len, const double *aqsntemp,
                         const double *aqsmtemp, const double *I_epsR_array,
                         int64_t nFreq, const double *vcoul, double *achsDtemp,
                         const bgw_options *opt);

/* Replaces asxDtemp_Kernel (FF/ff.cpp:211-293).  ekq [number_bands] (only
 * the first nvband entries are read), dFreqGrid [nFreq], I_epsR_array /
 * I_epsA_array complex [nFreq][ngpown][ncouls], aqsm/aqsn complex
 * [number_bands][ncouls]; asxDtemp: nfreqeval complex.  number_bands is the
 * row extent of aqsm/aqsn/ekq (the reference takes it from the ArrayMDs). */
int bgw_asxDtemp_Kernel(int64_t nvband, int64_t nfreqeval, int64_t ncouls,
                        int64_t ngpown, int64_t nFreq, double freqevalmin,
                        double freqevalstep, double occ, const double *ekq,
                        const double *dFreqGrid, const int32_t *inv_igp_index,
                        const int32_t *indinv, int64_t indinv_len,
                        const double *aqsmtemp, const double *aqsntemp,
                        int64_t number_bands, const double *vcoul,
                        const double *I_epsR_array, const double *I_epsA_array,
                        double *asxDtemp, const bgw_options *opt);

/* Replaces achDtemp_cor_Kernel (FF/ff.cpp:295-379, with
 * schDttt_corKernel1/2 :381-451); achDtemp_cor: nfreqeval complex.
 * flag_occ is evaluated per band (n1 < nvband), the intended meaning of the
 * reference's shared variable (ff.cpp:310, 334). */
int bgw_achDtemp_cor_Kernel(int64_t number_bands, int64_t nvband,
                            int64_t nfreqeval, int64_t ncouls, int64_t ngpown,
                            int64_t nFreq, double freqevalmin,
                            double freqevalstep, const double *ekq,
                            const double *dFreqGrid,
                            const int32_t *inv_igp_index,
                            const int32_t *indinv, int64_t indinv_len,
                            const double *aqsmtemp, const double *aqsntemp,
                            const double *vcoul, const double *I_epsR_array,
                            const double *I_epsA_array, double *achDtemp_cor,
                            const bgw_options *opt);

/* The three FF sums of one driver run (FF/ff.cpp:697-733) in one call that
 * stages each input once and launches one contraction over all three.
 * Outputs as the three entry points above; any output pointer may be NULL
 * to skip that sum. */
int bgw_ff_sigma(int64_t number_bands, int64_t nvband, int64_t nfreqeval,
                 int64_t ncouls, int64_t ngpown, int64_t nFreq,
                 double freqevalmin, double freqevalstep, double occ,
                 const double *ekq, const double *dFreqGrid,
                 const int32_t *inv_igp_index, const int32_t *indinv,
                 int64_t indinv_len, const double *aqsmtemp,
                 const double *aqsntemp, const double *vcoul,
                 const double *I_epsR_array, const double *I_epsA_array,
                 double *achsDtemp, double *asxDtemp, double *achDtemp_cor,
                 const bgw_options *opt);

/* ------------------------------------------------------- input generation --
 * Replaces the drivers' host-side, single-threaded fills of their inputs
 * (GPP/gpp.cpp:246-275, FF/ff.cpp:585-633) for seeded synthetic runs: the
 * values are generated on the GPU by a counter-based generator, so a
 * sub-block of an array (one rank's G' rows, a chunk) is generated on its
 * own and every value is independent of the device, grid and order.
 *   out[i], 0 <= i < n, is word offset + i of stream (seed, stream) of
 *   Philox4x64-10 (Salmon et al., SC'11): word w is word w % 4 of the block
 *   with counter (w / 4 + 1, 0, 0, 0) and key (seed, stream) -- numpy's
 *   np.random.Philox(key=seed + stream * 2**64).random_raw() sequence.
 *   It is mapped to u = (word >> 11) * 2^-53 in [0, 1) and then to
 *   lo + (hi - lo) * u, two roundings and no fused multiply-add, with
 *   (lo_even, hi_even) for even words and (lo_odd, hi_odd) for odd words
 *   (real and imaginary parts of an interleaved complex array).
 * opt->memory: DEVICE fills device memory on opt->stream (asynchronous with
 * BGW_FLAG_ASYNC); HOST generates on the GPU and copies into `out`. */
int bgw_fill_uniform(double *out, int64_t n, uint64_t seed, uint64_t stream,
                     int64_t offset, double lo_even, double hi_even,
                     double lo_odd, double hi_odd, const bgw_options *opt);

/* ------------------------------------------------------------- profiling --
 * Filled by a synchronous call made with BGW_FLAG_PROFILE; per thread. */
typedef struct bgw_profile {
  double main_kernel_ms; /* dominant kernel: GPP band loop / factored stream,
                            FF contraction (CUDA events on the call's stream) */
  double device_ms;      /* everything the call enqueued, staging included   */
  double flops;          /* algorithmic flops of the call (GPP: 63 per
                            (band, G', G) triple, i.e. 21 per frequency;
                            FF: 8 per complex multiply-add of the useful
                            contraction rows)                                */
  double main_bytes;     /* compulsory HBM bytes of the dominant kernel      */
  int32_t main_launches; /* launches of the dominant kernel                  */
  int32_t total_launches;/* kernel launches of the call                      */
  char main_kernel[48];  /* name of the dominant kernel                      */
} bgw_profile;
int bgw_last_profile(bgw_profile *out);

/* --------------------------------------------------------------- utility */
const char *bgw_status_string(int status);
int bgw_abi_version(void);
/* Number of kernel launches the library issued on this process so far (all
 * devices).  Lets a caller count launches inside a timed region. */
uint64_t bgw_launch_count(void);
/* Times FP64 DFMA and DMMA (mma.sync m8n8k4 f64) throughput microkernels on
 * `device` and returns TFLOP/s (2 flops per FMA).  Used as the measured
 * FP64 roofline denominators. */
int bgw_measure_fp64_peak(int32_t device, double *dfma_tflops,
                          double *dmma_tflops);
/* Releases the library's cached device workspace on `device` (-1: all). */
int bgw_release_workspace(int32_t device);

/* Test hook of the timeout path (no counterpart in the reference, whose
 * only failure handling is exit() on bad command-line sizes).  The kernels
 * that stage their inputs through double-buffered bulk copies -- the GPP
 * band loop (FP64 and mixed), both GPP adjoint kernels and the batched band
 * loop -- wait for each staged step with a bounded wait.  After
 * bgw_debug_inject_stall(step), every such kernel launched later (any call,
 * any device; a batch's kernels are fixed when bgw_gpp_batch_create captures
 * them) makes the wait of CTA-local step `step` on a barrier that never
 * completes, with a ~0.1 ms budget.  The wait runs out, the kernel lets its
 * copies in flight land and exits, and the call returns BGW_ERR_TIMEOUT; the
 * context stays usable.  step = -1 (the default) turns the stall off. */
int bgw_debug_inject_stall(int64_t step);

/* Accuracy probe of the kernels' reciprocals (no counterpart in the
 * reference, which divides with std::complex / double division).  For each
 * of the n host values in[i] it evaluates on the GPU, and copies back:
 *   refined[i]  the FP64 kernels' reciprocal (rcp.approx.ftz.f64 refined by
 *               one third-order Newton-Householder step);
 *   seed[i]     its starting value, rcp.approx.ftz.f64(in[i]);
 *   f32[i]      rcp.approx.ftz.f32((float)in[i]), the reciprocal of the
 *               mixed-precision remainder quotients. */
int bgw_debug_rcp_probe(const double *in, int64_t n, double *refined,
                        double *seed, float *f32, int32_t device);

#ifdef __cplusplus
}
#endif
#endif /* BGW_SIGMA_H */
