// capi.cu -- the extern "C" entry points of libbgwsigma.so (include/bgw_sigma.h).
//
// Each entry point validates its arguments on the host (no launch on a bad
// size or pointer), stages host inputs to the device when asked, enqueues
// the kernels of gpp.cu / ff.cu on the caller's stream and, unless
// BGW_FLAG_ASYNC, synchronises and returns the device-side status.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bgw_internal.cuh"

namespace bgw {

struct FFPlan;
int gpp_enqueue(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                int64_t indinv_len, const double *wx, int64_t wx_stride, const double2 *wt, const double2 *am,
                const double2 *an, const double2 *ie, const double *vc, double *achtemp_dev);
int gpp_run_host(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                 int64_t indinv_len, const double *wx, size_t wx_n, int64_t wx_stride, const double *wt,
                 const double *am, const double *an, const double *ie, const double *vc, double *achtemp_dev);

int gpp_sx_enqueue(CallEnv *env, int64_t nvband, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                   int64_t indinv_len, const double *wx, size_t wx_n, int64_t wx_stride, const double2 *wt,
                   const double2 *am, const double2 *an, const double2 *ie, const double *vc, double *asx_dev);
int gpp_sigma_factored_enqueue(CallEnv *env, int64_t nb, int64_t nv, int64_t P, int64_t G, const int32_t *inv,
                               const int32_t *indinv, int64_t indinv_len, const double *wx, const double2 *wt,
                               const double2 *am, const double2 *an, const double2 *ie, const double *vc,
                               double *ach_dev, double *asx_dev);

int gpp_adjoint_bandloop_enqueue(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv,
                                 const int32_t *indinv, int64_t indinv_len, const double *wx, int64_t wx_stride,
                                 const double2 *wt, const double2 *am, const double2 *an, const double2 *ie,
                                 const double *vc, const double2 *gcot, double2 *grad_wt, double2 *grad_ie,
                                 double *domega);

int gpp_adjoint_enqueue(CallEnv *env, int64_t nb, int64_t P, int64_t G, const int32_t *inv, const int32_t *indinv,
                        int64_t indinv_len, const double *wx, const double2 *wt, const double2 *am,
                        const double2 *an, const double2 *ie, const double *vc, const double2 *gcot,
                        double2 *grad_wt, double2 *grad_ie, double *domega);

int fill_uniform_enqueue(CallEnv *env, double *out, int64_t n, uint64_t seed, uint64_t stream, int64_t off,
                         double lo_even, double hi_even, double lo_odd, double hi_odd);

}  // namespace bgw

#include "ff_plan.cuh"

namespace bgw {
namespace {

// Guards against products that overflow the 64-bit byte counts.
bool dims_ok(int64_t a, int64_t b) { return a >= 0 && b >= 0 && (a == 0 || b <= (int64_t(1) << 40) / a); }

// Common prologue: begin_call + lock + status reset.
struct Call {
  CallEnv env;
  std::unique_lock<std::mutex> lock;
  int st = BGW_OK;
  explicit Call(const bgw_options *opt) {
    st = begin_call(opt, &env);
    if (st != BGW_OK) return;
    lock = std::unique_lock<std::mutex>(env.ws->mu);
    st = ws_acquire(env.ws, env.stream);
    if (st != BGW_OK) return;
    void *s = nullptr;
    st = ws_reserve(env.ws, SLOT_STATUS, sizeof(int32_t) * STATUS_WORDS, &s);
    if (st != BGW_OK) return;
    env.d_status = static_cast<int *>(s);
    st = prof_mark(&env, 0);
    if (st != BGW_OK) return;
    if (cudaMemsetAsync(s, 0, sizeof(int32_t) * STATUS_WORDS, env.stream) != cudaSuccess) st = BGW_ERR_CUDA;
  }
};

int out_buffer(CallEnv *env, double *user, size_t bytes, double **dev) {
  if (!env->host) {
    *dev = user;
    return BGW_OK;
  }
  void *d = nullptr;
  BGW_TRY(ws_reserve(env->ws, SLOT_OUT, bytes, &d));
  *dev = static_cast<double *>(d);
  return BGW_OK;
}

}  // namespace
}  // namespace bgw

using namespace bgw;

extern "C" int bgw_noflagOCC_solver(int64_t number_bands, int64_t ngpown, int64_t ncouls,
                                    const int32_t *inv_igp_index, const int32_t *indinv, int64_t indinv_len,
                                    const double *wx_array, const double *wtilde_array, const double *aqsmtemp,
                                    const double *aqsntemp, const double *I_eps_array, const double *vcoul,
                                    double *achtemp, const bgw_options *opt) {
  const int64_t nb = number_bands, P = ngpown, G = ncouls;
  if (nb < 0 || P < 0 || G <= 0 || G > INT32_MAX || nb > INT32_MAX || P > INT32_MAX) return BGW_ERR_INVALID_ARG;
  if (!dims_ok(nb, G) || !dims_ok(P, G) || indinv_len <= 0 || indinv_len > INT32_MAX) return BGW_ERR_INVALID_ARG;
  if (!achtemp || !vcoul || !indinv) return BGW_ERR_INVALID_ARG;
  if (P > 0 && (!inv_igp_index || !wtilde_array || !I_eps_array)) return BGW_ERR_INVALID_ARG;
  if (nb > 0 && P > 0 && (!aqsmtemp || !aqsntemp)) return BGW_ERR_INVALID_ARG;
  Call c(opt);
  if (c.st != BGW_OK) return c.st;
  CallEnv *env = &c.env;
  const int64_t stride = env->opt.wx_band_stride;
  // wx may be absent only when nothing reads it: no bands and per-band rows.
  if (!wx_array && (nb > 0 || stride == 0)) return BGW_ERR_INVALID_ARG;
  if (stride != 0 && stride < 3) return BGW_ERR_INVALID_ARG;
  const size_t wx_n = !wx_array ? 0 : stride == 0 ? 3 : (size_t)(nb > 0 ? (nb - 1) * stride + 3 : 3);
  double *out = nullptr;
  BGW_TRY(out_buffer(env, achtemp, 6 * sizeof(double), &out));
  if (env->host) {
    // Host inputs: staged in G'-row chunks on a copy stream, overlapped with
    // the per-chunk kernels.
    BGW_TRY(gpp_run_host(env, nb, P, G, inv_igp_index, indinv, indinv_len, wx_array, wx_n, stride, wtilde_array,
                         aqsmtemp, aqsntemp, I_eps_array, vcoul, out));
  } else {
    const void *inv = nullptr, *ind = nullptr, *wx = nullptr, *wt = nullptr, *am = nullptr, *an = nullptr,
               *ie = nullptr, *vc = nullptr;
    const size_t pg = (size_t)P * (size_t)G * 16, ng = (size_t)nb * (size_t)G * 16;
    BGW_TRY(stage_input(env, SLOT_IN0, inv_igp_index, sizeof(int32_t) * (size_t)P, &inv));
    BGW_TRY(stage_input(env, SLOT_IN1, indinv, sizeof(int32_t) * (size_t)indinv_len, &ind));
    BGW_TRY(stage_input(env, SLOT_IN2, wx_array, sizeof(double) * wx_n, &wx));
    BGW_TRY(stage_input(env, SLOT_IN3, wtilde_array, pg, &wt));
    BGW_TRY(stage_input(env, SLOT_IN4, aqsmtemp, ng, &am));
    BGW_TRY(stage_input(env, SLOT_IN5, aqsntemp, ng, &an));
    BGW_TRY(stage_input(env, SLOT_IN6, I_eps_array, pg, &ie));
    BGW_TRY(stage_input(env, SLOT_IN7, vcoul, sizeof(double) * (size_t)G, &vc));
    BGW_TRY(gpp_enqueue(env, nb, P, G, (const int32_t *)inv, (const int32_t *)ind, indinv_len, (const double *)wx,
                        stride, (const double2 *)wt, (const double2 *)am, (const double2 *)an, (const double2 *)ie,
                        (const double *)vc, out));
  }
  if (env->host) BGW_CUDA_TRY(cudaMemcpyAsync(achtemp, out, 6 * sizeof(double), cudaMemcpyDeviceToHost, env->stream));
  env->prof.flops = 63.0 * (double)nb * (double)P * (double)G;
  return finish_call(env);
}

extern "C" int bgw_gpp_sigma(int64_t number_bands, int64_t nvband, int64_t ngpown, int64_t ncouls,
                             const int32_t *inv_igp_index, const int32_t *indinv, int64_t indinv_len,
                             const double *wx_array, const double *wtilde_array, const double *aqsmtemp,
                             const double *aqsntemp, const double *I_eps_array, const double *vcoul,
                             double *achtemp, double *asxtemp, const bgw_options *opt) {
  const int64_t nb = number_bands, P = ngpown, G = ncouls;
  if (nb < 0 || P < 0 || G <= 0 || G > INT32_MAX || nb > INT32_MAX || P > INT32_MAX) return BGW_ERR_INVALID_ARG;
  if (nvband < 0 || nvband > nb) return BGW_ERR_INVALID_ARG;
  if (!dims_ok(nb, G) || !dims_ok(P, G) || indinv_len <= 0 || indinv_len > INT32_MAX) return BGW_ERR_INVALID_ARG;
  if ((!achtemp && !asxtemp) || !vcoul || !indinv) return BGW_ERR_INVALID_ARG;
  if (P > 0 && (!inv_igp_index || !wtilde_array || !I_eps_array)) return BGW_ERR_INVALID_ARG;
  if (nb > 0 && P > 0 && (!aqsmtemp || !aqsntemp)) return BGW_ERR_INVALID_ARG;
  Call c(opt);
  if (c.st != BGW_OK) return c.st;
  CallEnv *env = &c.env;
  const int64_t stride = env->opt.wx_band_stride;
  if (!wx_array && (nb > 0 || stride == 0)) return BGW_ERR_INVALID_ARG;
  if (stride != 0 && stride < 3) return BGW_ERR_INVALID_ARG;
  const size_t wx_n = !wx_array ? 0 : stride == 0 ? 3 : (size_t)(nb > 0 ? (nb - 1) * stride + 3 : 3);
  // Both sums read the same inputs: stage them once (host memory: copied,
  // large pageable arrays through the page-locked slots).
  const void *inv = nullptr, *ind = nullptr, *wx = nullptr, *wt = nullptr, *am = nullptr, *an = nullptr,
             *ie = nullptr, *vc = nullptr;
  const size_t pg = (size_t)P * (size_t)G * 16, ng = (size_t)nb * (size_t)G * 16;
  BGW_TRY(stage_input(env, SLOT_IN0, inv_igp_index, sizeof(int32_t) * (size_t)P, &inv));
  BGW_TRY(stage_input(env, SLOT_IN1, indinv, sizeof(int32_t) * (size_t)indinv_len, &ind));
  BGW_TRY(stage_input(env, SLOT_IN2, wx_array, sizeof(double) * wx_n, &wx));
  BGW_TRY(stage_input(env, SLOT_IN3, wtilde_array, pg, &wt));
  BGW_TRY(stage_input(env, SLOT_IN4, aqsmtemp, ng, &am));
  BGW_TRY(stage_input(env, SLOT_IN5, aqsntemp, ng, &an));
  BGW_TRY(stage_input(env, SLOT_IN6, I_eps_array, pg, &ie));
  BGW_TRY(stage_input(env, SLOT_IN7, vcoul, sizeof(double) * (size_t)G, &vc));
  double *out = nullptr;  // achtemp | asxtemp (6 doubles each)
  BGW_TRY(out_buffer(env, nullptr, 12 * sizeof(double), &out));
  double *o_ach = env->host ? out : achtemp, *o_asx = env->host ? out + 6 : asxtemp;
  const bool factored = env->opt.gpp_algorithm == BGW_GPP_FACTORED ||
                        (env->opt.gpp_algorithm == BGW_GPP_AUTO && stride == 0 &&
                         env->opt.precision == BGW_PRECISION_FP64);
  if (factored && (stride != 0 || env->opt.precision != BGW_PRECISION_FP64)) return BGW_ERR_UNSUPPORTED;
  if (factored && asxtemp && P > 0) {
    // Both outputs in one pass over wtilde / I_eps.
    BGW_TRY(gpp_sigma_factored_enqueue(env, nb, nvband, P, G, (const int32_t *)inv, (const int32_t *)ind,
                                       indinv_len, (const double *)wx, (const double2 *)wt, (const double2 *)am,
                                       (const double2 *)an, (const double2 *)ie, (const double *)vc,
                                       achtemp ? o_ach : nullptr, o_asx));
  } else {
    if (achtemp)
      BGW_TRY(gpp_enqueue(env, nb, P, G, (const int32_t *)inv, (const int32_t *)ind, indinv_len,
                          (const double *)wx, stride, (const double2 *)wt, (const double2 *)am, (const double2 *)an,
                          (const double2 *)ie, (const double *)vc, o_ach));
    if (asxtemp)
      BGW_TRY(gpp_sx_enqueue(env, nvband, P, G, (const int32_t *)inv, (const int32_t *)ind, indinv_len,
                             (const double *)wx, wx_n, stride, (const double2 *)wt, (const double2 *)am,
                             (const double2 *)an, (const double2 *)ie, (const double *)vc, o_asx));
  }
  if (env->host) {
    if (achtemp) BGW_CUDA_TRY(cudaMemcpyAsync(achtemp, o_ach, 6 * sizeof(double), cudaMemcpyDeviceToHost, env->stream));
    if (asxtemp) BGW_CUDA_TRY(cudaMemcpyAsync(asxtemp, o_asx, 6 * sizeof(double), cudaMemcpyDeviceToHost, env->stream));
  }
  env->prof.flops = 63.0 * (double)P * (double)G * ((achtemp ? (double)nb : 0.0) + (asxtemp ? 2.0 * nvband : 0.0));
  return finish_call(env);
}

extern "C" int bgw_noflagOCC_solver_backward(int64_t number_bands, int64_t ngpown, int64_t ncouls,
                                             const int32_t *inv_igp_index, const int32_t *indinv,
                                             int64_t indinv_len, const double *wx_array, const double *wtilde_array,
                                             const double *aqsmtemp, const double *aqsntemp,
                                             const double *I_eps_array, const double *vcoul,
                                             const double *grad_achtemp, double *grad_wtilde, double *grad_I_eps,
                                             double *dachtemp_domega, const bgw_options *opt) {
  const int64_t nb = number_bands, P = ngpown, G = ncouls;
  if (nb < 0 || P < 0 || G <= 0 || G > INT32_MAX || nb > INT32_MAX || P > INT32_MAX) return BGW_ERR_INVALID_ARG;
  if (!dims_ok(nb, G) || !dims_ok(P, G) || indinv_len <= 0 || indinv_len > INT32_MAX) return BGW_ERR_INVALID_ARG;
  if (!grad_achtemp || !wx_array || !vcoul || !indinv) return BGW_ERR_INVALID_ARG;
  if (!grad_wtilde && !grad_I_eps && !dachtemp_domega) return BGW_ERR_INVALID_ARG;
  if (P > 0 && (!inv_igp_index || !wtilde_array || !I_eps_array)) return BGW_ERR_INVALID_ARG;
  if (nb > 0 && P > 0 && (!aqsmtemp || !aqsntemp)) return BGW_ERR_INVALID_ARG;
  Call c(opt);
  if (c.st != BGW_OK) return c.st;
  CallEnv *env = &c.env;
  if (env->opt.pole_guard > 0.0) return BGW_ERR_UNSUPPORTED;  // no near-pole cut-off
  const int64_t stride = env->opt.wx_band_stride;
  if (stride != 0 && stride < 3) return BGW_ERR_INVALID_ARG;
  // The factored adjoint needs a band-independent wx; the band loop takes any.
  const bool bandloop = stride != 0 || env->opt.gpp_algorithm == BGW_GPP_BANDLOOP;
  const size_t wx_n = stride == 0 ? 3 : (size_t)(nb > 0 ? (nb - 1) * stride + 3 : 3);
  const void *inv = nullptr, *ind = nullptr, *wx = nullptr, *wt = nullptr, *am = nullptr, *an = nullptr,
             *ie = nullptr, *vc = nullptr, *gc = nullptr;
  const size_t pg = (size_t)P * (size_t)G * 16, ng = (size_t)nb * (size_t)G * 16;
  BGW_TRY(stage_input(env, SLOT_IN0, inv_igp_index, sizeof(int32_t) * (size_t)P, &inv));
  BGW_TRY(stage_input(env, SLOT_IN1, indinv, sizeof(int32_t) * (size_t)indinv_len, &ind));
  BGW_TRY(stage_input(env, SLOT_IN2, wx_array, sizeof(double) * wx_n, &wx));
  BGW_TRY(stage_input(env, SLOT_IN3, wtilde_array, pg, &wt));
  BGW_TRY(stage_input(env, SLOT_IN4, aqsmtemp, ng, &am));
  BGW_TRY(stage_input(env, SLOT_IN5, aqsntemp, ng, &an));
  BGW_TRY(stage_input(env, SLOT_IN6, I_eps_array, pg, &ie));
  BGW_TRY(stage_input(env, SLOT_IN7, vcoul, sizeof(double) * (size_t)G, &vc));
  BGW_TRY(stage_input(env, SLOT_IN8, grad_achtemp, sizeof(double) * 6, &gc));
  double *d_gw = grad_wtilde, *d_gi = grad_I_eps, *d_dw = dachtemp_domega;
  if (env->host) {
    void *p = nullptr;
    if (grad_wtilde) {
      BGW_TRY(ws_reserve(env->ws, SLOT_IN9, pg, &p));
      d_gw = static_cast<double *>(p);
    }
    if (grad_I_eps) {
      BGW_TRY(ws_reserve(env->ws, SLOT_IN10, pg, &p));
      d_gi = static_cast<double *>(p);
    }
    if (dachtemp_domega) {
      BGW_TRY(ws_reserve(env->ws, SLOT_IN11, sizeof(double) * 6, &p));
      d_dw = static_cast<double *>(p);
    }
  } else if (((uintptr_t)grad_wtilde | (uintptr_t)grad_I_eps) & 15u) {
    return BGW_ERR_INVALID_ARG;
  }
  if (bandloop)
    BGW_TRY(gpp_adjoint_bandloop_enqueue(env, nb, P, G, (const int32_t *)inv, (const int32_t *)ind, indinv_len,
                                         (const double *)wx, stride, (const double2 *)wt, (const double2 *)am,
                                         (const double2 *)an, (const double2 *)ie, (const double *)vc,
                                         (const double2 *)gc, (double2 *)d_gw, (double2 *)d_gi, d_dw));
  else
    BGW_TRY(gpp_adjoint_enqueue(env, nb, P, G, (const int32_t *)inv, (const int32_t *)ind, indinv_len,
                                (const double *)wx, (const double2 *)wt, (const double2 *)am, (const double2 *)an,
                                (const double2 *)ie, (const double *)vc, (const double2 *)gc, (double2 *)d_gw,
                                (double2 *)d_gi, d_dw));
  if (env->host) {
    if (grad_wtilde) BGW_CUDA_TRY(cudaMemcpyAsync(grad_wtilde, d_gw, pg, cudaMemcpyDeviceToHost, env->stream));
    if (grad_I_eps) BGW_CUDA_TRY(cudaMemcpyAsync(grad_I_eps, d_gi, pg, cudaMemcpyDeviceToHost, env->stream));
    if (dachtemp_domega)
      BGW_CUDA_TRY(cudaMemcpyAsync(dachtemp_domega, d_dw, sizeof(double) * 6, cudaMemcpyDeviceToHost, env->stream));
  }
  // Algorithmic flops: per (G', G, frequency) element (factored) or per
  // (band, G', G, frequency) term (band loop) the quotient (as the forward)
  // plus 4 complex products; 21 + 24 = 45.
  env->prof.flops = 45.0 * 3.0 * (double)P * (double)G * (bandloop ? (double)nb : 1.0);
  return finish_call(env);
}

namespace {

// Shared body of the three FF entry points and bgw_ff_sigma.
int ff_call(int64_t nb, int64_t nvband, int64_t nE, int64_t G, int64_t P, int64_t nFreq, double fmin, double fstep,
            double occ, const double *ekq, const double *grid, const int32_t *inv, const int32_t *indinv,
            int64_t indinv_len, const double *aqsm, const double *aqsn, const double *vcoul, const double *R,
            const double *A, double *achs, double *asx, double *cor, const bgw_options *opt) {
  if (nb < 0 || nvband < 0 || nE < 0 || P < 0 || G <= 0 || nFreq < 2) return BGW_ERR_INVALID_ARG;
  if (nb > INT32_MAX || P > INT32_MAX || G > INT32_MAX || nFreq > INT32_MAX || nE > INT32_MAX)
    return BGW_ERR_INVALID_ARG;
  if (P > G) return BGW_ERR_INVALID_ARG;  // the reference driver's guard, ff.cpp:492-499
  if ((asx || cor) && nvband > nb) return BGW_ERR_INVALID_ARG;
  if (!dims_ok(nb, G) || !dims_ok(nFreq, P) || !dims_ok(nFreq * P, G) || indinv_len <= 0 ||
      indinv_len > INT32_MAX)
    return BGW_ERR_INVALID_ARG;
  const bool want_achs = achs != nullptr, want_asx = asx != nullptr, want_cor = cor != nullptr;
  if (!want_achs && !want_asx && !want_cor) return BGW_ERR_INVALID_ARG;
  if (!indinv || !vcoul || (P > 0 && !inv)) return BGW_ERR_INVALID_ARG;
  if (nb > 0 && (!aqsm || !aqsn)) return BGW_ERR_INVALID_ARG;
  if ((want_asx || want_cor) && (!ekq || !grid || !R || !A)) return BGW_ERR_INVALID_ARG;
  if (want_achs && !R) return BGW_ERR_INVALID_ARG;

  Call c(opt);
  if (c.st != BGW_OK) return c.st;
  CallEnv *env = &c.env;

  // Band classification needs ekq and dFreqGrid on the host.
  const int64_t ne = (want_asx || want_cor) ? nb : 0;
  std::vector<double> ekq_h((size_t)std::max<int64_t>(ne, 1)), grid_h((size_t)nFreq);
  if (ne > 0 || want_asx || want_cor) {
    if (env->host) {
      if (ne) std::memcpy(ekq_h.data(), ekq, sizeof(double) * (size_t)ne);
      std::memcpy(grid_h.data(), grid, sizeof(double) * (size_t)nFreq);
    } else {
      if (ne)
        BGW_CUDA_TRY(cudaMemcpyAsync(ekq_h.data(), ekq, sizeof(double) * (size_t)ne, cudaMemcpyDeviceToHost,
                                     env->stream));
      BGW_CUDA_TRY(cudaMemcpyAsync(grid_h.data(), grid, sizeof(double) * (size_t)nFreq, cudaMemcpyDeviceToHost,
                                   env->stream));
      BGW_CUDA_TRY(cudaStreamSynchronize(env->stream));
    }
  }
  FFPlan plan;
  const bool per_iw = (env->opt.flags & BGW_FLAG_FF_WX_PER_IW) != 0;
  BGW_TRY(ff_make_plan(env, nb, nvband, P, G, nFreq, fmin, fstep, occ, ekq_h.data(), grid_h.data(), want_achs,
                       want_asx, want_cor, per_iw, nE, &plan));

  const size_t slice = (size_t)P * (size_t)G * 16;
  const size_t ng = (size_t)nb * (size_t)G * 16;
  const void *d_inv = nullptr, *d_ind = nullptr, *d_am = nullptr, *d_an = nullptr, *d_vc = nullptr;
  const void *d_R = nullptr, *d_A = nullptr;
  int r_f0 = 0, a_f0 = 0;
  BGW_TRY(stage_input(env, SLOT_IN0, inv, sizeof(int32_t) * (size_t)P, &d_inv));
  BGW_TRY(stage_input(env, SLOT_IN1, indinv, sizeof(int32_t) * (size_t)indinv_len, &d_ind));
  BGW_TRY(stage_input(env, SLOT_IN2, aqsm, ng, &d_am));
  BGW_TRY(stage_input(env, SLOT_IN3, aqsn, ng, &d_an));
  BGW_TRY(stage_input(env, SLOT_IN4, vcoul, sizeof(double) * (size_t)G, &d_vc));
  if (plan.r_hi >= plan.r_lo) {
    if (env->host) {
      r_f0 = plan.r_lo;
      BGW_TRY(stage_input(env, SLOT_IN5, R + (size_t)plan.r_lo * slice / 8,
                          slice * (size_t)(plan.r_hi - plan.r_lo + 1), &d_R));
    } else {
      BGW_TRY(stage_input(env, SLOT_IN5, R, slice, &d_R));
    }
  }
  if (plan.a_hi >= plan.a_lo) {
    if (env->host) {
      a_f0 = plan.a_lo;
      BGW_TRY(stage_input(env, SLOT_IN6, A + (size_t)plan.a_lo * slice / 8,
                          slice * (size_t)(plan.a_hi - plan.a_lo + 1), &d_A));
    } else {
      BGW_TRY(stage_input(env, SLOT_IN6, A, slice, &d_A));
    }
  }
  // Outputs: achs (2) | asx (2 nE) | cor (2 nE) doubles.
  double *o_achs = nullptr, *o_asx = nullptr, *o_cor = nullptr;
  if (env->host) {
    double *o = nullptr;
    BGW_TRY(out_buffer(env, nullptr, sizeof(double) * (2 + 4 * (size_t)nE), &o));
    o_achs = want_achs ? o : nullptr;
    o_asx = want_asx ? o + 2 : nullptr;
    o_cor = want_cor ? o + 2 + 2 * nE : nullptr;
  } else {
    o_achs = achs;
    o_asx = asx;
    o_cor = cor;
  }
  const int64_t nb_w = (want_achs || want_cor) ? nb : nvband;
  // Mixed precision: the fused kernel (digits cut inside the tensor-core
  // kernel) unless the staged path is asked for, which cuts both operands
  // into digit buffers first.
  const bool staged = (env->opt.flags & BGW_FLAG_FF_STAGED) != 0;
  if (env->opt.precision == BGW_PRECISION_MIXED && !staged)
    BGW_TRY(ff_launch_fused(env, plan, nb_w, nE, G, P, (const int32_t *)d_inv, (const int32_t *)d_ind, indinv_len,
                            (const double2 *)d_am, (const double2 *)d_an, (const double *)d_vc,
                            (const double2 *)d_R, r_f0, (const double2 *)d_A, a_f0,
                            (env->opt.flags & BGW_FLAG_FF_SLICE_ALL) ? 1 : 0, o_achs, o_asx, o_cor));
  else if (env->opt.precision == BGW_PRECISION_MIXED)
    BGW_TRY(ff_launch_mixed(env, plan, nb, nb_w, nE, G, P, (const int32_t *)d_inv, (const int32_t *)d_ind,
                            indinv_len, (const double2 *)d_am, (const double2 *)d_an, (const double *)d_vc,
                            (const double2 *)d_R, r_f0, (const double2 *)d_A, a_f0, o_achs, o_asx, o_cor));
  else
    BGW_TRY(ff_launch(env, plan, nb_w, nE, G, P, (const int32_t *)d_inv, (const int32_t *)d_ind, indinv_len,
                      (const double2 *)d_am, (const double2 *)d_an, (const double *)d_vc, (const double2 *)d_R,
                      r_f0, (const double2 *)d_A, a_f0, o_achs, o_asx, o_cor));
  if (env->host) {
    if (want_achs)
      BGW_CUDA_TRY(cudaMemcpyAsync(achs, o_achs, 2 * sizeof(double), cudaMemcpyDeviceToHost, env->stream));
    if (want_asx && nE)
      BGW_CUDA_TRY(cudaMemcpyAsync(asx, o_asx, 2 * sizeof(double) * nE, cudaMemcpyDeviceToHost, env->stream));
    if (want_cor && nE)
      BGW_CUDA_TRY(cudaMemcpyAsync(cor, o_cor, 2 * sizeof(double) * nE, cudaMemcpyDeviceToHost, env->stream));
  }
  return finish_call(env);
}

}  // namespace

extern "C" int bgw_achsDtemp_Kernel(int64_t number_bands, int64_t ngpown, int64_t ncouls,
                                    const int32_t *inv_igp_index, const int32_t *indinv, int64_t indinv_len,
                                    const double *aqsntemp, const double *aqsmtemp, const double *I_epsR_array,
                                    int64_t nFreq, const double *vcoul, double *achsDtemp, const bgw_options *opt) {
  if (!achsDtemp) return BGW_ERR_INVALID_ARG;
  return ff_call(number_bands, 0, 0, ncouls, ngpown, nFreq, 0.0, 0.0, 0.0, nullptr, nullptr, inv_igp_index, indinv,
                 indinv_len, aqsmtemp, aqsntemp, vcoul, I_epsR_array, nullptr, achsDtemp, nullptr, nullptr, opt);
}

extern "C" int bgw_asxDtemp_Kernel(int64_t nvband, int64_t nfreqeval, int64_t ncouls, int64_t ngpown,
                                   int64_t nFreq, double freqevalmin, double freqevalstep, double occ,
                                   const double *ekq, const double *dFreqGrid, const int32_t *inv_igp_index,
                                   const int32_t *indinv, int64_t indinv_len, const double *aqsmtemp,
                                   const double *aqsntemp, int64_t number_bands, const double *vcoul,
                                   const double *I_epsR_array, const double *I_epsA_array, double *asxDtemp,
                                   const bgw_options *opt) {
  if (!asxDtemp && nfreqeval > 0) return BGW_ERR_INVALID_ARG;
  double dummy[2];
  return ff_call(number_bands, nvband, nfreqeval, ncouls, ngpown, nFreq, freqevalmin, freqevalstep, occ, ekq,
                 dFreqGrid, inv_igp_index, indinv, indinv_len, aqsmtemp, aqsntemp, vcoul, I_epsR_array,
                 I_epsA_array, nullptr, nfreqeval > 0 ? asxDtemp : dummy, nullptr, opt);
}

extern "C" int bgw_achDtemp_cor_Kernel(int64_t number_bands, int64_t nvband, int64_t nfreqeval, int64_t ncouls,
                                       int64_t ngpown, int64_t nFreq, double freqevalmin, double freqevalstep,
                                       const double *ekq, const double *dFreqGrid, const int32_t *inv_igp_index,
                                       const int32_t *indinv, int64_t indinv_len, const double *aqsmtemp,
                                       const double *aqsntemp, const double *vcoul, const double *I_epsR_array,
                                       const double *I_epsA_array, double *achDtemp_cor, const bgw_options *opt) {
  if (!achDtemp_cor && nfreqeval > 0) return BGW_ERR_INVALID_ARG;
  double dummy[2];
  return ff_call(number_bands, nvband, nfreqeval, ncouls, ngpown, nFreq, freqevalmin, freqevalstep, 1.0, ekq,
                 dFreqGrid, inv_igp_index, indinv, indinv_len, aqsmtemp, aqsntemp, vcoul, I_epsR_array,
                 I_epsA_array, nullptr, nullptr, nfreqeval > 0 ? achDtemp_cor : dummy, opt);
}

extern "C" int bgw_ff_sigma(int64_t number_bands, int64_t nvband, int64_t nfreqeval, int64_t ncouls, int64_t ngpown,
                            int64_t nFreq, double freqevalmin, double freqevalstep, double occ, const double *ekq,
                            const double *dFreqGrid, const int32_t *inv_igp_index, const int32_t *indinv,
                            int64_t indinv_len, const double *aqsmtemp, const double *aqsntemp, const double *vcoul,
                            const double *I_epsR_array, const double *I_epsA_array, double *achsDtemp,
                            double *asxDtemp, double *achDtemp_cor, const bgw_options *opt) {
  return ff_call(number_bands, nvband, nfreqeval, ncouls, ngpown, nFreq, freqevalmin, freqevalstep, occ, ekq,
                 dFreqGrid, inv_igp_index, indinv, indinv_len, aqsmtemp, aqsntemp, vcoul, I_epsR_array,
                 I_epsA_array, achsDtemp, asxDtemp, achDtemp_cor, opt);
}

extern "C" int bgw_fill_uniform(double *out, int64_t n, uint64_t seed, uint64_t stream, int64_t offset,
                                double lo_even, double hi_even, double lo_odd, double hi_odd,
                                const bgw_options *opt) {
  if (n < 0 || offset < 0 || offset > INT64_MAX - n - 4) return BGW_ERR_INVALID_ARG;
  if (n > 0 && !out) return BGW_ERR_INVALID_ARG;
  if (!std::isfinite(lo_even) || !std::isfinite(hi_even) || !std::isfinite(lo_odd) || !std::isfinite(hi_odd))
    return BGW_ERR_INVALID_ARG;
  Call c(opt);
  if (c.st != BGW_OK) return c.st;
  CallEnv *env = &c.env;
  if (!env->host) {
    BGW_TRY(fill_uniform_enqueue(env, out, n, seed, stream, offset, lo_even, hi_even, lo_odd, hi_odd));
    return finish_call(env);
  }
  // Host memory: generated on the GPU in 32 MiB pieces, each copied back
  // before the next is generated into the same buffer (same stream).
  constexpr int64_t kPiece = int64_t(4) << 20;  // doubles
  void *buf = nullptr;
  BGW_TRY(ws_reserve(env->ws, SLOT_OUT, sizeof(double) * (size_t)std::min<int64_t>(std::max<int64_t>(n, 1), kPiece),
                     &buf));
  for (int64_t i = 0; i < n; i += kPiece) {
    const int64_t m = std::min<int64_t>(kPiece, n - i);
    BGW_TRY(fill_uniform_enqueue(env, static_cast<double *>(buf), m, seed, stream, offset + i, lo_even, hi_even,
                                 lo_odd, hi_odd));
    BGW_CUDA_TRY(cudaMemcpyAsync(out + i, buf, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost, env->stream));
  }
  return finish_call(env);
}
