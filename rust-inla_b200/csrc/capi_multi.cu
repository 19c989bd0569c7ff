// extern "C" boundary of the multi-model Laplace engine (independent models of uneven size).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "capi_common.hpp"
#include "inla_b200.h"
#include "model_select.hpp"
#include "multi.hpp"

using namespace inla;

struct inla_multi {
  cudaStream_t stream = nullptr;
  std::unique_ptr<MultiLaplace> eng;
  std::vector<double> pred_mean, pred_var;  // linear predictor moments of the last inla_multi_fit
  MultiFitResult last;                      // its model-selection inputs (moved from the fit)
  int m = 0;
  bool fitted = false;
};

extern "C" {

int inla_multi_create(int G, const int64_t* lat_off, const int64_t* obs_off, const int64_t* colptr,
                      const int64_t* rowidx, int ncomp, const double* comp, const int64_t* a_rowptr,
                      const int64_t* a_colidx, const double* a_vals, int family, const double* y, const double* p1,
                      const double* p2, int ordering, int max_batch, inla_multi** out) {
  inla_multi* h = nullptr;
  try {
    if (!out || G < 1 || !lat_off || !obs_off || !colptr || !rowidx || !comp || !a_rowptr || max_batch < 1)
      return fail(INLA_ERR_INVALID, "invalid argument");
    MultiSpec sp;
    sp.G = G;
    sp.lat_off.assign(lat_off, lat_off + G + 1);
    sp.obs_off.assign(obs_off, obs_off + G + 1);
    sp.n = lat_off[G];
    sp.nobs = obs_off[G];
    if (sp.n <= 0 || sp.nobs < 0) return fail(INLA_ERR_INVALID, "invalid offsets");
    if (ncomp < 1 || ncomp > 8) return fail(INLA_ERR_INVALID, "1..8 precision components supported");
    if (ordering < 0 || ordering > INLA_ORDER_ND || ordering == INLA_ORDER_CUSTOM)
      return fail(INLA_ERR_INVALID, "unsupported ordering");
    if (sp.nobs > 0 && (!y || !a_colidx || !a_vals)) return fail(INLA_ERR_INVALID, "null observation arrays");
    sp.colptr.assign(colptr, colptr + sp.n + 1);
    sp.rowidx.assign(rowidx, rowidx + colptr[sp.n]);
    sp.ncomp = ncomp;
    sp.comp.assign(comp, comp + (size_t)ncomp * colptr[sp.n]);
    sp.acp.assign(a_rowptr, a_rowptr + sp.nobs + 1);
    if (sp.nobs > 0) {
      sp.aci.assign(a_colidx, a_colidx + a_rowptr[sp.nobs]);
      sp.av.assign(a_vals, a_vals + a_rowptr[sp.nobs]);
      sp.y.assign(y, y + sp.nobs);
      if (p1) sp.p1.assign(p1, p1 + sp.nobs);
      if (p2) sp.p2.assign(p2, p2 + sp.nobs);
    }
    sp.family = family;
    sp.ordering = ordering;
    h = new inla_multi();
    INLA_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->eng.reset(new MultiLaplace(sp, max_batch, h->stream));
    *out = h;
    return INLA_OK;
  } catch (...) {
    int code = map_exception();
    inla_multi_free(h);
    return code;
  }
}

void inla_multi_free(inla_multi* h) {
  if (!h) return;
  h->eng.reset();
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int inla_multi_eval(inla_multi* h, int B, const double* coef, const double* p1scale, int flags, double* scalars,
                    double* x, double* var, double* grad_terms) {
  try {
    if (!h || !h->eng) return fail(INLA_ERR_INVALID, "null handle");
    MultiLaplace& E = *h->eng;
    if (B < 1 || B > E.max_batch()) return fail(INLA_ERR_DIM_MISMATCH, "batch size out of range");
    if (!coef || !scalars) return fail(INLA_ERR_INVALID, "null coefficient or output array");
    if (var) flags |= LAP_VARIANCES;
    MultiOut R;
    const int64_t before = E.launches();
    E.eval(B, coef, p1scale, flags, R);
    g_launches += E.launches() - before;
    const size_t BG = (size_t)B * E.G();
    const int T1 = E.ncomp() + 1;
    for (size_t q = 0; q < BG; ++q) {
      double* s = scalars + q * 8;
      s[0] = R.mlik[q];
      s[1] = R.ld_prior[q];
      s[2] = R.ld_post[q];
      s[3] = R.loglik[q];
      s[4] = R.quad[q];
      s[5] = R.iters[q];
      s[6] = R.status[q];
      s[7] = R.dll[q];
      if (grad_terms) {
        double* gt = grad_terms + q * 4 * T1;
        std::memcpy(gt, &R.trP[q * T1], sizeof(double) * T1);
        std::memcpy(gt + T1, &R.trQ[q * T1], sizeof(double) * T1);
        std::memcpy(gt + 2 * T1, &R.xMx[q * T1], sizeof(double) * T1);
        std::memcpy(gt + 3 * T1, &R.zMx[q * T1], sizeof(double) * T1);
      }
    }
    if (x) INLA_CUDA(cudaMemcpyAsync(x, E.d_x(), sizeof(double) * B * E.n(), cudaMemcpyDeviceToHost, E.stream()));
    if (var) INLA_CUDA(cudaMemcpyAsync(var, E.d_var(), sizeof(double) * B * E.n(), cudaMemcpyDeviceToHost, E.stream()));
    INLA_CUDA(cudaStreamSynchronize(E.stream()));
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_multi_fit(inla_multi* h, int m, const double* theta0, inla_multi_theta_map_fn map,
                   inla_multi_log_prior_fn prior, void* user, const inla_multi_fit_options* opt, double* mode,
                   double* hessian, double* mlik, double* latent_mean, double* latent_var, int* mode_iters,
                   int* status, double* info) {
  try {
    if (!h || !h->eng || !theta0 || !map || !prior || m < 1 || m > 5)
      return fail(INLA_ERR_INVALID, "invalid argument");
    MultiLaplace& E = *h->eng;
    MultiThetaMap tm = [&](int g, const double* th, double* c, double* dc, double* s, double* ds) {
      return map(g, th, m, c, dc, s, ds, user);
    };
    MultiLogPrior lp = [&](int g, const double* th, double* gr) { return prior(g, th, m, gr, user); };
    MultiDriver drv(E, m, tm, lp);
    MultiFitOptions fo;
    if (opt) {
      fo.hessian = opt->hessian;
      if (opt->f0 > 0) fo.f0 = opt->f0;
      if (opt->max_iter > 0) fo.max_iter = opt->max_iter;
      if (opt->tol > 0) fo.tol = opt->tol;
      if (opt->cancel) {
        inla_cancel_fn cf = opt->cancel;
        void* cu = opt->cancel_user;
        fo.cancel = [cf, cu] { return cf(cu) != 0; };
      }
    }
    MultiFitResult R;
    const int64_t before = E.launches();
    drv.fit(theta0, fo, R);
    g_launches += E.launches() - before;
    const int G = E.G();
    const int64_t n = E.n();
    if (mode) std::memcpy(mode, R.mode.data(), sizeof(double) * G * m);
    if (hessian) std::memcpy(hessian, R.hessian.data(), sizeof(double) * G * m * m);
    if (mlik) std::memcpy(mlik, R.mlik.data(), sizeof(double) * G);
    if (latent_mean) std::memcpy(latent_mean, R.latent_mean.data(), sizeof(double) * n);
    if (latent_var) std::memcpy(latent_var, R.latent_var.data(), sizeof(double) * n);
    if (mode_iters) std::memcpy(mode_iters, R.mode_iters.data(), sizeof(int) * G);
    if (status) std::memcpy(status, R.status.data(), sizeof(int) * G);
    if (info) {
      info[0] = R.seconds;
      info[1] = R.n_batches;
      info[2] = (double)R.n_model_evals;
    }
    h->pred_mean = std::move(R.pred_mean);
    h->pred_var = std::move(R.pred_var);
    h->last = std::move(R);
    h->m = m;
    h->fitted = true;
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_multi_fit_predictor(inla_multi* h, double* pred_mean, double* pred_var) {
  if (!h || !h->fitted) return fail(INLA_ERR_INVALID, "inla_multi_fit_predictor: no fit on this handle");
  const size_t bytes = sizeof(double) * h->pred_mean.size();
  if (pred_mean) std::memcpy(pred_mean, h->pred_mean.data(), bytes);
  if (pred_var) std::memcpy(pred_var, h->pred_var.data(), bytes);
  return INLA_OK;
}

int inla_multi_fit_model_selection(inla_multi* h, int g, int what, double* crit, double* cpo, double* pit) {
  try {
    if (!h || !h->fitted) return fail(INLA_ERR_INVALID, "inla_multi_fit_model_selection: no fit on this handle");
    const MultiFitResult& R = h->last;
    const MultiSpec& S = h->eng->spec();
    if (g < 0 || g >= S.G) return fail(INLA_ERR_INVALID, "inla_multi_fit_model_selection: model out of range");
    const int K = R.K;
    const double* w = &R.node_weight[(size_t)g * K];
    bool any = false;
    for (int k = 0; k < K; ++k) any |= w[k] != 0.0;
    if (!any) return fail(INLA_ERR_NONCONVERGED, "Newton-Raphson did not converge at any integration node");
    const int64_t o0 = S.obs_off[g], len = S.obs_off[g + 1] - o0;
    std::vector<double> ce((size_t)K * len), cv((size_t)K * len);
    for (int k = 0; k < K; ++k)
      for (int64_t r = 0; r < len; ++r) {
        ce[(size_t)k * len + r] = R.cond_eta[(size_t)k * S.nobs + o0 + r];
        cv[(size_t)k * len + r] = R.cond_eta_var[(size_t)k * S.nobs + o0 + r];
      }
    ObsView obs;
    obs.family = S.family;
    obs.nobs = len;
    obs.y = S.y.data() + o0;
    obs.p1 = S.p1.empty() ? nullptr : S.p1.data() + o0;
    obs.p2 = S.p2.empty() ? nullptr : S.p2.data() + o0;
    obs.p1scale = R.p1scale_mode[g];
    ModelSelection ms;
    const std::string err = model_selection(obs, K, w, R.mode_index, ce.data(), cv.data(), what, ms);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    const int m = h->m;
    std::vector<double> neg((size_t)m * m);
    for (int i = 0; i < m * m; ++i) neg[i] = -R.hessian[(size_t)g * m * m + i];
    double mg = NAN;
    if (!mlik_gaussian(R.logpost_mode[g], m, neg.data(), mg)) mg = NAN;
    if (crit) {
      crit[0] = ms.dic;
      crit[1] = ms.mean_deviance;
      crit[2] = ms.dic_p_eff;
      crit[3] = ms.waic;
      crit[4] = ms.lppd;
      crit[5] = ms.waic_p_eff;
      crit[6] = mg;
      crit[7] = (what & MS_CPO) ? (double)ms.cpo_failures : NAN;
    }
    for (int64_t r = 0; r < len; ++r) {
      if (cpo) cpo[r] = (what & MS_CPO) ? ms.cpo[r] : NAN;
      if (pit) pit[r] = (what & MS_CPO) ? ms.pit[r] : NAN;
    }
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_multi_theta_map_ar1_iid(int g, const double* theta, int m, double* coef, double* dcoef, double* p1scale,
                                 double* dp1scale, void* user) {
  (void)g;
  (void)user;
  // theta = [log tau, logit-type rho, log tau_iid]; components [M_int, K0, K1, K2, M_iid] with
  // the AR1 conditional precision tau (K0 + rho^2 K1 - rho K2) (ar1.rs:9-69, structured.rs:348-356)
  if (m != 3) return 1;
  const double tau = std::exp(theta[0]);
  const double rho_raw = 2.0 / (1.0 + std::exp(-theta[1])) - 1.0;
  const double rho = std::min(std::max(rho_raw, -0.999), 0.999);
  const double drho = rho == rho_raw ? (1.0 - rho_raw * rho_raw) / 2.0 : 0.0;
  const double ti = std::exp(theta[2]);
  const double c[5] = {1.0, tau, tau * rho * rho, -tau * rho, ti};
  for (int t = 0; t < 5; ++t) coef[t] = c[t];
  if (dcoef) {
    for (int i = 0; i < 15; ++i) dcoef[i] = 0.0;
    dcoef[1] = c[1];
    dcoef[2] = c[2];
    dcoef[3] = c[3];
    dcoef[5 + 2] = tau * 2.0 * rho * drho;
    dcoef[5 + 3] = -tau * drho;
    dcoef[10 + 4] = ti;
  }
  *p1scale = 1.0;
  if (dp1scale) dp1scale[0] = dp1scale[1] = dp1scale[2] = 0.0;
  return std::isfinite(tau) && std::isfinite(ti) && tau > 0.0 && ti > 0.0 ? 0 : 1;
}

double inla_multi_log_prior_set(int g, const double* theta, int m, double* grad, void* user) {
  (void)g;
  return inla_log_prior_set(theta, m, grad, user);
}

}  // extern "C"
