// extern "C" boundary of the Laplace engine and the INLA fit driver, plus
// the hyperprior densities used by the configurations.
#include <cmath>
#include <cstring>
#include <memory>

#include "aggregate.hpp"
#include "aggregate_dev.hpp"
#include "capi_common.hpp"
#include "driver.hpp"
#include "marginals.hpp"
#include "model_select.hpp"
#include "posterior.hpp"
#include "inla_b200.h"

using namespace inla;

struct inla_laplace {
  cudaStream_t stream = nullptr;
  std::unique_ptr<LaplaceEngine> eng;
  LaplaceSpec spec;  // the caller's model, before any constraint augmentation
  int max_batch = 0;
  // from the last inla_fit: linear predictor moments and the model-selection inputs
  std::vector<double> pred_mean, pred_var, cond_eta, cond_eta_var, node_weight, cond_mean, cond_var, node_theta;
  std::vector<double> coef_mode;
  int mode_index = 0, m = 0;
  double p1scale_mode = 1.0, mlik_gaussian = 0.0;
  bool fitted = false;
  double phase_s[4] = {0.0, 0.0, 0.0, 0.0};
  // device copies of cond_eta / cond_eta_var: the criteria of the fit are computed on the device
  DBuf<double> d_cond_eta, d_cond_eta_var;
  AggScratch agg;
};

namespace {

// pc.cor1 rate from P(rho > u) = alpha (priors.rs:611-660): coarse scan of lambda, then 60
// golden-section steps on the squared residual; NaN when the residual stays above 1e-6.
double pc_cor1_lambda(double u, double alpha) {
  if (!(u > -1.0 && u < 1.0)) return NAN;
  const double amin = std::sqrt((1.0 - u) / 2.0);
  if (!(alpha > amin && alpha < 1.0)) return NAN;
  auto fun = [&](double lam) {
    const double ff = (1.0 - std::exp(-lam * std::sqrt(1.0 - u))) / (1.0 - std::exp(-lam * M_SQRT2));
    return (ff - alpha) * (ff - alpha);
  };
  double best = 1.0, bf = fun(best);
  for (int i = 0; i < 110; ++i) {
    const double lam = i < 100 ? 1e-7 + (10.0 - 1e-7) * i / 99.0 : 10.0 + 90.0 * (i - 100) / 9.0;
    const double f = fun(lam);
    if (f < bf) bf = f, best = lam;
  }
  double lo = std::max(best * 0.5, 1e-8), hi = best * 2.0;
  for (int it = 0; it < 60; ++it) {
    const double m1 = lo + 0.382 * (hi - lo), m2 = lo + 0.618 * (hi - lo);
    if (fun(m1) < fun(m2)) hi = m2;
    else lo = m1;
  }
  const double lam = 0.5 * (lo + hi);
  return fun(lam) > 1e-6 ? NAN : lam;
}

// log density of pc.cor1 on theta with rho = 2 e^theta / (1 + e^theta) - 1 (priors.rs:662-683)
double pc_cor1_theta(double th, double lam) {
  const double e = std::exp(th), rho = 2.0 * e / (1.0 + e) - 1.0;
  if (!(rho > -1.0 && rho < 1.0)) return NAN;
  const double s = std::sqrt(1.0 - rho);
  return std::log(lam) - lam * s - std::log(1.0 - std::exp(-M_SQRT2 * lam)) - std::log(2.0 * s) + M_LN2 + th -
         2.0 * std::log1p(e);
}

// priors.rs:532-548 (pc.prec), 813-834 (pc.spde, d = 2), 836-855 (loggamma), 611-704 (pc.cor1)
double prior_one(const inla_prior_spec& s, const double* th, double* g) {
  switch (s.kind) {
    case INLA_PRIOR_PC_COR1: {
      const double lam = pc_cor1_lambda(s.p[0], s.p[1]);
      const double t = th[s.slot];
      const double v = pc_cor1_theta(t, lam);
      if (g) {
        const double e = std::exp(t), rho = 2.0 * e / (1.0 + e) - 1.0;
        const double sq = std::sqrt(std::max(1.0 - rho, 0.0));
        if (sq < 1e-8) {  // central difference near rho = 1 (priors.rs:690-696)
          const double h = 1e-5;
          g[s.slot] += (pc_cor1_theta(t + h, lam) - pc_cor1_theta(t - h, lam)) / (2.0 * h);
        } else {
          g[s.slot] += (lam * sq + 1.0) * (1.0 + rho) / 4.0 - rho;
        }
      }
      return v;
    }
    case INLA_PRIOR_PC_PREC: {
      const double lam = -std::log(s.p[1]) / s.p[0];
      const double e = std::exp(-0.5 * th[s.slot]);
      if (g) g[s.slot] += 0.5 * lam * e - 0.5;
      return std::log(lam) - M_LN2 - lam * e - 0.5 * th[s.slot];
    }
    case INLA_PRIOR_LOGGAMMA: {
      const double a = s.p[0], b = s.p[1], e = std::exp(th[s.slot]);
      if (g) g[s.slot] += a - b * e;
      return a * std::log(b) - std::lgamma(a) + a * th[s.slot] - b * e;
    }
    case INLA_PRIOR_PC_SPDE: {
      const double d = 2.0, dh = d / 2.0;
      const double lam1 = -std::log(s.p[1]) * std::pow(s.p[0], dh);
      const double lam2 = -std::log(s.p[3]) / s.p[2];
      const double t1 = th[s.slot], t2 = th[s.slot + 1];
      const double log_rho = 0.5 * std::log(8.0) - t2;
      const double log_sigma = -0.5 * std::log(4.0 * M_PI) - t1 - t2;
      const double er = std::exp(-dh * log_rho), es = std::exp(log_sigma);
      const double s_rho = std::log(lam1 * dh) - dh * log_rho - lam1 * er;
      const double s_sig = std::log(lam2) + log_sigma - lam2 * es;
      if (g) {
        const double dsr = -dh + lam1 * dh * er;  // d s_rho / d log_rho
        const double dss = 1.0 - lam2 * es;       // d s_sig / d log_sigma
        g[s.slot] += -dss;
        g[s.slot + 1] += -dsr - dss;
      }
      return s_rho + s_sig;
    }
    case INLA_PRIOR_GAUSSIAN: {
      const double mu = s.p[0], prec = s.p[1], r = th[s.slot] - mu;
      if (g) g[s.slot] += -prec * r;
      return -0.9189385332046728 + 0.5 * std::log(prec) - 0.5 * prec * r * r;
    }
  }
  return NAN;
}

}  // namespace

extern "C" {

double inla_prior_log_density(const inla_prior_spec* specs, int nspec, const double* theta, int m, double* grad) {
  if (grad)
    for (int i = 0; i < m; ++i) grad[i] = 0.0;
  double s = 0.0;
  for (int k = 0; k < nspec; ++k) {
    const int need = specs[k].kind == INLA_PRIOR_PC_SPDE ? 2 : 1;
    if (specs[k].slot < 0 || specs[k].slot + need > m) return NAN;
    s += prior_one(specs[k], theta, grad);
  }
  return s;
}

double inla_log_prior_set(const double* theta, int m, double* grad, void* user) {
  const inla_prior_set* ps = (const inla_prior_set*)user;
  if (!ps || ps->nspec < 0 || ps->nspec > 8) return NAN;
  return inla_prior_log_density(ps->specs, ps->nspec, theta, m, grad);
}

int inla_theta_map_spde(const double* theta, int m, double* coef, double* dcoef, double* p1scale, double* dp1scale,
                        void* user) {
  (void)user;
  // theta = [log prec_eps, log tau, log kappa]; Q = tau^2 (kappa^4 C + 2 kappa^2 G + G C^-1 G)
  if (m != 3) return 1;
  const double t2 = std::exp(2.0 * theta[1]), k2 = std::exp(2.0 * theta[2]);
  const double c[3] = {t2 * k2 * k2, 2.0 * t2 * k2, t2};
  for (int t = 0; t < 3; ++t) coef[t] = c[t];
  if (dcoef) {
    // rows: d/d theta_0, theta_1, theta_2
    for (int t = 0; t < 3; ++t) dcoef[t] = 0.0;
    for (int t = 0; t < 3; ++t) dcoef[3 + t] = 2.0 * c[t];
    dcoef[6] = 4.0 * c[0];
    dcoef[7] = 2.0 * c[1];
    dcoef[8] = 0.0;
  }
  *p1scale = std::exp(theta[0]);
  if (dp1scale) {
    dp1scale[0] = *p1scale;
    dp1scale[1] = dp1scale[2] = 0.0;
  }
  return std::isfinite(c[0]) && std::isfinite(*p1scale) && c[2] > 0.0 ? 0 : 1;
}

int inla_laplace_create(int64_t n, const int64_t* colptr, const int64_t* rowidx, int ncomp, const double* comp,
                        int64_t nobs, const int64_t* a_rowptr, const int64_t* a_colidx, const double* a_vals,
                        int family, const double* y, const double* p1, const double* p2, int ordering, int max_batch,
                        inla_laplace** out) {
  inla_laplace* h = nullptr;
  try {
    if (!out || !colptr || !rowidx || !comp || !y || n <= 0 || nobs <= 0 || max_batch < 1)
      return fail(INLA_ERR_INVALID, "invalid argument");
    LaplaceSpec sp;
    sp.n = n;
    sp.colptr.assign(colptr, colptr + n + 1);
    const int64_t nnz = colptr[n];
    sp.rowidx.assign(rowidx, rowidx + nnz);
    sp.ncomp = ncomp;
    sp.comp.assign(comp, comp + (size_t)ncomp * nnz);
    sp.nobs = nobs;
    sp.identity_a = a_rowptr == nullptr;
    if (!sp.identity_a) {
      sp.acp.assign(a_rowptr, a_rowptr + nobs + 1);
      sp.aci.assign(a_colidx, a_colidx + a_rowptr[nobs]);
      sp.av.assign(a_vals, a_vals + a_rowptr[nobs]);
    }
    sp.family = family;
    sp.y.assign(y, y + nobs);
    if (p1) sp.p1.assign(p1, p1 + nobs);
    if (p2) sp.p2.assign(p2, p2 + nobs);
    sp.ordering = ordering;
    h = new inla_laplace();
    INLA_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->eng.reset(new LaplaceEngine(sp, max_batch, h->stream));
    h->spec = std::move(sp);
    h->max_batch = max_batch;
    *out = h;
    return INLA_OK;
  } catch (...) {
    int code = map_exception();
    inla_laplace_free(h);
    return code;
  }
}

void inla_laplace_free(inla_laplace* h) {
  if (!h) return;
  h->eng.reset();
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int inla_laplace_set_constraints(inla_laplace* h, int k, const double* c, const double* e, int method) {
  try {
    if (!h || !h->eng) return fail(INLA_ERR_INVALID, "null handle");
    if (k < 0 || (k > 0 && (!c || !e))) return fail(INLA_ERR_INVALID, "invalid constraint arguments");
    if (method < INLA_CONSTR_AUTO || method > INLA_CONSTR_BORDERED)
      return fail(INLA_ERR_INVALID, "unknown constraint method");
    const int64_t n = h->spec.n;
    LaplaceSpec sp = h->spec;
    sp.kc = k;
    sp.cA.assign(c ? c : nullptr, c ? c + (size_t)k * n : nullptr);
    sp.ce.assign(e ? e : nullptr, e ? e + k : nullptr);
    sp.cmethod = method;
    const LaplaceSpec& prev = h->eng->spec();
    LaplaceSpec keep = h->spec;  // previous constraints, restored if the new set is rejected
    keep.kc = prev.kc;
    keep.cA = prev.cA;
    keep.ce = prev.ce;
    keep.cmethod = prev.cmethod;
    INLA_CUDA(cudaStreamSynchronize(h->stream));
    h->eng.reset();
    try {
      h->eng.reset(new LaplaceEngine(sp, h->max_batch, h->stream));
    } catch (...) {
      int code = map_exception();
      try {
        h->eng.reset(new LaplaceEngine(keep, h->max_batch, h->stream));
      } catch (...) {
        h->eng.reset();
      }
      return code;
    }
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_laplace_eval(inla_laplace* h, int B, const double* coef, const double* p1scale, int flags, double* scalars,
                      double* x, double* var, double* grad_terms) {
  try {
    if (!h || !h->eng) return fail(INLA_ERR_INVALID, "null handle");
    LaplaceEngine& E = *h->eng;
    if (B < 1 || B > E.max_batch()) return fail(INLA_ERR_DIM_MISMATCH, "batch size out of range");
    if (var) flags |= LAP_VARIANCES;
    LaplaceOut R;
    int64_t before = E.launches();
    E.eval(B, coef, p1scale, flags, R);
    g_launches += E.launches() - before;
    const int T1 = E.ncomp() + 1;
    for (int b = 0; b < B; ++b) {
      double* s = scalars + (size_t)b * 8;
      s[0] = R.mlik[b];
      s[1] = R.ld_prior[b];
      s[2] = R.ld_post[b];
      s[3] = R.loglik[b];
      s[4] = R.quad[b];
      s[5] = R.iters[b];
      s[6] = R.status[b];
      s[7] = R.dll[b];
      if (grad_terms) {
        double* gt = grad_terms + (size_t)b * 4 * T1;
        std::memcpy(gt, &R.trP[(size_t)b * T1], sizeof(double) * T1);
        std::memcpy(gt + T1, &R.trQ[(size_t)b * T1], sizeof(double) * T1);
        std::memcpy(gt + 2 * T1, &R.xMx[(size_t)b * T1], sizeof(double) * T1);
        std::memcpy(gt + 3 * T1, &R.zMx[(size_t)b * T1], sizeof(double) * T1);
      }
    }
    const size_t w = sizeof(double) * E.n(), pitch = sizeof(double) * E.xstride();
    if (x) INLA_CUDA(cudaMemcpy2DAsync(x, w, E.d_x(), pitch, w, B, cudaMemcpyDeviceToHost, E.stream()));
    if (var) INLA_CUDA(cudaMemcpy2DAsync(var, w, E.d_var(), pitch, w, B, cudaMemcpyDeviceToHost, E.stream()));
    INLA_CUDA(cudaStreamSynchronize(E.stream()));
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_fit(inla_laplace* h, int m, const double* theta0, inla_theta_map_fn map, inla_log_prior_fn prior,
             void* user, const inla_fit_options* opt, double* mode, double* hessian, double* latent_mean,
             double* latent_var, double* node_theta, double* node_weight, double* info) {
  try {
    if (!h || !h->eng || (!theta0 && m > 0) || !map || !prior || !opt || m < 0 || m > 5 || opt->mode_search < 0 ||
        opt->mode_search > 3)
      return fail(INLA_ERR_INVALID, "invalid argument");
    LaplaceEngine& E = *h->eng;
    ThetaMap tm = [&](const double* th, double* c, double* dc, double* s, double* ds) {
      return map(th, m, c, dc, s, ds, user);
    };
    LogPrior lp = [&](const double* th, double* g) { return prior(th, m, g, user); };
    InlaDriver drv(E, m, tm, lp);
    FitOptions fo;
    fo.mode_search = opt->mode_search;
    fo.batched = opt->batched;
    fo.strategy = opt->strategy;
    fo.f0 = opt->f0 > 0 ? opt->f0 : 1.0;
    fo.hessian = opt->hessian;
    fo.max_iter = opt->max_iter > 0 ? opt->max_iter : (opt->mode_search ? 100 : 200);
    fo.tol = opt->tol > 0 ? opt->tol : (opt->mode_search ? 1e-4 : 1e-6);
    fo.nm_step = opt->nm_step > 0 ? opt->nm_step : 0.1;
    if (opt->cancel) {
      inla_cancel_fn cf = opt->cancel;
      void* cu = opt->cancel_user;
      fo.cancel = [cf, cu] { return cf(cu) != 0; };
    }
    FitResult R;
    R.d_cond_eta = &h->d_cond_eta;
    R.d_cond_eta_var = &h->d_cond_eta_var;
    int64_t before = E.launches();
    drv.fit(theta0, fo, R);
    g_launches += E.launches() - before;
    const int64_t n = E.n();
    const int K = (int)R.node_theta.size() / std::max(m, 1);  // m = 0: no integration nodes
    if (mode && m > 0) std::memcpy(mode, R.mode.data(), sizeof(double) * m);
    if (hessian && m > 0) std::memcpy(hessian, R.hessian.data(), sizeof(double) * m * m);
    if (latent_mean) std::memcpy(latent_mean, R.latent_mean.data(), sizeof(double) * n);
    if (latent_var) std::memcpy(latent_var, R.latent_var.data(), sizeof(double) * n);
    if (node_theta) std::memcpy(node_theta, R.node_theta.data(), sizeof(double) * std::min(K, 64) * m);
    if (node_weight) std::memcpy(node_weight, R.node_weight.data(), sizeof(double) * std::min(K, 64));
    if (info) {
      info[0] = R.mlik;
      info[1] = R.seconds;
      info[2] = R.n_evals;
      info[3] = R.n_batches;
      info[4] = R.mode_iters;
      info[5] = K;
    }
    h->pred_mean = std::move(R.pred_mean);
    h->pred_var = std::move(R.pred_var);
    h->cond_eta = std::move(R.cond_eta);
    h->cond_eta_var = std::move(R.cond_eta_var);
    h->node_weight = R.node_weight;
    h->cond_mean = std::move(R.cond_mean);
    h->cond_var = std::move(R.cond_var);
    h->node_theta = R.node_theta;
    h->coef_mode = R.coef_mode;
    h->m = m;
    h->mode_index = R.mode_index;
    h->p1scale_mode = R.p1scale_mode;
    h->mlik_gaussian = R.mlik_gaussian;
    std::memcpy(h->phase_s, R.phase_s, sizeof(h->phase_s));
    h->fitted = true;
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_fit_phase_seconds(inla_laplace* h, double* out4) {
  if (!h || !h->fitted || !out4) return fail(INLA_ERR_INVALID, "inla_fit_phase_seconds: no fit on this handle");
  std::memcpy(out4, h->phase_s, sizeof(h->phase_s));
  return INLA_OK;
}

int inla_fit_predictor(inla_laplace* h, double* pred_mean, double* pred_var) {
  if (!h || !h->fitted) return fail(INLA_ERR_INVALID, "inla_fit_predictor: no fit on this handle");
  const size_t bytes = sizeof(double) * h->pred_mean.size();
  if (pred_mean) std::memcpy(pred_mean, h->pred_mean.data(), bytes);
  if (pred_var) std::memcpy(pred_var, h->pred_var.data(), bytes);
  return INLA_OK;
}

namespace {

void fill_crit(const ModelSelection& ms, double mlik_g, double* crit, double* cpo, double* pit, int64_t nobs,
               int what) {
  if (crit) {
    crit[0] = ms.dic;
    crit[1] = ms.mean_deviance;
    crit[2] = ms.dic_p_eff;
    crit[3] = ms.waic;
    crit[4] = ms.lppd;
    crit[5] = ms.waic_p_eff;
    crit[6] = mlik_g;
    crit[7] = (what & MS_CPO) ? (double)ms.cpo_failures : NAN;
  }
  for (int64_t i = 0; i < nobs; ++i) {
    if (cpo) cpo[i] = (what & MS_CPO) ? ms.cpo[i] : NAN;
    if (pit) pit[i] = (what & MS_CPO) ? ms.pit[i] : NAN;
  }
}

}  // namespace

int inla_fit_model_selection(inla_laplace* h, int what, double* crit, double* cpo, double* pit) {
  try {
    if (!h || !h->fitted) return fail(INLA_ERR_INVALID, "inla_fit_model_selection: no fit on this handle");
    const LaplaceSpec& S = h->spec;
    ObsView obs;
    obs.family = S.family;
    obs.nobs = S.nobs;
    obs.y = S.y.data();
    obs.p1 = S.p1.empty() ? nullptr : S.p1.data();
    obs.p2 = S.p2.empty() ? nullptr : S.p2.data();
    obs.p1scale = h->p1scale_mode;
    ModelSelection ms;
    std::string err;
    if (h->eng && h->d_cond_eta.p) {  // on the device, from the fit's per-node predictors
      const LaplaceEngine& E = *h->eng;
      DevObs dobs;
      dobs.family = S.family;
      dobs.nobs = S.nobs;
      dobs.y = E.d_y();
      dobs.p1 = E.d_p1();
      dobs.p2 = E.d_p2();
      dobs.p1scale = h->p1scale_mode;
      err = dev_model_selection(E.stream(), dobs, (int)h->node_weight.size(), h->node_weight.data(), h->mode_index,
                                h->d_cond_eta.p, h->d_cond_eta_var.p, what, h->agg, ms);
    } else {
      err = model_selection(obs, (int)h->node_weight.size(), h->node_weight.data(), h->mode_index,
                            h->cond_eta.data(), h->cond_eta_var.data(), what, ms);
    }
    if (!err.empty()) return fail(INLA_ERR_INVALID, err.c_str());
    fill_crit(ms, h->mlik_gaussian, crit, cpo, pit, S.nobs, what);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

namespace {

int copy_block(const CscBlock& b, int64_t* nnz, int64_t* colptr, int64_t* rowidx, double* vals) {
  if (nnz) *nnz = (int64_t)b.rowidx.size();
  if (colptr) std::memcpy(colptr, b.colptr.data(), sizeof(int64_t) * b.colptr.size());
  if (rowidx) std::memcpy(rowidx, b.rowidx.data(), sizeof(int64_t) * b.rowidx.size());
  if (vals) std::memcpy(vals, b.val.data(), sizeof(double) * b.val.size());
  return INLA_OK;
}

}  // namespace

int inla_fit_posterior_precision(inla_laplace* h, int64_t* nnz, int64_t* colptr, int64_t* rowidx, double* vals) {
  try {
    if (!h || !h->fitted) return fail(INLA_ERR_INVALID, "inla_fit_posterior_precision: no fit on this handle");
    const LaplaceSpec& S = h->spec;
    const int K = (int)h->node_weight.size();
    if ((int)h->coef_mode.size() != S.ncomp || K < 1)
      return fail(INLA_ERR_INVALID, "inla_fit_posterior_precision: the theta map failed at the mode");
    const int64_t n = S.n;
    if (!h->eng || (int64_t)h->cond_mean.size() < (int64_t)(h->mode_index + 1) * n)
      return fail(INLA_ERR_INVALID, "inla_fit_posterior_precision: no node results");
    const double* x = h->cond_mean.data() + (size_t)h->mode_index * n;
    const LaplaceSpec& E = h->eng->spec();  // the constraints in force (the base spec has none)
    CscBlock q;
    const std::string err = posterior_precision(
        n, S.colptr.data(), S.rowidx.data(), S.ncomp, S.comp.data(), h->coef_mode.data(), S.nobs,
        S.identity_a ? nullptr : S.acp.data(), S.aci.data(), S.av.data(), S.family, S.y.data(),
        S.p1.empty() ? nullptr : S.p1.data(), S.p2.empty() ? nullptr : S.p2.data(), x, E.kc,
        E.kc > 0 ? E.cA.data() : nullptr, q);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    return copy_block(q, nnz, colptr, rowidx, vals);
  } catch (...) {
    return map_exception();
  }
}

int inla_posterior_precision(int64_t n, const int64_t* colptr, const int64_t* rowidx, int ncomp, const double* comp,
                             const double* coef, int64_t nobs, const int64_t* a_rowptr, const int64_t* a_colidx,
                             const double* a_vals, int family, const double* y, const double* p1, const double* p2,
                             const double* x, int kc, const double* c, int64_t* nnz, int64_t* colptr_out,
                             int64_t* rowidx_out, double* vals) {
  try {
    if (n <= 0 || !colptr || !rowidx || ncomp < 1 || !comp || !coef || !x || nobs < 0 || (nobs > 0 && !y) ||
        family < 0 || family > 3 || kc < 0 || (kc > 0 && !c))
      return fail(INLA_ERR_INVALID, "inla_posterior_precision: invalid argument");
    if (colptr[0] != 0) return fail(INLA_ERR_INVALID, "inla_posterior_precision: colptr[0] must be 0");
    for (int64_t j = 0; j < n; ++j) {
      if (colptr[j + 1] < colptr[j]) return fail(INLA_ERR_INVALID, "inla_posterior_precision: colptr not monotone");
      for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p)
        if (rowidx[p] < 0 || rowidx[p] >= n) return fail(INLA_ERR_INVALID, "inla_posterior_precision: row index");
    }
    if (!a_rowptr) {
      if (nobs != n) return fail(INLA_ERR_DIM_MISMATCH, "inla_posterior_precision: A = I needs nobs == n");
    } else {
      if (!a_colidx || !a_vals || a_rowptr[0] != 0) return fail(INLA_ERR_INVALID, "inla_posterior_precision: A");
      for (int64_t r = 0; r < nobs; ++r) {
        if (a_rowptr[r + 1] < a_rowptr[r]) return fail(INLA_ERR_INVALID, "inla_posterior_precision: A row pointer");
        for (int64_t p = a_rowptr[r]; p < a_rowptr[r + 1]; ++p)
          if (a_colidx[p] < 0 || a_colidx[p] >= n)
            return fail(INLA_ERR_DIM_MISMATCH, "inla_posterior_precision: A column out of range");
      }
    }
    CscBlock q;
    const std::string err = posterior_precision(n, colptr, rowidx, ncomp, comp, coef, nobs, a_rowptr, a_colidx,
                                                a_vals, family, y, p1, p2, x, kc, c, q);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    return copy_block(q, nnz, colptr_out, rowidx_out, vals);
  } catch (...) {
    return map_exception();
  }
}

int inla_fit_marginal(inla_laplace* h, int kind, int64_t index, int n_points, double n_sd, double* x, double* y) {
  try {
    if (!h || !h->fitted) return fail(INLA_ERR_INVALID, "inla_fit_marginal: no fit on this handle");
    if (!x || !y || kind < 0 || kind > 2) return fail(INLA_ERR_INVALID, "inla_fit_marginal: invalid argument");
    const int K = (int)h->node_weight.size();
    std::vector<double> mk(K), vk(K);
    std::string err;
    if (kind == 2) {
      if (index < 0 || index >= h->m) return fail(INLA_ERR_INVALID, "hyperparameter index out of range");
      for (int k = 0; k < K; ++k) mk[k] = h->node_theta[(size_t)k * h->m + index];
      err = hyperpar_marginal(K, mk.data(), h->node_weight.data(), n_points, n_sd, x, y);
    } else {
      const std::vector<double>& cm = kind == 0 ? h->cond_mean : h->cond_eta;
      const std::vector<double>& cv = kind == 0 ? h->cond_var : h->cond_eta_var;
      const int64_t len = (int64_t)cm.size() / std::max(K, 1);
      if (index < 0 || index >= len)
        return fail(INLA_ERR_INVALID, kind == 0 ? "latent marginal index out of range"
                                                : "predictor marginal index out of range");
      for (int k = 0; k < K; ++k) {
        mk[k] = cm[(size_t)k * len + index];
        vk[k] = cv[(size_t)k * len + index];
      }
      err = mixture_marginal(K, mk.data(), vk.data(), h->node_weight.data(), n_points, n_sd, x, y);
    }
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_mixture_marginal(int K, const double* means, const double* vars, const double* weights, int n_points,
                          double n_sd, double* x, double* y) {
  if (K < 0 || (K > 0 && (!means || !vars || !weights)) || !x || !y)
    return fail(INLA_ERR_INVALID, "inla_mixture_marginal: invalid argument");
  const std::string err = mixture_marginal(K, means, vars, weights, n_points, n_sd, x, y);
  return err.empty() ? INLA_OK : fail(INLA_ERR_INVALID, err);
}

int inla_hyperpar_marginal(int K, const double* theta, const double* weights, int n_points, double n_sd, double* x,
                           double* y) {
  if (K < 0 || (K > 0 && (!theta || !weights)) || !x || !y)
    return fail(INLA_ERR_INVALID, "inla_hyperpar_marginal: invalid argument");
  const std::string err = hyperpar_marginal(K, theta, weights, n_points, n_sd, x, y);
  return err.empty() ? INLA_OK : fail(INLA_ERR_INVALID, err);
}

int inla_marginal_quantiles(int n, const double* x, const double* y, int np, const double* probs, double* q) {
  if (n < 0 || np < 0 || (n > 0 && (!x || !y)) || (np > 0 && (!probs || !q)))
    return fail(INLA_ERR_INVALID, "inla_marginal_quantiles: invalid argument");
  const std::string err = marginal_quantiles(n, x, y, np, probs, q);
  return err.empty() ? INLA_OK : fail(INLA_ERR_INVALID, err);
}

int inla_model_selection(int family, int64_t nobs, const double* y, const double* p1, const double* p2, int K,
                         const double* weight, int mode_index, const double* cond_eta, const double* cond_eta_var,
                         int what, double* crit, double* cpo, double* pit) {
  try {
    if (family < 0 || family > 3 || nobs < 0 || (nobs > 0 && !y) || K < 1 || !weight || mode_index < 0 ||
        mode_index >= K || (nobs > 0 && (!cond_eta || !cond_eta_var)))
      return fail(INLA_ERR_INVALID, "inla_model_selection: invalid argument");
    ObsView obs;
    obs.family = family;
    obs.nobs = nobs;
    obs.y = y;
    obs.p1 = p1;
    obs.p2 = p2;
    ModelSelection ms;
    const std::string err = model_selection(obs, K, weight, mode_index, cond_eta, cond_eta_var, what, ms);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err.c_str());
    fill_crit(ms, NAN, crit, cpo, pit, nobs, what);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_mlik_gaussian(double log_post_mode, int m, const double* neg_hessian, double* out) {
  if (m < 0 || (m > 0 && !neg_hessian) || !out) return fail(INLA_ERR_INVALID, "inla_mlik_gaussian: invalid argument");
  if (!mlik_gaussian(log_post_mode, m, neg_hessian, *out))
    return fail(INLA_ERR_NOT_PD, "negative Hessian is not positive-definite");
  return INLA_OK;
}

int inla_observation_cdf(int family, double y, double p1, double eta, double variance, double* out) {
  if (!out) return fail(INLA_ERR_INVALID, "inla_observation_cdf: invalid argument");
  return observation_cdf(family, y, p1, eta, variance, *out) ? INLA_OK
                                                              : fail(INLA_ERR_INVALID, "no CDF for this family");
}

int inla_cpo_failure(int family, double y, double p1, double p2, double mu, double var) {
  return cpo_failure(family, y, p1, p2, mu, var) ? 1 : 0;
}

int inla_predictor_moments(int64_t nobs, int64_t n, const int64_t* a_rowptr, const int64_t* a_colidx,
                           const double* a_vals, int K, const double* weight, const double* cond_mean,
                           const double* cond_var, double* pred_mean, double* pred_var) {
  try {
    if (n < 0 || K < 1 || !weight || !cond_mean || !cond_var || !pred_mean || !pred_var)
      return fail(INLA_ERR_INVALID, "inla_predictor_moments: invalid argument");
    if (!a_rowptr) {
      if (nobs != n) return fail(INLA_ERR_DIM_MISMATCH, "inla_predictor_moments: eta = x needs nobs == n");
    } else {
      if (nobs < 0 || !a_colidx || !a_vals || a_rowptr[0] != 0)
        return fail(INLA_ERR_INVALID, "inla_predictor_moments: invalid CSR");
      for (int64_t r = 0; r < nobs; ++r)
        if (a_rowptr[r + 1] < a_rowptr[r]) return fail(INLA_ERR_INVALID, "inla_predictor_moments: invalid CSR");
      for (int64_t p = 0; p < a_rowptr[nobs]; ++p)
        if (a_colidx[p] < 0 || a_colidx[p] >= n)
          return fail(INLA_ERR_DIM_MISMATCH, "inla_predictor_moments: column out of range");
    }
    predictor_moments(nobs, n, a_rowptr, a_colidx, a_vals, K, weight, cond_mean, cond_var, pred_mean, pred_var);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// device forms of the post-node aggregation (caller's device buffers)
// ---------------------------------------------------------------------------

namespace {
AggScratch& thread_agg_scratch() {
  static thread_local AggScratch sc;
  return sc;
}
}  // namespace

int inla_predictor_moments_dev(int64_t nobs, int64_t n, const int64_t* d_a_rowptr, const int* d_a_colidx,
                               const double* d_a_vals, int K, const double* d_weight, const double* d_cond_mean,
                               const double* d_cond_var, double* d_cond_eta, double* d_cond_eta_var,
                               double* d_pred_mean, double* d_pred_var, void* stream) {
  try {
    if (nobs < 1 || n < 1 || K < 1 || !d_weight || !d_cond_mean || !d_cond_var || !d_cond_eta || !d_cond_eta_var ||
        !d_pred_mean || !d_pred_var || (d_a_rowptr && (!d_a_colidx || !d_a_vals)) || (!d_a_rowptr && nobs != n))
      return fail(INLA_ERR_INVALID, "inla_predictor_moments_dev: invalid argument");
    cudaStream_t st = (cudaStream_t)stream;
    DevCsrA A;
    A.rp = d_a_rowptr;
    A.ci = d_a_colidx;
    A.v = d_a_vals;
    dev_project_nodes(st, nobs, A, K, d_cond_mean, n, d_cond_var, n, d_cond_eta, d_cond_eta_var);
    dev_mixture_moments(st, K, nobs, d_weight, d_cond_eta, nobs, d_cond_eta_var, nobs, d_pred_mean, d_pred_var);
    g_launches += 2;
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_model_selection_dev(int family, int64_t nobs, const double* d_y, const double* d_p1, const double* d_p2,
                             int K, const double* weight, int mode_index, const double* d_cond_eta,
                             const double* d_cond_eta_var, int what, double* crit, double* cpo, double* pit,
                             void* stream) {
  try {
    if (family < 0 || family > 3 || nobs < 0 || (nobs > 0 && !d_y) || K < 1 || !weight || mode_index < 0 ||
        mode_index >= K || (nobs > 0 && (!d_cond_eta || !d_cond_eta_var)))
      return fail(INLA_ERR_INVALID, "inla_model_selection_dev: invalid argument");
    DevObs obs;
    obs.family = family;
    obs.nobs = nobs;
    obs.y = d_y;
    obs.p1 = d_p1;
    obs.p2 = d_p2;
    ModelSelection ms;
    const std::string err = dev_model_selection((cudaStream_t)stream, obs, K, weight, mode_index, d_cond_eta,
                                                d_cond_eta_var, what, thread_agg_scratch(), ms);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err.c_str());
    fill_crit(ms, NAN, crit, cpo, pit, nobs, what);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}
