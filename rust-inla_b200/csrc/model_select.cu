// Host code (no kernels): the model-selection criteria of an INLA fit. Compiled as CUDA
// source only to share the likelihood code of the device kernels (likelihood.cuh).
#include <algorithm>
#include <cmath>
#include <limits>

#include "host_par.hpp"
#include "likelihood.cuh"
#include "model_select.hpp"
#include "model_select_core.cuh"

namespace inla {

namespace {

struct Lik {
  double logp, grad, hess;
};

// eval_likelihood for observation i of `obs` at eta; false where the reference returns Err.
bool lik_at(const ObsView& obs, int64_t i, double eta, Lik& out) {
  double dw;
  const double q1 = (obs.p1 ? obs.p1[i] : 1.0) * obs.p1scale, q2 = obs.p2 ? obs.p2[i] : 1.0;
  return d_eval_lik(obs.family, eta, obs.y[i], q1, q2, out.logp, out.grad, out.hess, dw) == 0;
}

}  // namespace

bool observation_cdf(int family, double y, double p1, double eta, double variance, double& out) {
  return ms_observation_cdf(family, y, p1, eta, variance, out);
}

double normal_cdf(double x) { return ms_normal_cdf(x); }

double poisson_cdf(double lambda, uint64_t k) { return ms_poisson_cdf(lambda, k); }

double binomial_cdf(uint64_t n, double p, uint64_t k) { return ms_binomial_cdf(n, p, k); }

bool cpo_failure(int family, double y, double p1, double p2, double mu, double var) {
  return ms_cpo_failure(family, y, p1, p2, mu, var);
}

bool mlik_gaussian(double log_post_mode, int m, const double* neg_hessian, double& out) {
  if (m == 0) {
    out = log_post_mode;
    return true;
  }
  std::vector<double> a(neg_hessian, neg_hessian + (size_t)m * m);
  double log_det = 0.0;
  for (int j = 0; j < m; ++j) {
    for (int k = 0; k < j; ++k) {
      const double ljk = a[j * m + k];
      a[j * m + j] -= ljk * ljk;
    }
    if (a[j * m + j] <= 0.0) return false;
    log_det += std::log(a[j * m + j]);
    const double djj = std::sqrt(a[j * m + j]);
    a[j * m + j] = djj;
    for (int i = j + 1; i < m; ++i) {
      for (int k = 0; k < j; ++k) a[i * m + j] -= a[i * m + k] * a[j * m + k];
      a[i * m + j] /= djj;
    }
  }
  out = log_post_mode + 0.5 * (double)m * std::log(2.0 * 3.14159265358979323846) - 0.5 * log_det;
  return true;
}

std::string model_selection(const ObsView& obs, int K, const double* w, int mode_index, const double* cond_eta,
                            const double* cond_eta_var, int what, ModelSelection& out) {
  const int64_t n = obs.nobs;
  if (K < 1 || mode_index < 0 || mode_index >= K) return "model selection: invalid node count or mode index";
  out = ModelSelection();
  const double NaN = std::numeric_limits<double>::quiet_NaN();

  if (what & (MS_DIC | MS_WAIC)) {
    // log-likelihood of every (node, observation); ok[k][i] = 0 where the reference returns Err
    std::vector<double> ll((size_t)K * n);
    std::vector<char> ok((size_t)K * n);
    parallel_for(n, [&](int64_t i0, int64_t i1) {
      Lik e;
      for (int k = 0; k < K; ++k)
        for (int64_t i = i0; i < i1; ++i) {
          const bool good = lik_at(obs, i, cond_eta[(size_t)k * n + i], e);
          ok[(size_t)k * n + i] = good;
          ll[(size_t)k * n + i] = good ? e.logp : NaN;
        }
    }, 4096);
    if (what & MS_DIC) {  // compute_dic (model_selection.rs:101-150), node-major like the reference
      std::vector<double> dev(K);
      for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) {
          if (!ok[(size_t)k * n + i]) return "DIC: likelihood evaluation failed at observation " + std::to_string(i);
          s += ll[(size_t)k * n + i];
        }
        dev[k] = -2.0 * s;
      }
      double mean_dev = 0.0;
      for (int k = 0; k < K; ++k) mean_dev += w[k] * dev[k];
      out.mean_deviance = mean_dev;
      out.dic_p_eff = mean_dev - dev[mode_index];
      out.dic = mean_dev + out.dic_p_eff;
    }
    if (what & MS_WAIC) {  // compute_waic (model_selection.rs:152-211)
      std::vector<double> lppd_i(n), pw_i(n);
      std::vector<char> bad(n, 0);
      parallel_for(n, [&](int64_t i0, int64_t i1) {
        for (int64_t i = i0; i < i1; ++i) {
          double mx = -std::numeric_limits<double>::infinity();
          for (int k = 0; k < K; ++k) {
            if (!ok[(size_t)k * n + i]) {
              bad[i] = 1;
              break;
            }
            mx = std::fmax(mx, ll[(size_t)k * n + i]);
          }
          if (bad[i]) continue;
          double sum_w_exp = 0.0, mean_ll = 0.0;
          for (int k = 0; k < K; ++k) {
            const double l = ll[(size_t)k * n + i];
            sum_w_exp += w[k] * std::exp(l - mx);
            mean_ll += w[k] * l;
          }
          if (!(std::isfinite(sum_w_exp) && sum_w_exp > 0.0)) {
            bad[i] = 2;
            continue;
          }
          lppd_i[i] = mx + std::log(sum_w_exp);
          double v = 0.0;
          for (int k = 0; k < K; ++k) {
            const double d = ll[(size_t)k * n + i] - mean_ll;
            v += w[k] * d * d;
          }
          pw_i[i] = v;
        }
      }, 4096);
      double lppd = 0.0, p_waic = 0.0;
      for (int64_t i = 0; i < n; ++i) {
        if (bad[i] == 1) return "WAIC: likelihood evaluation failed at observation " + std::to_string(i);
        if (bad[i] == 2) return "WAIC: non-finite predictive density at obs " + std::to_string(i);
        lppd += lppd_i[i];
        p_waic += pw_i[i];
      }
      out.lppd = lppd;
      out.waic_p_eff = p_waic;
      out.waic = -2.0 * (lppd - p_waic);
    }
  }

  if (what & MS_CPO) {  // compute_cpo_pit (model_selection.rs:222-325)
    out.cpo.assign(n, NaN);
    out.pit.assign(n, NaN);
    std::vector<char> failed(n, 0);
    parallel_for(n, [&](int64_t i0, int64_t i1) {
      for (int64_t i = i0; i < i1; ++i) {
        const double q1 = (obs.p1 ? obs.p1[i] : 1.0) * obs.p1scale, q2 = obs.p2 ? obs.p2[i] : 1.0;
        if (!ms_cpo_pit_obs(obs.family, obs.y[i], q1, q2, K, w, cond_eta + i, cond_eta_var + i, n, out.cpo[i],
                            out.pit[i]))
          failed[i] = 1;
      }
    }, 2048);
    for (int64_t i = 0; i < n; ++i) out.cpo_failures += failed[i];
  }
  return std::string();
}

}  // namespace inla
