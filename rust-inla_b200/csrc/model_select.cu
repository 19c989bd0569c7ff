// Host code (no kernels): the model-selection criteria of an INLA fit. Compiled as CUDA
// source only to share the likelihood code of the device kernels (likelihood.cuh).
#include <algorithm>
#include <cmath>
#include <limits>

#include "host_par.hpp"
#include "likelihood.cuh"
#include "model_select.hpp"

namespace inla {

namespace {

constexpr double kCpoDiff = 3.0;  // CPO_DIFF (model_selection.rs:7)

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
  // the count CDFs below sum term by term up to floor(y); counts beyond 1e15 (and non-finite y)
  // get no CDF instead of a loop of that length
  if (!std::isfinite(y) || (family != FAM_GAUSSIAN && y > 1e15)) return false;
  switch (family) {
    case FAM_GAUSSIAN: {
      const double total_var = 1.0 / p1 + variance;
      if (total_var <= 0.0) return false;
      out = normal_cdf((y - eta) / std::sqrt(total_var));
      return true;
    }
    case FAM_POISSON: {
      const double lambda = p1 * std::exp(eta);
      if (lambda < 0.0 || !std::isfinite(lambda)) return false;
      const double yf = std::floor(y);
      if (yf < 0.0) {
        out = 0.0;
        return true;
      }
      out = poisson_cdf(lambda, (uint64_t)yf);
      return true;
    }
    case FAM_BINOMIAL: {
      const double prob = d_logistic(eta);
      const uint64_t n = (std::isfinite(p1) && p1 > 0.0) ? (uint64_t)p1 : 0;  // f64 as u64 saturates at 0
      const double yf = std::floor(y);
      if (yf < 0.0) {
        out = 0.0;
        return true;
      }
      out = binomial_cdf(n, prob, yf >= (double)n ? n : (uint64_t)yf);
      return true;
    }
    default:
      return false;  // negative binomial: no CDF in the reference
  }
}

double normal_cdf(double x) {
  // Abramowitz & Stegun 7.1.26 rational approximation of erf, as the reference uses
  const double A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741, A4 = -1.453152027, A5 = 1.061405429,
               P = 0.3275911;
  const double sign = x < 0.0 ? -1.0 : 1.0;
  const double ax = std::fabs(x);
  const double t = 1.0 / (1.0 + P * ax);
  const double y = 1.0 - (((((A5 * t + A4) * t) + A3) * t + A2) * t + A1) * t * std::exp(-ax * ax / 2.0);
  return 0.5 * (1.0 + sign * y);
}

double poisson_cdf(double lambda, uint64_t k) {
  if (lambda <= 0.0) return 1.0;
  double cdf = 0.0, log_pmf = -lambda;
  for (uint64_t j = 0; j <= k; ++j) {
    cdf += std::exp(log_pmf);
    if (j < k) log_pmf += std::log(lambda) - std::log((double)(j + 1));
  }
  return std::min(cdf, 1.0);
}

double binomial_cdf(uint64_t n, double p, uint64_t k) {
  if (p <= 0.0) return 1.0;
  if (p >= 1.0) return k >= n ? 1.0 : 0.0;
  double cdf = 0.0;
  for (uint64_t j = 0; j <= k; ++j) {
    const double log_choose =
        d_log_gamma((double)n + 1.0) - d_log_gamma((double)j + 1.0) - d_log_gamma((double)(n - j) + 1.0);
    const double log_pmf = log_choose + (double)j * std::log(p) + (double)(n - j) * std::log(1.0 - p);
    cdf += std::exp(log_pmf);
  }
  return std::min(cdf, 1.0);
}

bool cpo_failure(int family, double y, double p1, double p2, double mu, double var) {
  if (var <= 0.0 || !std::isfinite(var)) return true;
  double lp, g, h, dw;
  if (d_eval_lik(family, mu, y, p1, p2, lp, g, h, dw)) return true;
  const double c = -h;
  const double tau_loo = 1.0 / var - c;
  if (tau_loo <= 0.0 || !std::isfinite(tau_loo)) return true;
  const double var_loo = 1.0 / tau_loo, std_loo = std::sqrt(var_loo);
  const double mu_loo = var_loo * (mu / var - c * mu + g);
  const double steps[5] = {-3.0, -1.5, 0.0, 1.5, 3.0};
  double ld[5];
  for (int s = 0; s < 5; ++s) {
    const double x = mu_loo + steps[s] * std_loo;
    const double prior = -0.5 * (x - mu) * (x - mu) / var;
    if (d_eval_lik(family, x, y, p1, p2, lp, g, h, dw)) return true;
    ld[s] = prior + lp;
  }
  bool inc = true, dec = true;
  for (int s = 1; s < 5; ++s) {
    if (ld[s] < ld[s - 1]) inc = false;
    if (ld[s] > ld[s - 1]) dec = false;
  }
  if (inc || dec) return true;
  double mx = -std::numeric_limits<double>::infinity();
  for (int s = 0; s < 5; ++s) mx = std::fmax(mx, ld[s]);
  return mx - ld[0] < kCpoDiff || mx - ld[4] < kCpoDiff;
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
      std::vector<double> lls(K);
      for (int64_t i = i0; i < i1; ++i) {
        const double y = obs.y[i];
        const double q1 = (obs.p1 ? obs.p1[i] : 1.0) * obs.p1scale, q2 = obs.p2 ? obs.p2[i] : 1.0;
        bool fail = false;
        for (int k = 0; k < K && !fail; ++k)
          fail = cpo_failure(obs.family, y, q1, q2, cond_eta[(size_t)k * n + i], cond_eta_var[(size_t)k * n + i]);
        Lik e;
        for (int k = 0; k < K && !fail; ++k) {
          if (!lik_at(obs, i, cond_eta[(size_t)k * n + i], e)) fail = true;
          else lls[k] = e.logp;
        }
        if (fail || K < 2) {
          failed[i] = 1;
          continue;
        }
        double max_neg = -std::numeric_limits<double>::infinity();
        for (int k = 0; k < K; ++k) max_neg = std::fmax(max_neg, -lls[k]);
        double inv = 0.0;
        for (int k = 0; k < K; ++k) inv += w[k] * std::exp(-lls[k] - max_neg);
        const double inv_scaled = inv * std::exp(max_neg);
        if (!std::isfinite(inv_scaled) || inv_scaled <= 0.0) {
          failed[i] = 1;
          continue;
        }
        out.cpo[i] = 1.0 / inv_scaled;
        double pit = 0.0;
        bool pit_ok = true;
        for (int k = 0; k < K && pit_ok; ++k) {
          double f;
          if (observation_cdf(obs.family, y, q1, cond_eta[(size_t)k * n + i], cond_eta_var[(size_t)k * n + i], f))
            pit += w[k] * f;
          else
            pit_ok = false;
        }
        if (pit_ok && std::isfinite(pit)) out.pit[i] = std::min(std::max(pit, 0.0), 1.0);
      }
    }, 2048);
    for (int64_t i = 0; i < n; ++i) out.cpo_failures += failed[i];
  }
  return std::string();
}

}  // namespace inla
