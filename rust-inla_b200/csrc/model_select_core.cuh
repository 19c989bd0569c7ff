// Per-observation pieces of the model-selection criteria, shared by the host code and the
// device kernels: observation CDFs, the CPO failure heuristic and the per-(node,
// observation) likelihood. Plain functions of their arguments (no allocation).
//
// Reference: crates/inla_stats/src/model_selection.rs:327-396 (check_cpo_failure_for_obs),
// 398-515 (observation_cdf, normal / Poisson / binomial CDFs).
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "likelihood.cuh"

namespace inla {
namespace {

constexpr double kCpoDiff = 3.0;  // CPO_DIFF (model_selection.rs:7)

__host__ __device__ inline double ms_normal_cdf(double x) {
  // Abramowitz & Stegun 7.1.26 rational approximation of erf, as the reference uses
  const double A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741, A4 = -1.453152027, A5 = 1.061405429,
               P = 0.3275911;
  const double sign = x < 0.0 ? -1.0 : 1.0;
  const double ax = fabs(x);
  const double t = 1.0 / (1.0 + P * ax);
  const double y = 1.0 - (((((A5 * t + A4) * t) + A3) * t + A2) * t + A1) * t * exp(-ax * ax / 2.0);
  return 0.5 * (1.0 + sign * y);
}

__host__ __device__ inline double ms_poisson_cdf(double lambda, uint64_t k) {
  if (lambda <= 0.0) return 1.0;
  double cdf = 0.0, log_pmf = -lambda;
  for (uint64_t j = 0; j <= k; ++j) {
    cdf += exp(log_pmf);
    if (j < k) log_pmf += log(lambda) - log((double)(j + 1));
  }
  return fmin(cdf, 1.0);
}

__host__ __device__ inline double ms_binomial_cdf(uint64_t n, double p, uint64_t k) {
  if (p <= 0.0) return 1.0;
  if (p >= 1.0) return k >= n ? 1.0 : 0.0;
  double cdf = 0.0;
  for (uint64_t j = 0; j <= k; ++j) {
    const double log_choose =
        d_log_gamma((double)n + 1.0) - d_log_gamma((double)j + 1.0) - d_log_gamma((double)(n - j) + 1.0);
    const double log_pmf = log_choose + (double)j * log(p) + (double)(n - j) * log(1.0 - p);
    cdf += exp(log_pmf);
  }
  return fmin(cdf, 1.0);
}

// observation_cdf (model_selection.rs:398-448) with p1 the family's first parameter; false
// where the reference gives None (negative binomial, invalid rate or variance)
__host__ __device__ inline bool ms_observation_cdf(int family, double y, double p1, double eta, double variance,
                                                   double& out) {
  // the count CDFs sum term by term up to floor(y); counts beyond 1e15 (and non-finite y)
  // get no CDF instead of a loop of that length
  if (!isfinite(y) || (family != FAM_GAUSSIAN && y > 1e15)) return false;
  switch (family) {
    case FAM_GAUSSIAN: {
      const double total_var = 1.0 / p1 + variance;
      if (total_var <= 0.0) return false;
      out = ms_normal_cdf((y - eta) / sqrt(total_var));
      return true;
    }
    case FAM_POISSON: {
      const double lambda = p1 * exp(eta);
      if (lambda < 0.0 || !isfinite(lambda)) return false;
      const double yf = floor(y);
      if (yf < 0.0) {
        out = 0.0;
        return true;
      }
      out = ms_poisson_cdf(lambda, (uint64_t)yf);
      return true;
    }
    case FAM_BINOMIAL: {
      const double prob = d_logistic(eta);
      const uint64_t n = (isfinite(p1) && p1 > 0.0) ? (uint64_t)p1 : 0;  // f64 as u64 saturates at 0
      const double yf = floor(y);
      if (yf < 0.0) {
        out = 0.0;
        return true;
      }
      out = ms_binomial_cdf(n, prob, yf >= (double)n ? n : (uint64_t)yf);
      return true;
    }
    default:
      return false;  // negative binomial: no CDF in the reference
  }
}

// check_cpo_failure_for_obs (model_selection.rs:327-396)
__host__ __device__ inline bool ms_cpo_failure(int family, double y, double p1, double p2, double mu, double var) {
  if (var <= 0.0 || !isfinite(var)) return true;
  double lp, g, h, dw;
  if (d_eval_lik(family, mu, y, p1, p2, lp, g, h, dw)) return true;
  const double c = -h;
  const double tau_loo = 1.0 / var - c;
  if (tau_loo <= 0.0 || !isfinite(tau_loo)) return true;
  const double var_loo = 1.0 / tau_loo, std_loo = sqrt(var_loo);
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
  double mx = -INFINITY;
  for (int s = 0; s < 5; ++s) mx = fmax(mx, ld[s]);
  return mx - ld[0] < kCpoDiff || mx - ld[4] < kCpoDiff;
}

// CPO and PIT of one observation over K nodes (compute_cpo_pit, model_selection.rs:222-325):
// returns false when the observation counts as a CPO failure; cpo / pit are NaN where the
// reference gives None. eta, var: the observation's node values with stride `stride`.
__host__ __device__ inline bool ms_cpo_pit_obs(int family, double y, double q1, double q2, int K, const double* w,
                                               const double* eta, const double* var, int64_t stride, double& cpo,
                                               double& pit) {
  cpo = NAN;
  pit = NAN;
  for (int k = 0; k < K; ++k)
    if (ms_cpo_failure(family, y, q1, q2, eta[(int64_t)k * stride], var[(int64_t)k * stride])) return false;
  if (K < 2) return false;
  double max_neg = -INFINITY;
  double lp, g, h, dw;
  for (int k = 0; k < K; ++k) {
    if (d_eval_lik(family, eta[(int64_t)k * stride], y, q1, q2, lp, g, h, dw)) return false;
    max_neg = fmax(max_neg, -lp);
  }
  double inv = 0.0;
  for (int k = 0; k < K; ++k) {
    d_eval_lik(family, eta[(int64_t)k * stride], y, q1, q2, lp, g, h, dw);
    inv += w[k] * exp(-lp - max_neg);
  }
  const double inv_scaled = inv * exp(max_neg);
  if (!isfinite(inv_scaled) || inv_scaled <= 0.0) return false;
  cpo = 1.0 / inv_scaled;
  double acc = 0.0;
  for (int k = 0; k < K; ++k) {
    double f;
    if (!ms_observation_cdf(family, y, q1, eta[(int64_t)k * stride], var[(int64_t)k * stride], f)) return true;
    acc += w[k] * f;
  }
  if (isfinite(acc)) pit = fmin(fmax(acc, 0.0), 1.0);
  return true;
}

}  // namespace
}  // namespace inla
