// Observation likelihoods (value, gradient, Fisher/observed Hessian) shared by the device
// kernels and the host code of the model-selection criteria.
//
// Reference: crates/inla_stats/src/inference.rs:170-311 (eval_likelihood), 1641-1664
// (logistic), 1896-1920 (log_gamma).
#pragma once
#include <cmath>
#include <cuda_runtime.h>

namespace inla {
namespace {

enum Family : int { FAM_GAUSSIAN = 0, FAM_POISSON = 1, FAM_BINOMIAL = 2, FAM_NBINOMIAL = 3 };

// Lanczos log-gamma, g = 7, 9 coefficients (inference.rs:1896-1920 uses the
// same published series).
__host__ __device__ __forceinline__ double d_log_gamma_pos(double z) {
  const double PI = 3.14159265358979323846;
  const double z1 = z - 1.0;
  double x = 0.99999999999980993;
  x += 676.5203681218851 / (z1 + 1.0);
  x += -1259.1392167224028 / (z1 + 2.0);
  x += 771.32342877765313 / (z1 + 3.0);
  x += -176.61502916214059 / (z1 + 4.0);
  x += 12.507343278686905 / (z1 + 5.0);
  x += -0.13857109526572012 / (z1 + 6.0);
  x += 9.9843695780195716e-6 / (z1 + 7.0);
  x += 1.5056327351493116e-7 / (z1 + 8.0);
  const double t = z1 + 7.5;
  return 0.5 * log(2.0 * PI) + (z1 + 0.5) * log(t) - t + log(x);
}
__host__ __device__ __forceinline__ double d_log_gamma(double z) {
  const double PI = 3.14159265358979323846;
  if (z < 0.5) return log(PI) - log(sin(PI * z)) - d_log_gamma_pos(1.0 - z);
  return d_log_gamma_pos(z);
}

__host__ __device__ __forceinline__ double d_logistic(double x) {
  if (x >= 0.0) {
    double z = exp(-x);
    return 1.0 / (1.0 + z);
  }
  double z = exp(x);
  return z / (1.0 + z);
}

// Eval1D: returns 0 on success, 1 on an invalid input (reference: Err).
// p1: gaussian precision / poisson exposure / binomial trials / nb size.
// p2: nb exposure. dw: d(-hess)/d eta (for the adjoint's implicit term).
__host__ __device__ __forceinline__ int d_eval_lik(int fam, double eta, double y, double p1, double p2, double& logp,
                                          double& grad, double& hess, double& dw) {
  if (!isfinite(eta)) return 1;
  switch (fam) {
    case FAM_GAUSSIAN: {
      if (!(p1 > 0.0) || !isfinite(p1) || !isfinite(y)) return 1;
      const double r = eta - y;
      logp = -0.9189385332046728 + 0.5 * log(p1) - 0.5 * p1 * r * r;
      grad = -p1 * r;
      hess = -p1;
      dw = 0.0;
      return 0;
    }
    case FAM_POISSON: {
      if (p1 < 0.0 || !isfinite(p1) || y < 0.0 || !isfinite(y)) return 1;
      const double lam = exp(eta);
      const double mu = p1 * lam, dmu = p1 * lam;
      if (mu > 0.0) {
        logp = y * log(mu) - mu - d_log_gamma(y + 1.0);
        grad = (y / mu - 1.0) * dmu;
        hess = -(dmu * dmu) / mu;  // Fisher scoring
        dw = mu;
      } else {
        logp = (y == 0.0) ? 0.0 : -INFINITY;
        grad = -dmu;
        hess = -fabs(p1 * lam);
        dw = 0.0;
      }
      return 0;
    }
    case FAM_BINOMIAL: {
      if (p1 < 0.0 || y < 0.0 || y > p1 || !isfinite(p1) || !isfinite(y)) return 1;
      const double p = d_logistic(eta), dp = p * (1.0 - p);
      const double lc = d_log_gamma(p1 + 1.0) - d_log_gamma(y + 1.0) - d_log_gamma(p1 - y + 1.0);
      if (p == 0.0) logp = (y == 0.0) ? lc : -INFINITY;
      else if (p == 1.0) logp = (y == p1) ? lc : -INFINITY;
      else logp = lc + y * log(p) + (p1 - y) * log(1.0 - p);
      const double a = (p > 0.0 && p < 1.0) ? y / p - (p1 - y) / (1.0 - p) : 0.0;
      grad = a * dp;
      hess = -p1 * dp;  // Fisher scoring
      dw = p1 * dp * (1.0 - 2.0 * p);
      return 0;
    }
    case FAM_NBINOMIAL: {
      const double r = p1, E = p2;
      if (y < 0.0 || !isfinite(y) || E < 0.0 || !isfinite(E) || !(r > 0.0) || !isfinite(r)) return 1;
      const double base = exp(eta);
      if (!(base > 0.0)) return 1;
      const double mu = E * base;
      if (!(mu > 0.0)) return 1;
      const double mr = mu + r;
      logp = d_log_gamma(y + r) - d_log_gamma(r) - d_log_gamma(y + 1.0) + r * log(r / mr) + y * log(mu / mr);
      const double d1 = y / mu - (y + r) / mr;
      const double d2 = -y / (mu * mu) + (y + r) / (mr * mr);
      const double d3 = 2.0 * y / (mu * mu * mu) - 2.0 * (y + r) / (mr * mr * mr);
      grad = d1 * mu;
      hess = d2 * mu * mu + d1 * mu;  // observed Hessian
      dw = -(d3 * mu * mu * mu + 3.0 * d2 * mu * mu + d1 * mu);
      return 0;
    }
  }
  return 1;
}

}  // namespace
}  // namespace inla
