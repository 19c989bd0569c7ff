#include "marginals.hpp"

#include <algorithm>
#include <cmath>

namespace inla {

namespace {

double phi(double x, double mu, double var) {
  if (!(var > 0.0 && std::isfinite(var))) return 0.0;
  const double s = std::sqrt(var);
  const double z = (x - mu) / s;
  return std::exp(-0.5 * z * z) / (s * std::sqrt(2.0 * 3.14159265358979323846));
}

double trapezoid_mass(int n, const double* x, const double* y) {
  if (n < 2) return 0.0;
  double s = 0.0;
  for (int i = 0; i + 1 < n; ++i) s += 0.5 * (y[i] + y[i + 1]) * (x[i + 1] - x[i]);
  return s;
}

}  // namespace

std::string mixture_marginal(int K, const double* means, const double* vars, const double* w, int n_points,
                             double n_sd, double* x, double* y) {
  if (K < 1) return "empty mixture";
  if (n_points < 5) return "n_points must be >= 5";
  double mu = 0.0;
  for (int k = 0; k < K; ++k) mu += w[k] * means[k];
  double var = 0.0;
  for (int k = 0; k < K; ++k) {
    const double d = means[k] - mu;
    var += w[k] * (vars[k] + d * d);
  }
  if (!(var > 0.0 && std::isfinite(var))) var = 1e-8;
  const double half = std::fmax(n_sd, 1.0) * std::sqrt(var);
  const double lo = mu - half, hi = mu + half;
  for (int i = 0; i < n_points; ++i) {
    const double xi = lo + (hi - lo) * (double)i / (double)(n_points - 1);
    double yi = 0.0;
    for (int k = 0; k < K; ++k) yi += w[k] * phi(xi, means[k], vars[k]);
    x[i] = xi;
    y[i] = yi;
  }
  const double mass = trapezoid_mass(n_points, x, y);
  if (mass > 0.0 && std::isfinite(mass))
    for (int i = 0; i < n_points; ++i) y[i] /= mass;
  return std::string();
}

std::string hyperpar_marginal(int K, const double* theta, const double* w, int n_points, double n_sd, double* x,
                              double* y) {
  if (K < 1) return "theta_j/weights mismatch or empty";
  double mu = 0.0;
  for (int k = 0; k < K; ++k) mu += w[k] * theta[k];
  double v = 0.0;
  for (int k = 0; k < K; ++k) {
    const double d = theta[k] - mu;
    v += w[k] * d * d;
  }
  const std::vector<double> vars(K, std::fmax(v, 1e-8) * 1.0);
  return mixture_marginal(K, theta, vars.data(), w, n_points, n_sd, x, y);
}

std::string marginal_quantiles(int n, const double* x, const double* y, int np, const double* probs, double* q) {
  if (n < 2) return "marginal too short or x/y length mismatch";
  std::vector<double> f(n, 0.0);
  for (int i = 0; i + 1 < n; ++i) f[i + 1] = f[i] + 0.5 * (y[i] + y[i + 1]) * (x[i + 1] - x[i]);
  const double mass = f[n - 1];
  if (mass > 0.0)
    for (double& v : f) v /= mass;
  for (int j = 0; j < np; ++j) {
    const double p = probs[j];
    if (!(p > 0.0 && p < 1.0)) return "probability must be in (0, 1)";
    double qj = x[n - 1];
    for (int i = 1; i < n; ++i)
      if (f[i] >= p) {
        const double t = std::fabs(f[i] - f[i - 1]) < 1e-15 ? 0.0 : (p - f[i - 1]) / (f[i] - f[i - 1]);
        qj = x[i - 1] + t * (x[i] - x[i - 1]);
        break;
      }
    q[j] = qj;
  }
  return std::string();
}

}  // namespace inla
