// Model-selection criteria of an INLA fit: DIC, WAIC, CPO / PIT and the Gaussian
// approximation of the log marginal likelihood, computed on the host from the per-node
// linear predictors, their variances and the normalised node weights.
//
// Reference: crates/inla_stats/src/model_selection.rs:25-73 (Gaussian-approximation mlik),
// 82-150 (DIC), 152-211 (WAIC), 222-396 (CPO / PIT and the failure heuristic), 398-515
// (observation CDFs); call site crates/inla_stats/src/inference.rs:1470-1514 (observations
// built at the mode, mode index = the node with the smallest |z|).
#pragma once
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

namespace inla {

enum ModelSelectionWhat : int { MS_DIC = 1, MS_WAIC = 2, MS_CPO = 4 };

struct ModelSelection {
  double dic = NAN, mean_deviance = NAN, dic_p_eff = NAN;
  double waic = NAN, lppd = NAN, waic_p_eff = NAN;
  int64_t cpo_failures = 0;
  std::vector<double> cpo, pit;  // NaN where the reference gives None
};

// Observations of one family: y, p1 (gaussian precision / poisson exposure / binomial trials /
// nb size; nullptr = 1) times p1scale, p2 (nb exposure; nullptr = 1).
struct ObsView {
  int family = 0;
  int64_t nobs = 0;
  const double* y = nullptr;
  const double* p1 = nullptr;
  const double* p2 = nullptr;
  double p1scale = 1.0;
};

// cond_eta, cond_eta_var: [K][nobs]; w: [K]. Returns an empty string on success, else the
// reference's error (a likelihood that cannot be evaluated, a non-finite WAIC density); the
// criteria not asked for in `what` stay NaN.
std::string model_selection(const ObsView& obs, int K, const double* w, int mode_index, const double* cond_eta,
                            const double* cond_eta_var, int what, ModelSelection& out);

// log pi(theta*|y) + m/2 log(2 pi) - 1/2 log det(-H) by an in-place Cholesky of -H (row-major
// m x m); false when -H is not positive definite.
bool mlik_gaussian(double log_post_mode, int m, const double* neg_hessian, double& out);

// Helpers exposed for the tests of the reference's known answers.
double normal_cdf(double x);
double poisson_cdf(double lambda, uint64_t k);
double binomial_cdf(uint64_t n, double p, uint64_t k);
bool cpo_failure(int family, double y, double p1, double p2, double mu, double var);
// observation_cdf (model_selection.rs:398-448) with p1 the family's first parameter; false
// where the reference gives None (negative binomial, invalid rate or variance)
bool observation_cdf(int family, double y, double p1, double eta, double variance, double& out);

}  // namespace inla
