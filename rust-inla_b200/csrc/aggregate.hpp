// Moments of the posterior mixture over integration nodes.
//
// Reference: crates/inla_stats/src/inference.rs:1370-1384 (per-node predictor and its
// variance), 1436-1466 (mixture mean and variance of the latent field and of the predictor);
// crates/inla_math/src/design.rs:52-70 (matvec_csc) and 198-210 (predictor_variances_diag).
#pragma once
#include <cstdint>

namespace inla {

// Mixture over K nodes with normalised weights w: mean = sum_k w_k m_k and
// var = sum_k w_k (v_k + (m_k - mean)^2), element by element, k ascending.
// cmean, cvar: [K][len].
void mixture_moments(int K, int64_t len, const double* w, const double* cmean, const double* cvar, double* mean,
                     double* var);

// Per node eta_k = A x_k (columns with x_kj == 0 skipped, as matvec_csc does) and
// eta-var_k = sum_j A_ij^2 var_kj, each summed in the row's stored order. A: nobs x n in CSR
// (acp == nullptr: eta = x, nobs == n). cmean, cvar: [K][n]; eta, eta_var: [K][nobs].
void project_nodes(int64_t nobs, int64_t n, const int64_t* acp, const int64_t* aci, const double* av, int K,
                   const double* cmean, const double* cvar, double* eta, double* eta_var);

// Linear-predictor moments: per node eta_k = A x_k (columns with x_kj == 0 skipped, as
// matvec_csc does) and eta-var_k = sum_j A_ij^2 var_kj, each summed in the row's stored order
// (ascending columns give the reference's order), then mixed as mixture_moments does.
// A: nobs x n in CSR; acp == nullptr means eta = x (nobs == n). cmean, cvar: [K][n].
void predictor_moments(int64_t nobs, int64_t n, const int64_t* acp, const int64_t* aci, const double* av, int K,
                       const double* w, const double* cmean, const double* cvar, double* mean, double* var);

}  // namespace inla
