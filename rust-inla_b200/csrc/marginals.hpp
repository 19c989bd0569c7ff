// One-dimensional posterior marginals of a fit: Gaussian-mixture densities of latent and
// predictor entries over the integration nodes, kernel densities of the hyperparameters, and
// quantiles by the cumulative trapezoid. Host code.
//
// Reference: crates/inla_stats/src/marginals.rs:20-41 (trapezoid mass and normalisation),
// 73-135 (gaussian_mixture_marginal), 137-162 (hyperpar_marginal_from_nodes), 183-226
// (marginal_cdf, marginal_quantiles).
#pragma once
#include <string>
#include <vector>

namespace inla {

// Uniform grid of n_points over mean +- max(n_sd, 1) sd of the mixture, density
// sum_k w_k N(x; m_k, v_k), normalised to unit trapezoid mass. Empty string on success.
std::string mixture_marginal(int K, const double* means, const double* vars, const double* w, int n_points,
                             double n_sd, double* x, double* y);
// Kernel mixture at the node values theta_k with the weighted sample variance (at least 1e-8)
// as every kernel's variance.
std::string hyperpar_marginal(int K, const double* theta, const double* w, int n_points, double n_sd, double* x,
                              double* y);
// Quantiles of a gridded density: the CDF by cumulative trapezoid normalised to 1, inverted
// linearly at each probability in (0, 1).
std::string marginal_quantiles(int n, const double* x, const double* y, int np, const double* probs, double* q);

}  // namespace inla
