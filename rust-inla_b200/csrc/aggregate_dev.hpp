// Post-node aggregation of an INLA fit on the device: per-node linear predictor and its
// diagonal variance, mixture moments over the integration nodes, and the model-selection
// criteria (DIC, WAIC, CPO / PIT) over observations x nodes.
//
// Reference: crates/inla_stats/src/inference.rs:1370-1384, 1436-1466 (per-node predictor,
// mixture moments), 1470-1514 (criteria at the end of a fit); crates/inla_math/src/design.rs:
// 52-70 (matvec_csc), 198-210 (predictor_variances_diag); crates/inla_stats/src/
// model_selection.rs:101-150 (DIC), 152-211 (WAIC), 222-325 (CPO / PIT).
//
// The predictor and the mixture are bit-identical to the host code in aggregate.cpp (same
// operations in the same order, no contracted multiply-adds). The criteria's sums over
// observations use a fixed reduction tree, so they agree with the host's sequential sums to
// rounding and are identical run to run.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "gpu_factor.hpp"
#include "model_select.hpp"

namespace inla {

// Device CSR of A (nobs x n); rp == nullptr means eta = x (nobs == n).
struct DevCsrA {
  const int64_t* rp = nullptr;
  const int* ci = nullptr;
  const double* v = nullptr;
};

// Observations on the device, as ObsView.
struct DevObs {
  int family = 0;
  int64_t nobs = 0;
  const double* y = nullptr;
  const double* p1 = nullptr;  // nullptr = 1
  const double* p2 = nullptr;  // nullptr = 1
  double p1scale = 1.0;
};

// Scratch of the device criteria (grown on demand, kept between calls).
struct AggScratch {
  DBuf<double> w, ll, lppd, pw, red, cpo, pit;
  DBuf<int> bad, nodebad, ired;
  DBuf<unsigned char> ok;
};

// eta[k][i] = sum_p A_ip x_k[col] (entries with x == 0 skipped), eta_var[k][i] =
// sum_p A_ip^2 v_k[col], for K nodes whose means / variances sit at cmean + k * ldm and
// cvar + k * ldv; outputs [K][nobs].
void dev_project_nodes(cudaStream_t st, int64_t nobs, const DevCsrA& A, int K, const double* cmean, int64_t ldm,
                       const double* cvar, int64_t ldv, double* eta, double* eta_var);

// mean = sum_k w_k m_k, var = sum_k w_k (v_k + (m_k - mean)^2) entry by entry; w on the device.
void dev_mixture_moments(cudaStream_t st, int K, int64_t len, const double* d_w, const double* cmean, int64_t ldm,
                         const double* cvar, int64_t ldv, double* mean, double* var);

// The criteria of `what` (MS_* bits) from the per-node predictors d_eta, d_eta_var [K][nobs]
// and the host weights w [K]; returns the reference's error message, or an empty string.
// Synchronizes the stream.
std::string dev_model_selection(cudaStream_t st, const DevObs& obs, int K, const double* w, int mode_index,
                                const double* d_eta, const double* d_eta_var, int what, AggScratch& scratch,
                                ModelSelection& out);

}  // namespace inla
