// Theta-level INLA driver over the batched Laplace engine.
//
// Reference path (crates/inla_stats/src/inference.rs:1116-1466 and
// crates/inla_math/src/{hyper_opt,integration}.rs): Nelder-Mead mode search
// on -(mlik + log pi(theta)) (1e12 on a failed Laplace), finite-difference
// Hessian with h = max(1e-4, 0.05|theta|), eigen-rotated CCD (or grid)
// design, per-node Laplace + selected-inverse variances, weight
// normalisation and Gaussian-mixture moments.
//
// Batched path: the same design and aggregation, with the mode found by
// BFGS on exact adjoint gradients (a batched multi-step line search per
// iteration), and every theta-set (line-search candidates, Hessian stencil,
// CCD nodes) evaluated as one batched launch sequence.
#pragma once
#include <functional>
#include <vector>

#include "laplace.hpp"

namespace inla {

// theta -> component coefficients (+ d/dtheta) and the likelihood p1 scale.
// dcoef: [m][ncomp]; dp1scale: [m]. Returns 0 on success.
using ThetaMap = std::function<int(const double* theta, double* coef, double* dcoef, double* p1scale,
                                   double* dp1scale)>;
// log pi(theta) and its gradient (grad may be null).
using LogPrior = std::function<double(const double* theta, double* grad)>;

struct FitOptions {
  int mode_search = 0;  // 0 Nelder-Mead (reference), 1 BFGS on adjoint gradients, 2 batched Newton
                        // (central FD-of-gradient Hessian), 3 batched Newton (forward FD-of-gradient)
  int batched = 0;      // 0: one theta-point per evaluation; 1: batched theta-sets
  int strategy = 0;     // 0 CCD, 1 grid
  double f0 = 1.0;      // CCD f0 (reference default 1.0) / grid step
  int hessian = 0;      // 0 FD of values (reference stencil), 1 central FD of adjoint gradients
  int max_iter = 200;   // NM iterations (hyper_opt.rs:34) / BFGS iterations
  double tol = 1e-6;    // NM f-spread tolerance / BFGS gradient infinity-norm tolerance
  double nm_step = 0.1;
  // Polled before every evaluation; returning true stops the fit with INLA_ERR_CANCELLED
  // (check_cancel of inference.rs:1116-1130, hyper_opt.rs:21-47).
  std::function<bool()> cancel;
};

struct FitResult {
  // device copies of the per-node predictor and its variance [K][nobs] (filled when set; the
  // model-selection criteria of the fit read them on the device)
  DBuf<double>* d_cond_eta = nullptr;
  DBuf<double>* d_cond_eta_var = nullptr;
  std::vector<double> mode, hessian, latent_mean, latent_var, node_theta, node_weight, node_logpost;
  std::vector<double> pred_mean, pred_var;  // linear predictor eta = A x: mixture mean and variance
  std::vector<double> cond_eta, cond_eta_var;  // [K][nobs] per-node predictor and its variance
  std::vector<double> cond_mean, cond_var;     // [K][n] per-node mode and marginal variances
  int mode_index = 0;                          // node with the smallest |z| (inference.rs:1296-1304)
  double p1scale_mode = 1.0;                   // likelihood p1 scale at the mode (observations at the mode)
  std::vector<double> coef_mode;               // component coefficients of Q at the mode
  double mlik_gaussian = 0.0;                  // Gaussian approximation of the log marginal likelihood
  double mlik = 0.0;
  int n_evals = 0, n_batches = 0, mode_iters = 0;
  double seconds = 0.0;
  // wall seconds of the fit's phases: mode search, Hessian, integration design + node
  // evaluations, aggregation (mixture, predictor, model-selection inputs); they add up to
  // `seconds` up to the host bookkeeping between them
  double phase_s[4] = {0.0, 0.0, 0.0, 0.0};
};

class InlaDriver {
 public:
  InlaDriver(LaplaceEngine& eng, int m, ThetaMap map, LogPrior prior) : eng_(eng), m_(m), map_(map), prior_(prior) {}
  void fit(const double* theta0, const FitOptions& opt, FitResult& out);

  // Evaluate f = -(mlik + log prior) (and its gradient when grad != null) at K points.
  void evaluate(int K, const double* thetas, bool want_grad, bool batched, double* f, double* grad,
                std::vector<LaplaceOut>* keep = nullptr);

  int n_evals() const { return n_evals_; }
  int n_batches() const { return n_batches_; }

 private:
  void nelder_mead(std::vector<double>& theta, const FitOptions& opt, int& iters);
  void bfgs(std::vector<double>& theta, const FitOptions& opt, int& iters);
  void newton(std::vector<double>& theta, const FitOptions& opt, int& iters);
  void eval_stencils(const std::vector<std::vector<double>>& centers, double h, std::vector<double>& f,
                     std::vector<double>& g, std::vector<double>& H, bool one_sided = false);
  void fd_hessian(const std::vector<double>& mode, double h, bool batched, std::vector<double>& H);
  void grad_hessian(const std::vector<double>& mode, double h, bool batched, std::vector<double>& H);
  void fit_single_node(FitResult& out);  // m = 0
  void check_cancel() const;

  LaplaceEngine& eng_;
  int m_;
  ThetaMap map_;
  LogPrior prior_;
  int n_evals_ = 0, n_batches_ = 0;
  std::function<bool()> cancel_;
};

// integration.rs restatements
void ccd_design(int m, double f0, std::vector<double>& points, std::vector<double>& weights);
bool invert_symmetric_matrix(const std::vector<double>& h, int m, std::vector<double>& inv);
void symmetric_eigen(const std::vector<double>& a, int m, std::vector<double>& lambda, std::vector<double>& V);

}  // namespace inla
