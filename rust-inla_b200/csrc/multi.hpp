// Batched Laplace evaluation of G independent latent models of uneven size in one
// launch sequence per step: the models are held as one block-diagonal latent
// field with one symbolic analysis (the elimination forest has one tree per model,
// so every level launch works on all models' fronts at once, without padding),
// and B theta-sets are evaluated together, each carrying per-model coefficients.
//
// Reference control flow per model: find_latent_mode_a_with_solver
// (crates/inla_stats/src/inference.rs:776-975), as in laplace.hpp; every
// decision of the Newton loop (step cap, halving, convergence, confirmation
// refactorization) is taken per (theta-set, model), and a model that has
// converged keeps its mode while the others iterate.
#pragma once
#include <functional>
#include <memory>
#include <vector>

#include "gpu_factor.hpp"
#include "laplace.hpp"

namespace inla {

struct MultiSpec {
  int G = 0;                             // models
  int64_t n = 0, nobs = 0;               // union sizes
  std::vector<int64_t> lat_off, obs_off; // G+1: model g owns latent [lat_off[g], lat_off[g+1]) and observations
  std::vector<int64_t> colptr, rowidx;   // block-diagonal full symmetric pattern (contains A^T A, diagonal)
  int ncomp = 0;
  std::vector<double> comp;              // [ncomp][nnz]
  std::vector<int64_t> acp, aci;         // A in CSR (nobs x n), block-diagonal
  std::vector<double> av;
  int family = 0;
  std::vector<double> y, p1, p2;
  int max_iter = 200;
  double tol = 1e-5;
  int ordering = ORDER_ND;               // applied to every model's block
};

struct MultiOut {
  // per (theta-set b, model g), index b * G + g
  std::vector<double> mlik, ld_prior, ld_post, loglik, quad, dll;
  std::vector<int> status, iters;
  // [b][g][ncomp+1]: as LaplaceOut
  std::vector<double> trP, trQ, xMx, zMx;
};

class MultiLaplace {
 public:
  MultiLaplace(const MultiSpec& spec, int max_batch, cudaStream_t stream);
  ~MultiLaplace();

  // coef: [B][G][ncomp] host; p1scale: [B][G] host (nullptr = 1).
  void eval(int B, const double* coef, const double* p1scale, int flags, MultiOut& out);

  int G() const { return spec_.G; }
  int64_t n() const { return spec_.n; }
  int64_t nobs() const { return spec_.nobs; }
  int ncomp() const { return spec_.ncomp; }
  int max_batch() const { return max_batch_; }
  const std::vector<int64_t>& lat_off() const { return spec_.lat_off; }
  const MultiSpec& spec() const { return spec_; }
  const double* d_x() const { return x_.p; }      // [B][n]
  const double* d_var() const { return var_.p; }  // [B][n]
  GpuFactor& factor() { return *F_; }
  int64_t launches() const { return launches_ + F_->launches(); }
  cudaStream_t stream() const { return stream_; }

 private:
  void eval_lik(int B, const double* d_xsrc);
  // posterior with `skip`: the pairs whose mask entry (active_, [B][G]) is 0 keep their factor
  void factor(int B, bool posterior, bool skip = false);

  MultiSpec spec_;
  int max_batch_;
  cudaStream_t stream_;
  int64_t nnz_ = 0;
  std::unique_ptr<GpuFactor> F_;
  DBuf<double> comp_, y_, p1_, p2_, av_, atv_, cprod_;
  DBuf<int64_t> qcp_, acp_, atp_, opptr_, oppos_, latoff_, obsoff_, poff_, eoff_;
  DBuf<int> qri_, aci_, ati_, cptr_, cobs_, segc_, sego_, pseg_;
  DBuf<unsigned char> pdiag_, active_;
  DBuf<double> coef_, p1s_, x_, xt_, step_, eta_, logp_, grad_, w_, dw_, var_, sig_, tmp_n_, tmp_o_, stats_, alpha_,
      mdiff_, scal_, ld_, red_;
  DBuf<int> bad_, st_;
  int64_t launches_ = 0;
};

// ---------------------------------------------------------------------------
// Fit of G independent models in lockstep (run_inla_inference_a_cancellable,
// inference.rs:1116-1466, per model): every model runs the batched Newton mode
// search of InlaDriver::newton on adjoint gradients with its own state (direction,
// trust radius, backtracking candidate), the Hessian for the CCD design (the
// reference's FD of values with h = max(1e-4, 0.05 max|theta_g|), or FD of
// gradients), and the CCD nodes with variances; batch b of every evaluation
// holds point b of every model, so one launch sequence serves all models.
// ---------------------------------------------------------------------------
using MultiThetaMap = std::function<int(int g, const double* theta, double* coef, double* dcoef, double* p1scale,
                                        double* dp1scale)>;
using MultiLogPrior = std::function<double(int g, const double* theta, double* grad)>;

struct MultiFitOptions {
  int hessian = 0;       // 0 FD of values (reference stencil), 1 central FD of adjoint gradients
  double f0 = 1.0;       // CCD f0
  int max_iter = 100;    // Newton iterations per model
  double tol = 1e-4;     // gradient infinity-norm tolerance
  std::function<bool()> cancel;  // polled before every evaluation; true stops with INLA_ERR_CANCELLED
};

struct MultiFitResult {
  std::vector<double> mode, hessian, mlik;   // [G][m], [G][m][m], [G]
  std::vector<double> latent_mean, latent_var;  // [n]
  std::vector<double> pred_mean, pred_var;      // [nobs]: linear predictor eta = A x per model
  // model-selection inputs: per-node predictor and its variance [K][nobs], node weights [G][K]
  // (0 for the nodes of a model without a finite node), the node of D(theta*) and the
  // likelihood p1 scale at each model's mode [G]
  std::vector<double> cond_eta, cond_eta_var, node_weight, p1scale_mode, logpost_mode;
  int K = 0, mode_index = 0;
  std::vector<int> mode_iters, status;       // [G]; status 0 ok, 1 no finite node, 2 singular Hessian
  int n_batches = 0;
  int64_t n_model_evals = 0;
  double seconds = 0.0;
};

class MultiDriver {
 public:
  MultiDriver(MultiLaplace& eng, int m, MultiThetaMap map, MultiLogPrior prior)
      : eng_(eng), m_(m), map_(std::move(map)), prior_(std::move(prior)) {}
  void fit(const double* theta0, const MultiFitOptions& opt, MultiFitResult& out);
  // f = -(mlik + log prior) [B][G] (1e12 where the Laplace evaluation failed) and its
  // gradient [B][G][m] at the theta-sets th [B][G][m]; B may exceed the engine's batch.
  void evaluate(int B, const double* th, bool want_grad, bool want_var, double* f, double* grad,
                std::vector<double>* x = nullptr, std::vector<double>* var = nullptr);

 private:
  MultiLaplace& eng_;
  int m_;
  MultiThetaMap map_;
  MultiLogPrior prior_;
  int n_batches_ = 0;
  int64_t n_model_evals_ = 0;
  std::function<bool()> cancel_;
};

}  // namespace inla
