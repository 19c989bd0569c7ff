// Batched Laplace evaluation at B theta-points sharing one symbolic analysis:
// prior log-determinant, Newton mode of pi(x | theta, y), posterior
// log-determinant, marginal likelihood, marginal variances (selected
// inverse) and the trace / quadratic-form pieces of the adjoint gradient.
//
// Reference control flow: find_latent_mode_a_with_solver
// (crates/inla_stats/src/inference.rs:776-975) — prior factorization of
// Q + 1e-12 I, Gaussian-identity closed form (845-870), Newton loop with
// step cap 10, at most 12 halvings while the objective is non-finite,
// convergence when max|dx| < tol or max|step| < tol, confirmation
// refactorization at x*, mlik = loglik - x*'Qx*/2 + log|Q|/2 - log|Q_post|/2.
#pragma once
#include <memory>
#include <vector>

#include "gpu_factor.hpp"

namespace inla {

struct LaplaceSpec {
  int64_t n = 0;
  std::vector<int64_t> colptr, rowidx;  // full symmetric pattern (must contain A^T A and the diagonal)
  int ncomp = 0;
  std::vector<double> comp;             // [ncomp][nnz]: Q(theta) = sum_t coef_t comp_t
  int64_t nobs = 0;
  bool identity_a = false;              // eta = x (nobs == n)
  std::vector<int64_t> acp, aci;        // A in CSR (nobs x n)
  std::vector<double> av;
  int family = 0;
  std::vector<double> y, p1, p2;        // p1 may be scaled per problem (family theta)
  int max_iter = 200;
  double tol = 1e-5;
  int ordering = ORDER_AMD;
};

enum LaplaceFlags : int { LAP_VARIANCES = 1, LAP_GRADIENT = 2, LAP_MODE = 4, LAP_NO_PRIOR_SHARING = 8 };

// Per-problem status (also reported through the C ABI).
enum LaplaceStatus : int {
  LAP_OK = 0,
  LAP_SINGULAR_PRIOR = 1,
  LAP_SINGULAR_POST = 2,
  LAP_BAD_LIKELIHOOD = 3,
  LAP_NONFINITE_STEP = 4,
  LAP_NONCONVERGED = 5,
};

struct LaplaceOut {
  // per problem
  std::vector<double> mlik, ld_prior, ld_post, loglik, quad, dll;
  std::vector<int> status, iters;
  // per problem, ncomp+1 each: trP[t]=tr(Sigma_prior M_t); trQ[t]=tr(Sigma_post M_t),
  // trQ[ncomp]=tr(Sigma_post A^T W A); xMx[t]=x*'M_t x*; zMx[t]=z'M_t x* (GLM implicit term)
  std::vector<double> trP, trQ, xMx, zMx;
};

class LaplaceEngine {
 public:
  LaplaceEngine(const LaplaceSpec& spec, int max_batch, cudaStream_t stream);
  ~LaplaceEngine();

  // coef: [B][ncomp] host; p1scale: [B] host (nullptr = 1).
  void eval(int B, const double* coef, const double* p1scale, int flags, LaplaceOut& out);

  int64_t n() const { return spec_.n; }
  int64_t nobs() const { return spec_.nobs; }
  int64_t nnz() const { return nnz_; }
  int ncomp() const { return spec_.ncomp; }
  int family() const { return spec_.family; }
  int max_batch() const { return max_batch_; }
  const double* d_x() const { return x_.p; }      // [B][n] modes
  const double* d_var() const { return var_.p; }  // [B][n] marginal variances
  const double* d_eta() const { return eta_.p; }  // [B][nobs] predictor at the mode
  GpuFactor& factor() { return *F_; }
  int64_t launches() const { return launches_ + F_->launches(); }
  cudaStream_t stream() const { return stream_; }

 private:
  void fill_factor(int B, bool posterior, double diag_add);
  void eval_lik(int B, const double* d_xsrc);

  LaplaceSpec spec_;
  int max_batch_;
  cudaStream_t stream_;
  int64_t nnz_ = 0;
  std::unique_ptr<GpuFactor> F_;
  // static device data
  DBuf<double> comp_, y_, p1_, p2_, av_, atv_, cprod_;
  DBuf<int64_t> qcp_, acp_, atp_, opptr_, oppos_;
  DBuf<int> qri_, aci_, ati_, cptr_, cobs_;
  DBuf<unsigned char> pdiag_;
  // per-batch work
  DBuf<double> coef_, p1s_, x_, xt_, step_, eta_, logp_, grad_, w_, dw_, var_, sig_, red_, stats_, alpha_, tmp_n_,
      tmp_o_, ldp_, gpart_, coefp_, coefall_;
  DBuf<unsigned> gtick_;  // grid-reduction partials and tickets
  DBuf<int> bad_, stp_;
  int64_t launches_ = 0;
  std::vector<double> h_buf_;
};

}  // namespace inla
