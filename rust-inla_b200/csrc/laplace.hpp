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
//
// Hard constraints follow the reference's Augmented method (inference.rs:819-830,
// constraints.rs:268-353): the working prior is Q + kappa C^T C with kappa = 3.059023205018258e6,
// held here as one more fixed component (coefficient 1) on a pattern widened by
// the support of C^T C; the prior log-determinant takes no jitter; every Newton
// trial point and the final mode are projected onto C x = e.
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
  // hard linear constraints C x = e (ConstraintSpec, crates/inla_math/src/constraints.rs:16-25):
  // kc rows of the dense row-major kc x n matrix cA, right-hand side ce (kc = 0: none)
  int kc = 0;
  std::vector<double> cA, ce;
  int cmethod = 0;  // ConstraintMethodGpu
};

// How Q + kappa C^T C is held (the results are the same up to rounding):
//  CONSTR_AUGMENTED: as the reference builds it -- kappa C^T C added on a pattern widened by
//    its support (every constrained block becomes dense);
//  CONSTR_BORDERED: the sparse bordered matrix M = [[Q, C^T], [C, -I/kappa]] of order n + k,
//    whose Schur complement is Q + kappa C^T C: log|Q + kappa C^T C| = log|det M| + k log kappa,
//    the leading n x n block of M^-1 is (Q + kappa C^T C)^-1, and the system M [x; l] = [b; 0]
//    solves (Q + kappa C^T C) x = b. The elimination order puts, per constraint row, its
//    latest-eliminated supported node after the k border nodes, so that the nodes eliminated
//    before the border carry a positive definite block even when Q is intrinsic;
//  CONSTR_AUTO: augmented while kappa C^T C adds at most 2^22 entries, else bordered.
enum ConstraintMethodGpu : int { CONSTR_AUTO = 0, CONSTR_AUGMENTED = 1, CONSTR_BORDERED = 2 };

// HARD_CONSTRAINT_KAPPA (constraints.rs:268): the literal 3.059023205018258e6, which its
// comment calls exp(15) (that is 3.269e6); results must match the literal
constexpr double kHardConstraintKappa = 3.059023205018258e6;

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

  int64_t n() const { return n_; }               // latent dimension of the caller's model
  int64_t xstride() const { return spec_.n; }    // per-problem stride of d_x / d_var (n + k when bordered)
  bool bordered() const { return border_; }
  int64_t nobs() const { return spec_.nobs; }
  int64_t nnz() const { return nnz_; }
  int ncomp() const { return nuser_; }  // components the caller supplies coefficients for
  int nconstr() const { return spec_.kc; }
  const LaplaceSpec& spec() const { return spec_; }
  int family() const { return spec_.family; }
  int max_batch() const { return max_batch_; }
  const double* d_x() const { return x_.p; }      // [B][n] modes
  const double* d_var() const { return var_.p; }  // [B][n] marginal variances
  const double* d_eta() const { return eta_.p; }  // [B][nobs] predictor at the mode
  // the model's A (CSR; d_acp() is nullptr when eta = x) and observations on the device
  const int64_t* d_acp() const { return spec_.identity_a ? nullptr : acp_.p; }
  const int* d_aci() const { return aci_.p; }
  const double* d_av() const { return av_.p; }
  const double* d_y() const { return y_.p; }
  const double* d_p1() const { return spec_.p1.empty() ? nullptr : p1_.p; }
  const double* d_p2() const { return spec_.p2.empty() ? nullptr : p2_.p; }
  GpuFactor& factor() { return *F_; }
  int64_t launches() const { return launches_ + F_->launches(); }
  cudaStream_t stream() const { return stream_; }

 private:
  void fill_factor(int B, bool posterior, double diag_add);
  void eval_lik(int B, const double* d_xsrc);
  void augment_constraints();         // host, once: C, C^T, (C C^T)^-1, then one of
  void augment_dense();               //   widen the pattern by supp(C^T C), append kappa C^T C
  void augment_bordered();            //   border the pattern with C and -I/kappa (order n + k)
  // x <- x - C^T (C C^T)^-1 (C x - e) for B problems; bordered, the multiplier entries are set to
  // kappa C x when `final` (the mode, whose x^T M x is then x^T (Q + kappa C^T C) x) and to 0
  // otherwise (Newton iterates: the right-hand side b - M x is then [A^T g - Q x; -C x] and the
  // solve returns the new multiplier directly, with no kappa-sized terms in the right-hand side)
  void project(int B, double* d_x, bool final = false);

  LaplaceSpec spec_;
  int nuser_ = 0;
  int64_t n_ = 0;        // the caller's latent dimension
  bool border_ = false;  // CONSTR_BORDERED in use
  std::vector<int64_t> border_perm_;  // elimination order of the bordered matrix
  // host copies of C (CSR) for the two constructions
  std::vector<int64_t> h_crp_;
  std::vector<int> h_cci_;
  std::vector<double> h_cv_;
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
  // constraints: C and C^T in CSR, e, (C C^T)^-1, residuals [B][kc], max |x_trial - x| [B]
  DBuf<int64_t> crp_, ctp_;
  DBuf<int> cci_, cta_;
  DBuf<double> cv_, ctv_, ce_, cginv_, cres_, mdiff_;
  DBuf<int> bad_, stp_;
  int64_t launches_ = 0;
  std::vector<double> h_buf_;
};

}  // namespace inla
