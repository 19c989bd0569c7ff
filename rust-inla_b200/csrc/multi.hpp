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
  const double* d_x() const { return x_.p; }      // [B][n]
  const double* d_var() const { return var_.p; }  // [B][n]
  GpuFactor& factor() { return *F_; }
  int64_t launches() const { return launches_ + F_->launches(); }
  cudaStream_t stream() const { return stream_; }

 private:
  void eval_lik(int B, const double* d_xsrc);
  void factor(int B, bool posterior);

  MultiSpec spec_;
  int max_batch_;
  cudaStream_t stream_;
  int64_t nnz_ = 0;
  std::unique_ptr<GpuFactor> F_;
  DBuf<double> comp_, y_, p1_, p2_, av_, atv_, cprod_;
  DBuf<int64_t> qcp_, acp_, atp_, opptr_, oppos_, latoff_, obsoff_, poff_, eoff_;
  DBuf<int> qri_, aci_, ati_, cptr_, cobs_, segc_, sego_, pseg_;
  DBuf<unsigned char> pdiag_;
  DBuf<double> coef_, p1s_, x_, xt_, step_, eta_, logp_, grad_, w_, dw_, var_, sig_, tmp_n_, tmp_o_, stats_, alpha_,
      mdiff_, scal_, ld_, red_;
  DBuf<int> bad_, st_;
  int64_t launches_ = 0;
};

}  // namespace inla
