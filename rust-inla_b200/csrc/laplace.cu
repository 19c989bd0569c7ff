// Batched Laplace engine: host control of the device Newton loop.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "laplace.hpp"
#include "laplace_kernels.cuh"

namespace inla {

namespace {
inline int cdiv(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
inline unsigned grid1(int64_t n, int threads = 256, int cap = 2048) {
  return (unsigned)std::max(1, std::min<int>(cdiv(n, threads), cap));
}
// CTAs of a multi-CTA reduction over len elements (at least one).
inline unsigned nchunks(int64_t len, int per_cta) { return (unsigned)std::max(1, cdiv(len, per_cta)); }
}  // namespace

// u[b][j] = sum_a A[a,j] v[b][a]   (A^T in CSR)
__global__ void k_spmv_at(int n, const int64_t* __restrict__ atp, const int* __restrict__ ati,
                          const double* __restrict__ atv, int64_t nobs, const double* __restrict__ v,
                          double* __restrict__ u) {
  const int b = blockIdx.y;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double s = 0.0;
    if (atp) {
      for (int64_t a = atp[j]; a < atp[j + 1]; ++a) s += atv[a] * v[(int64_t)b * nobs + ati[a]];
    } else {
      s = v[(int64_t)b * nobs + j];
    }
    u[(int64_t)b * n + j] = s;
  }
}

__global__ void k_mul(int64_t len, const double* a, const double* b, double* c) {  // c may alias a
  const int bb = blockIdx.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
    c[(int64_t)bb * len + i] = a[(int64_t)bb * len + i] * b[(int64_t)bb * len + i];
}

LaplaceEngine::LaplaceEngine(const LaplaceSpec& spec, int max_batch, cudaStream_t stream)
    : spec_(spec), max_batch_(max_batch), stream_(stream) {
  const int64_t n = spec_.n;
  if (n <= 0 || (int64_t)spec_.colptr.size() != n + 1) throw std::runtime_error("laplace: invalid pattern");
  nnz_ = spec_.colptr[n];
  if ((int64_t)spec_.rowidx.size() != nnz_) throw std::runtime_error("laplace: rowidx length");
  if (spec_.ncomp < 1 || spec_.ncomp > 8) throw std::runtime_error("laplace: 1..8 precision components supported");
  if ((int64_t)spec_.comp.size() != spec_.ncomp * nnz_) throw std::runtime_error("laplace: component values length");
  const int64_t nobs = spec_.nobs;
  if (spec_.identity_a && nobs != n) throw std::runtime_error("laplace: identity projector needs nobs == n");
  if ((int64_t)spec_.y.size() != nobs) throw std::runtime_error("laplace: y length");
  if (spec_.family < 0 || spec_.family > 3) throw std::runtime_error("laplace: unknown family");
  for (int64_t c = 0; c < n; ++c)
    if (!std::is_sorted(spec_.rowidx.begin() + spec_.colptr[c], spec_.rowidx.begin() + spec_.colptr[c + 1]))
      throw std::runtime_error("laplace: pattern row indices must be sorted");

  const auto t0 = std::chrono::steady_clock::now();
  Symbolic sym;
  SymbolicOptions opt;
  opt.ordering = spec_.ordering;
  analyze(n, spec_.colptr.data(), spec_.rowidx.data(), opt, nullptr, sym);
  const auto t1 = std::chrono::steady_clock::now();
  // twice the slots: a Gaussian evaluation factorizes prior representatives and
  // posterior problems in one batch
  F_.reset(new GpuFactor(sym, 2 * max_batch, stream_));
  const auto t2 = std::chrono::steady_clock::now();
  if (std::getenv("INLA_DEBUG"))
    std::fprintf(stderr, "laplace setup: symbolic %.1f ms, device factor %.1f ms\n",
                 std::chrono::duration<double, std::milli>(t1 - t0).count(),
                 std::chrono::duration<double, std::milli>(t2 - t1).count());

  auto find = [&](int64_t row, int64_t col) -> int64_t {
    auto b = spec_.rowidx.begin() + spec_.colptr[col], e = spec_.rowidx.begin() + spec_.colptr[col + 1];
    auto it = std::lower_bound(b, e, row);
    if (it == e || *it != row) return -1;
    return it - spec_.rowidx.begin();
  };
  std::vector<unsigned char> pdiag(nnz_, 0);
  std::vector<int> qri(nnz_);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = spec_.colptr[c]; p < spec_.colptr[c + 1]; ++p) {
      qri[p] = (int)spec_.rowidx[p];
      if (spec_.rowidx[p] == c) pdiag[p] = 1;
    }
  for (int64_t c = 0; c < n; ++c)
    if (find(c, c) < 0) throw std::runtime_error("laplace: pattern must contain the diagonal");

  // observation contributions to A^T diag(w) A on the pattern, A^T, pair positions
  std::vector<int64_t> acp, opptr(nobs + 1, 0), oppos;
  std::vector<int> aci;
  std::vector<double> av;
  if (spec_.identity_a) {
    acp.resize(nobs + 1);
    aci.resize(nobs);
    av.assign(nobs, 1.0);
    for (int64_t i = 0; i <= nobs; ++i) acp[i] = i;
    for (int64_t i = 0; i < nobs; ++i) aci[i] = (int)i;
  } else {
    if ((int64_t)spec_.acp.size() != nobs + 1) throw std::runtime_error("laplace: A row pointer length");
    acp = spec_.acp;
    aci.resize(spec_.aci.size());
    for (size_t a = 0; a < spec_.aci.size(); ++a) {
      if (spec_.aci[a] < 0 || spec_.aci[a] >= n) throw std::runtime_error("laplace: A column out of range");
      aci[a] = (int)spec_.aci[a];
    }
    av = spec_.av;
  }
  std::vector<int64_t> cnt(nnz_ + 1, 0);
  for (int64_t i = 0; i < nobs; ++i) {
    int64_t na = acp[i + 1] - acp[i];
    opptr[i + 1] = opptr[i] + na * na;
  }
  oppos.resize(opptr[nobs]);
  for (int64_t i = 0; i < nobs; ++i) {
    int64_t q = opptr[i];
    for (int64_t a = acp[i]; a < acp[i + 1]; ++a)
      for (int64_t c = acp[i]; c < acp[i + 1]; ++c, ++q) {
        int64_t p = find(aci[a], aci[c]);
        if (p < 0) throw std::runtime_error("laplace: pattern must contain A^T A");
        oppos[q] = p;
        cnt[p + 1]++;
      }
  }
  for (int64_t p = 0; p < nnz_; ++p) cnt[p + 1] += cnt[p];
  if (cnt[nnz_] >= (1LL << 31)) throw std::runtime_error("laplace: too many observation contributions");
  std::vector<int> cptr(nnz_ + 1), cobs(cnt[nnz_]);
  std::vector<double> cprod(cnt[nnz_]);
  {
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t i = 0; i < nobs; ++i) {
      int64_t q = opptr[i];
      for (int64_t a = acp[i]; a < acp[i + 1]; ++a)
        for (int64_t c = acp[i]; c < acp[i + 1]; ++c, ++q) {
          int64_t p = oppos[q];
          cobs[fill[p]] = (int)i;
          cprod[fill[p]++] = av[a] * av[c];
        }
    }
    for (int64_t p = 0; p <= nnz_; ++p) cptr[p] = (int)cnt[p];
  }
  // A^T in CSR
  std::vector<int64_t> atp(n + 1, 0);
  for (size_t a = 0; a < aci.size(); ++a) atp[aci[a] + 1]++;
  for (int64_t j = 0; j < n; ++j) atp[j + 1] += atp[j];
  std::vector<int> ati(aci.size());
  std::vector<double> atv(aci.size());
  {
    std::vector<int64_t> fill(atp.begin(), atp.end() - 1);
    for (int64_t i = 0; i < nobs; ++i)
      for (int64_t a = acp[i]; a < acp[i + 1]; ++a) {
        ati[fill[aci[a]]] = (int)i;
        atv[fill[aci[a]]++] = av[a];
      }
  }

  comp_.upload(spec_.comp, stream_);
  y_.upload(spec_.y, stream_);
  if (!spec_.p1.empty()) p1_.upload(spec_.p1, stream_);
  if (!spec_.p2.empty()) p2_.upload(spec_.p2, stream_);
  qcp_.upload(spec_.colptr, stream_);
  qri_.upload(qri, stream_);
  pdiag_.upload(pdiag, stream_);
  cptr_.upload(cptr, stream_);
  cobs_.upload(cobs, stream_);
  cprod_.upload(cprod, stream_);
  opptr_.upload(opptr, stream_);
  oppos_.upload(oppos, stream_);
  if (!spec_.identity_a) {
    acp_.upload(acp, stream_);
    aci_.upload(aci, stream_);
    av_.upload(av, stream_);
    atp_.upload(atp, stream_);
    ati_.upload(ati, stream_);
    atv_.upload(atv, stream_);
  } else {
    acp_.upload(acp, stream_);  // needed by the predictor-variance kernel
    av_.upload(av, stream_);
  }
  const size_t B = max_batch_;
  coef_.alloc(B * spec_.ncomp);
  coefp_.alloc(B * spec_.ncomp);
  coefall_.alloc(2 * B * spec_.ncomp);
  p1s_.alloc(B);
  x_.alloc(B * n);
  xt_.alloc(B * n);
  step_.alloc(B * n);
  tmp_n_.alloc(B * n);
  var_.alloc(B * n);
  eta_.alloc(B * std::max<int64_t>(nobs, 1));
  logp_.alloc(B * std::max<int64_t>(nobs, 1));
  grad_.alloc(B * std::max<int64_t>(nobs, 1));
  w_.alloc(B * std::max<int64_t>(nobs, 1));
  dw_.alloc(B * std::max<int64_t>(nobs, 1));
  tmp_o_.alloc(B * std::max<int64_t>(nobs, 1));
  sig_.alloc(B * nnz_);
  red_.alloc(B * 4 * (spec_.ncomp + 1) + B * 8);
  {
    const int64_t maxch = std::max<int64_t>({1, (nnz_ + kRedChunk - 1) / kRedChunk, (nobs + kRedChunk - 1) / kRedChunk,
                                             (n + kColChunk - 1) / kColChunk});
    gpart_.alloc(B * maxch * 9);
    gtick_.alloc(B);
    INLA_CUDA(cudaMemsetAsync(gtick_.p, 0, sizeof(unsigned) * B, stream_));
  }
  stats_.alloc(2 * B);
  alpha_.alloc(B);
  ldp_.alloc(B);
  bad_.alloc(B);
  stp_.alloc(B);
  INLA_CUDA(cudaStreamSynchronize(stream_));
}

LaplaceEngine::~LaplaceEngine() = default;

void LaplaceEngine::fill_factor(int B, bool posterior, double diag_add) {
  F_->factor_model(spec_.ncomp, comp_.p, coef_.p, diag_add, pdiag_.p, cptr_.p, cobs_.p, cprod_.p,
                   posterior ? w_.p : nullptr, spec_.nobs, B, posterior ? 0 : B, diag_add);
}

void LaplaceEngine::eval_lik(int B, const double* d_xsrc) {
  const int64_t nobs = spec_.nobs;
  k_spmv_a<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(nobs, (int)spec_.n, spec_.identity_a ? nullptr : acp_.p, aci_.p,
                                                      av_.p, d_xsrc, eta_.p);
  INLA_CUDA(cudaMemsetAsync(bad_.p, 0, sizeof(int) * B, stream_));
  k_eval_lik<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(spec_.family, nobs, eta_.p, y_.p, p1_.p, p2_.p, p1s_.p,
                                                        logp_.p, grad_.p, w_.p, dw_.p, bad_.p);
  launches_ += 2;
}

void LaplaceEngine::eval(int B, const double* coef, const double* p1scale, int flags, LaplaceOut& R) {
  if (B < 1 || B > max_batch_) throw std::runtime_error("laplace: batch size out of range");
  const int64_t n = spec_.n, nobs = spec_.nobs;
  const int T = spec_.ncomp;
  const int T1 = T + 1;
  R.mlik.assign(B, NAN);
  R.ld_prior.assign(B, NAN);
  R.ld_post.assign(B, NAN);
  R.loglik.assign(B, NAN);
  R.quad.assign(B, NAN);
  R.dll.assign(B, 0.0);
  R.status.assign(B, LAP_OK);
  R.iters.assign(B, 0);
  R.trP.assign((size_t)B * T1, 0.0);
  R.trQ.assign((size_t)B * T1, 0.0);
  R.xMx.assign((size_t)B * T1, 0.0);
  R.zMx.assign((size_t)B * T1, 0.0);

  INLA_CUDA(cudaMemcpyAsync(coef_.p, coef, sizeof(double) * B * T, cudaMemcpyHostToDevice, stream_));
  std::vector<double> ones(B, 1.0);
  INLA_CUDA(cudaMemcpyAsync(p1s_.p, p1scale ? p1scale : ones.data(), sizeof(double) * B, cudaMemcpyHostToDevice,
                            stream_));
  const bool grad = flags & LAP_GRADIENT;
  const bool want_var = (flags & LAP_VARIANCES) || grad;
  double* d_trP = red_.p;
  double* d_trQ = red_.p + (size_t)B * T1;
  double* d_xMx = red_.p + (size_t)2 * B * T1;
  double* d_zMx = red_.p + (size_t)3 * B * T1;
  double* d_scal = red_.p + (size_t)4 * B * T1;  // [B][8]: loglik, dll

  // ---- prior log-determinant: Q + 1e-12 I (inference.rs:831-837) ----------
  // Batch members whose prior coefficient vectors are proportional (c_b = s c_r,
  // s > 0; e.g. FD-stencil points that differ only in a precision scale) share one
  // prior factorization: log|Q_b| = log|Q_r| + n log s and tr(Q_b^-1 M_t) =
  // tr(Q_r^-1 M_t) / s. The 1e-12 jitter of the representative then stands for a
  // jitter of 1e-12 / s on the member, a log-det difference of about
  // 1e-12 |1/s - 1| tr(Q_r^-1). Identical vectors (s = 1) are shared exactly.
  std::vector<int> prep(B);
  std::vector<double> pscale(B, 1.0);
  std::vector<int> reps;
  for (int b = 0; b < B; ++b) {
    const double* cb = coef + (size_t)b * T;
    int t0 = 0;
    while (t0 < T && cb[t0] == 0.0) ++t0;
    int match = -1;
    double ratio = 1.0;
    if (!(flags & LAP_NO_PRIOR_SHARING) && t0 < T) {
      for (size_t g = 0; g < reps.size() && match < 0; ++g) {
        const double* cr = coef + (size_t)reps[g] * T;
        if (cr[t0] == 0.0) continue;
        const double rt = cb[t0] / cr[t0];
        if (!(rt > 0.0) || !std::isfinite(rt)) continue;
        bool same = true;
        for (int t = 0; t < T && same; ++t) {
          const double d = cb[t] - rt * cr[t];
          same = (t < t0) ? cr[t] == 0.0 : std::fabs(d) <= 1e-13 * std::fabs(cb[t]) + 1e-300;
        }
        if (same) match = (int)g, ratio = rt;
      }
    }
    if (match < 0) {
      match = (int)reps.size();
      reps.push_back(b);
      ratio = 1.0;
    }
    prep[b] = match;
    pscale[b] = ratio;
  }
  const int Bp = (int)reps.size();
  {
    std::vector<double> cp((size_t)Bp * T);
    for (int g = 0; g < Bp; ++g)
      for (int t = 0; t < T; ++t) cp[(size_t)g * T + t] = coef[(size_t)reps[g] * T + t];
    INLA_CUDA(cudaMemcpyAsync(coefp_.p, cp.data(), sizeof(double) * Bp * T, cudaMemcpyHostToDevice, stream_));
  }
  // Gaussian likelihood: the posterior precision does not depend on the mode, so
  // the prior representatives (slots [0, Bp)) and the posterior problems (slots
  // [Bp, Bp + B)) are factorized -- and, for the gradient, selectively inverted --
  // in one batched launch sequence: the latency-bound top levels of the
  // elimination tree are paid once instead of twice.
  const bool merged = spec_.family == FAM_GAUSSIAN;
  const int post0 = merged ? Bp : 0;  // slot of the first posterior problem
  auto prior_traces = [&]() {
    k_pattern_full<<<dim3(grid1(nnz_), Bp), 256, 0, stream_>>>(nnz_, F_->d_spos_full(), F_->d_sigma(0),
                                                               F_->front_total(), sig_.p);
    k_trace_contract_g<<<dim3(nchunks(nnz_, kRedChunk), Bp), 256, 0, stream_>>>(
        nnz_, T, comp_.p, sig_.p, cptr_.p, cobs_.p, cprod_.p, nullptr, nobs, gpart_.p, gtick_.p, d_trP);
    launches_ += 2;
  };
  if (!merged) {
    F_->factor_model(spec_.ncomp, comp_.p, coefp_.p, 1e-12, pdiag_.p, cptr_.p, cobs_.p, cprod_.p, nullptr,
                     spec_.nobs, Bp, Bp);
    INLA_CUDA(cudaMemcpyAsync(ldp_.p, F_->d_logdet(), sizeof(double) * Bp, cudaMemcpyDeviceToDevice, stream_));
    INLA_CUDA(cudaMemcpyAsync(stp_.p, F_->d_status(), sizeof(int) * Bp, cudaMemcpyDeviceToDevice, stream_));
    if (grad) {
      F_->selinv(Bp);
      prior_traces();
    }
  }

  // ---- mode --------------------------------------------------------------------
  std::vector<int> prior_status(B);
  INLA_CUDA(cudaMemsetAsync(x_.p, 0, sizeof(double) * B * n, stream_));
  const int64_t at_null = 0;
  (void)at_null;
  const int64_t* atp = spec_.identity_a ? nullptr : atp_.p;
  auto newton_system = [&](const double* d_x) {
    eval_lik(B, d_x);
    fill_factor(B, true, 0.0);
    k_newton_rhs<<<dim3(grid1(n), B), 256, 0, stream_>>>((int)n, T, qcp_.p, qri_.p, comp_.p, nnz_, coef_.p, atp,
                                                         ati_.p, atv_.p, nobs, grad_.p, d_x, step_.p);
    F_->solve(step_.p, n, B);
    k_step_stats<256><<<B, 256, 0, stream_>>>((int)n, step_.p, stats_.p);
    launches_ += 2;
  };
  std::vector<double> st(2 * B);
  std::vector<int> bad(B), pst(B);
  auto fetch = [&]() {
    INLA_CUDA(cudaMemcpyAsync(st.data(), stats_.p, sizeof(double) * 2 * B, cudaMemcpyDeviceToHost, stream_));
    INLA_CUDA(cudaMemcpyAsync(bad.data(), bad_.p, sizeof(int) * B, cudaMemcpyDeviceToHost, stream_));
    INLA_CUDA(cudaMemcpyAsync(pst.data(), F_->d_status() + post0, sizeof(int) * B, cudaMemcpyDeviceToHost, stream_));
    INLA_CUDA(cudaStreamSynchronize(stream_));
  };
  std::vector<char> active(B, 1);
  if (spec_.family == FAM_GAUSSIAN) {
    // closed form (inference.rs:845-870): one Newton system from x = 0, with the
    // prior representatives in the same factorization
    eval_lik(B, x_.p);
    INLA_CUDA(cudaMemcpyAsync(coefall_.p, coefp_.p, sizeof(double) * Bp * T, cudaMemcpyDeviceToDevice, stream_));
    INLA_CUDA(cudaMemcpyAsync(coefall_.p + (size_t)Bp * T, coef_.p, sizeof(double) * B * T,
                              cudaMemcpyDeviceToDevice, stream_));
    F_->factor_model(spec_.ncomp, comp_.p, coefall_.p, 1e-12, pdiag_.p, cptr_.p, cobs_.p, cprod_.p, w_.p, spec_.nobs,
                     Bp + B, Bp, 0.0);
    INLA_CUDA(cudaMemcpyAsync(ldp_.p, F_->d_logdet(), sizeof(double) * Bp, cudaMemcpyDeviceToDevice, stream_));
    INLA_CUDA(cudaMemcpyAsync(stp_.p, F_->d_status(), sizeof(int) * Bp, cudaMemcpyDeviceToDevice, stream_));
    k_newton_rhs<<<dim3(grid1(n), B), 256, 0, stream_>>>((int)n, T, qcp_.p, qri_.p, comp_.p, nnz_, coef_.p, atp,
                                                         ati_.p, atv_.p, nobs, grad_.p, x_.p, step_.p);
    F_->solve(step_.p, n, B, post0);
    k_step_stats<256><<<B, 256, 0, stream_>>>((int)n, step_.p, stats_.p);
    launches_ += 2;
    INLA_CUDA(cudaMemcpyAsync(x_.p, step_.p, sizeof(double) * B * n, cudaMemcpyDeviceToDevice, stream_));
    fetch();
    for (int b = 0; b < B; ++b) {
      R.iters[b] = 1;
      if (bad[b] & 1) R.status[b] = LAP_BAD_LIKELIHOOD;
      else if (pst[b]) R.status[b] = LAP_SINGULAR_POST;
      else if (st[2 * b + 1] == 0.0) R.status[b] = LAP_NONFINITE_STEP;
    }
  } else {
    std::vector<double> alpha(B, 0.0), max_step(B, 0.0);
    int it = 0;
    for (; it < spec_.max_iter; ++it) {
      newton_system(x_.p);
      fetch();
      bool any = false;
      for (int b = 0; b < B; ++b) {
        alpha[b] = 0.0;
        if (!active[b]) continue;
        if (bad[b] & 1) R.status[b] = LAP_BAD_LIKELIHOOD;
        else if (pst[b]) R.status[b] = LAP_SINGULAR_POST;
        else if (st[2 * b + 1] == 0.0) R.status[b] = LAP_NONFINITE_STEP;
        if (R.status[b] != LAP_OK) {
          active[b] = 0;
          continue;
        }
        max_step[b] = st[2 * b];
        alpha[b] = max_step[b] > 10.0 ? 10.0 / max_step[b] : 1.0;
        any = true;
      }
      if (!any) break;
      // backtracking while the trial objective is non-finite (inference.rs:888-914)
      std::vector<char> need(B, 0);
      for (int b = 0; b < B; ++b) need[b] = active[b];
      for (int bt = 0; bt < 12; ++bt) {
        INLA_CUDA(cudaMemcpyAsync(alpha_.p, alpha.data(), sizeof(double) * B, cudaMemcpyHostToDevice, stream_));
        k_axpy_trial<<<dim3(grid1(n), B), 256, 0, stream_>>>((int)n, x_.p, step_.p, alpha_.p, xt_.p);
        ++launches_;
        eval_lik(B, xt_.p);
        INLA_CUDA(cudaMemcpyAsync(bad.data(), bad_.p, sizeof(int) * B, cudaMemcpyDeviceToHost, stream_));
        INLA_CUDA(cudaStreamSynchronize(stream_));
        bool again = false;
        for (int b = 0; b < B; ++b) {
          if (!need[b]) continue;
          if (bad[b] == 0) {
            need[b] = 0;
            continue;
          }
          alpha[b] *= 0.5;
          if (alpha[b] < 1e-8) {
            R.status[b] = LAP_NONFINITE_STEP;
            active[b] = 0;
            need[b] = 0;
            alpha[b] = 0.0;
            continue;
          }
          again = true;
        }
        if (!again) break;
      }
      // x <- x_trial for active problems (alpha = 0 keeps the others unchanged)
      INLA_CUDA(cudaMemcpyAsync(alpha_.p, alpha.data(), sizeof(double) * B, cudaMemcpyHostToDevice, stream_));
      k_axpy_trial<<<dim3(grid1(n), B), 256, 0, stream_>>>((int)n, x_.p, step_.p, alpha_.p, xt_.p);
      ++launches_;
      INLA_CUDA(cudaMemcpyAsync(x_.p, xt_.p, sizeof(double) * B * n, cudaMemcpyDeviceToDevice, stream_));
      bool left = false;
      for (int b = 0; b < B; ++b) {
        if (!active[b]) continue;
        R.iters[b] = it + 1;
        const double max_diff = alpha[b] * max_step[b];
        if (max_diff < spec_.tol || max_step[b] < spec_.tol) active[b] = 0;  // converged
        else left = true;
      }
      if (!left) break;
    }
    for (int b = 0; b < B; ++b)
      if (active[b] && R.status[b] == LAP_OK) R.status[b] = LAP_NONCONVERGED;
    // confirmation refactorization at x* (inference.rs:923-937)
    eval_lik(B, x_.p);
    fill_factor(B, true, 0.0);
  }

  // ---- marginal likelihood pieces (inference.rs:953-972) ------------------------
  eval_lik(B, x_.p);
  k_row_sum_g<<<dim3(nchunks(nobs, kRedChunk), B), 256, 0, stream_>>>(nobs, logp_.p, gpart_.p, gtick_.p, d_scal);
  k_quad_forms_g<<<dim3(nchunks(n, kColChunk), B), 256, 0, stream_>>>((int)n, T, qcp_.p, qri_.p, comp_.p, nnz_,
                                                                      coef_.p, nullptr, x_.p, gpart_.p, gtick_.p,
                                                                      d_xMx);
  launches_ += 2;
  if (spec_.family == FAM_GAUSSIAN && grad) {
    k_gauss_dll_g<<<dim3(nchunks(nobs, kRedChunk), B), 256, 0, stream_>>>(nobs, eta_.p, y_.p, w_.p, gpart_.p,
                                                                          gtick_.p, d_scal + B);
    ++launches_;
  }
  std::vector<double> ldpost(B), ldprior(B), scal(2 * B), xmx((size_t)B * T1);
  INLA_CUDA(cudaMemcpyAsync(ldpost.data(), F_->d_logdet() + post0, sizeof(double) * B, cudaMemcpyDeviceToHost,
                            stream_));
  INLA_CUDA(cudaMemcpyAsync(pst.data(), F_->d_status() + post0, sizeof(int) * B, cudaMemcpyDeviceToHost, stream_));

  // ---- selected inverse of Q_post: variances and trace pieces --------------------
  if (merged && grad) {
    F_->selinv(Bp + B, 0);  // prior representatives and posterior problems together
    prior_traces();
  }
  if (want_var) {
    if (!(merged && grad)) F_->selinv(B, post0);
    F_->extract_diag(var_.p, n, B, post0);
    if (grad) {
      k_pattern_full<<<dim3(grid1(nnz_), B), 256, 0, stream_>>>(nnz_, F_->d_spos_full(), F_->d_sigma(post0),
                                                                F_->front_total(), sig_.p);
      k_trace_contract_g<<<dim3(nchunks(nnz_, kRedChunk), B), 256, 0, stream_>>>(
          nnz_, T, comp_.p, sig_.p, cptr_.p, cobs_.p, cprod_.p, w_.p, nobs, gpart_.p, gtick_.p, d_trQ);
      launches_ += 2;
      if (spec_.family != FAM_GAUSSIAN) {
        // implicit term: u = A^T (dw .* v), v_i = a_i' Sigma a_i; z = Q_post^-1 u
        k_predictor_var<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(nobs, acp_.p, av_.p, oppos_.p, opptr_.p, sig_.p,
                                                                   nnz_, tmp_o_.p);
        k_mul<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(nobs, tmp_o_.p, dw_.p, tmp_o_.p);
        k_spmv_at<<<dim3(grid1(n), B), 256, 0, stream_>>>((int)n, atp, ati_.p, atv_.p, nobs, tmp_o_.p, tmp_n_.p);
        F_->solve(tmp_n_.p, n, B);
        k_quad_forms_g<<<dim3(nchunks(n, kColChunk), B), 256, 0, stream_>>>(
            (int)n, T, qcp_.p, qri_.p, comp_.p, nnz_, coef_.p, tmp_n_.p, x_.p, gpart_.p, gtick_.p, d_zMx);
        launches_ += 4;
      }
    }
  }
  INLA_CUDA(cudaMemcpyAsync(ldprior.data(), ldp_.p, sizeof(double) * Bp, cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaMemcpyAsync(prior_status.data(), stp_.p, sizeof(int) * Bp, cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaMemcpyAsync(scal.data(), d_scal, sizeof(double) * 2 * B, cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaMemcpyAsync(xmx.data(), d_xMx, sizeof(double) * B * T1, cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaMemcpyAsync(bad.data(), bad_.p, sizeof(int) * B, cudaMemcpyDeviceToHost, stream_));
  std::vector<double> trp_rep;
  if (grad) {
    trp_rep.resize((size_t)Bp * T1);
    INLA_CUDA(cudaMemcpyAsync(trp_rep.data(), d_trP, sizeof(double) * Bp * T1, cudaMemcpyDeviceToHost, stream_));
    INLA_CUDA(cudaMemcpyAsync(R.trQ.data(), d_trQ, sizeof(double) * B * T1, cudaMemcpyDeviceToHost, stream_));
    if (spec_.family != FAM_GAUSSIAN)
      INLA_CUDA(cudaMemcpyAsync(R.zMx.data(), d_zMx, sizeof(double) * B * T1, cudaMemcpyDeviceToHost, stream_));
  }
  INLA_CUDA(cudaStreamSynchronize(stream_));
  INLA_CUDA(cudaGetLastError());
  // expand the shared prior results to every batch member (representatives were
  // evaluated in slots 0..Bp-1)
  {
    std::vector<double> ldp_rep(ldprior.begin(), ldprior.begin() + Bp);
    std::vector<int> stp_rep(prior_status.begin(), prior_status.begin() + Bp);
    for (int b = 0; b < B; ++b) {
      const int g = prep[b];
      const double sc = pscale[b];
      ldprior[b] = ldp_rep[g] + (double)n * std::log(sc);
      prior_status[b] = stp_rep[g];
      if (grad)
        for (int t = 0; t < T1; ++t) R.trP[(size_t)b * T1 + t] = trp_rep[(size_t)g * T1 + t] / sc;
    }
  }

  for (int b = 0; b < B; ++b) {
    if (prior_status[b]) R.status[b] = LAP_SINGULAR_PRIOR;
    if (R.status[b] == LAP_OK && pst[b]) R.status[b] = LAP_SINGULAR_POST;
    if (R.status[b] == LAP_OK && (bad[b] & 1)) R.status[b] = LAP_BAD_LIKELIHOOD;
    R.ld_prior[b] = ldprior[b];
    R.ld_post[b] = ldpost[b];
    R.loglik[b] = scal[b];
    R.dll[b] = scal[B + b];
    R.quad[b] = xmx[(size_t)b * T1];
    for (int t = 0; t < T; ++t) R.xMx[(size_t)b * T1 + t] = xmx[(size_t)b * T1 + 1 + t];
    R.mlik[b] = R.status[b] == LAP_OK ? R.loglik[b] - 0.5 * R.quad[b] + 0.5 * R.ld_prior[b] - 0.5 * R.ld_post[b]
                                      : NAN;
  }
}

}  // namespace inla
