// Multi-model Laplace engine: G independent models, one block-diagonal symbolic
// analysis, B theta-sets, per-(theta-set, model) Newton control.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>

#include "multi.hpp"
#include "multi_kernels.cuh"
#include "host_par.hpp"

namespace inla {

namespace {
inline int cdiv(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
inline unsigned grid1(int64_t n, int threads = 256, int cap = 2048) {
  return (unsigned)std::max(1, std::min<int>(cdiv(n, threads), cap));
}

// Fill-reducing order of one model's block (perm[new] = old, local indices).
std::vector<int64_t> block_order(int64_t nb, const std::vector<int64_t>& cp, const std::vector<int64_t>& ri,
                                 int ordering) {
  std::vector<int64_t> perm;
  if (ordering == ORDER_ND) {
    nd_order(nb, cp.data(), ri.data(), perm);
  } else if (ordering == ORDER_AMD) {
    amd_order(nb, cp.data(), ri.data(), perm);
  } else if (ordering == ORDER_NATURAL) {
    perm.resize(nb);
    std::iota(perm.begin(), perm.end(), 0);
  } else {
    Symbolic s;
    SymbolicOptions o;
    o.ordering = ordering;
    analyze(nb, cp.data(), ri.data(), o, nullptr, s);
    perm = s.perm;
  }
  return perm;
}
}  // namespace

MultiLaplace::MultiLaplace(const MultiSpec& spec, int max_batch, cudaStream_t stream)
    : spec_(spec), max_batch_(max_batch), stream_(stream) {
  const int G = spec_.G;
  const int64_t n = spec_.n, nobs = spec_.nobs;
  if (G < 1) throw std::runtime_error("multi: at least one model");
  if (max_batch < 1) throw std::runtime_error("multi: max_batch must be >= 1");
  if (n <= 0 || (int64_t)spec_.colptr.size() != n + 1) throw std::runtime_error("multi: invalid pattern");
  nnz_ = spec_.colptr[n];
  if ((int64_t)spec_.rowidx.size() != nnz_) throw std::runtime_error("multi: rowidx length");
  if (spec_.ncomp < 1 || spec_.ncomp > 8) throw std::runtime_error("multi: 1..8 precision components supported");
  if ((int64_t)spec_.comp.size() != spec_.ncomp * nnz_) throw std::runtime_error("multi: component values length");
  if ((int64_t)spec_.lat_off.size() != G + 1 || (int64_t)spec_.obs_off.size() != G + 1)
    throw std::runtime_error("multi: offset tables need G+1 entries");
  if (spec_.lat_off[0] != 0 || spec_.lat_off[G] != n || spec_.obs_off[0] != 0 || spec_.obs_off[G] != nobs)
    throw std::runtime_error("multi: offsets must start at 0 and end at n / nobs");
  for (int g = 0; g < G; ++g)
    if (spec_.lat_off[g + 1] <= spec_.lat_off[g] || spec_.obs_off[g + 1] < spec_.obs_off[g])
      throw std::runtime_error("multi: every model needs latent nodes; offsets must not decrease");
  if ((int64_t)spec_.y.size() != nobs) throw std::runtime_error("multi: y length");
  if ((int64_t)spec_.acp.size() != nobs + 1) throw std::runtime_error("multi: A row pointer length");
  if (spec_.family < 0 || spec_.family > 3) throw std::runtime_error("multi: unknown family");

  std::vector<int> segc(n), sego(std::max<int64_t>(nobs, 1), 0);
  for (int g = 0; g < G; ++g) {
    for (int64_t j = spec_.lat_off[g]; j < spec_.lat_off[g + 1]; ++j) segc[j] = g;
    for (int64_t i = spec_.obs_off[g]; i < spec_.obs_off[g + 1]; ++i) sego[i] = g;
  }
  std::vector<int> pseg(nnz_);
  std::vector<unsigned char> pdiag(nnz_, 0);
  std::vector<int> qri(nnz_);
  for (int64_t c = 0; c < n; ++c) {
    if (!std::is_sorted(spec_.rowidx.begin() + spec_.colptr[c], spec_.rowidx.begin() + spec_.colptr[c + 1]))
      throw std::runtime_error("multi: pattern row indices must be sorted");
    bool diag = false;
    for (int64_t p = spec_.colptr[c]; p < spec_.colptr[c + 1]; ++p) {
      const int64_t r = spec_.rowidx[p];
      if (r < 0 || r >= n || segc[r] != segc[c]) throw std::runtime_error("multi: pattern is not block-diagonal");
      qri[p] = (int)r;
      pseg[p] = segc[c];
      if (r == c) pdiag[p] = 1, diag = true;
    }
    if (!diag) throw std::runtime_error("multi: pattern must contain the diagonal");
  }
  for (int g = 0; g < G; ++g)
    for (int64_t i = spec_.obs_off[g]; i < spec_.obs_off[g + 1]; ++i)
      for (int64_t a = spec_.acp[i]; a < spec_.acp[i + 1]; ++a)
        if (spec_.aci[a] < spec_.lat_off[g] || spec_.aci[a] >= spec_.lat_off[g + 1])
          throw std::runtime_error("multi: observation of model g touches another model's latent nodes");

  // one elimination order per block (blocks ordered concurrently), concatenated
  std::vector<int64_t> perm(n);
  parallel_for(
      G,
      [&](int64_t g0, int64_t g1) {
        for (int64_t g = g0; g < g1; ++g) {
          const int64_t j0 = spec_.lat_off[g], nb = spec_.lat_off[g + 1] - j0;
          std::vector<int64_t> cp(nb + 1, 0), ri;
          ri.reserve(spec_.colptr[j0 + nb] - spec_.colptr[j0]);
          for (int64_t j = 0; j < nb; ++j) {
            for (int64_t p = spec_.colptr[j0 + j]; p < spec_.colptr[j0 + j + 1]; ++p)
              ri.push_back(spec_.rowidx[p] - j0);
            cp[j + 1] = (int64_t)ri.size();
          }
          const std::vector<int64_t> pb = block_order(nb, cp, ri, spec_.ordering);
          for (int64_t k = 0; k < nb; ++k) perm[j0 + k] = pb[k] + j0;
        }
      },
      1);
  Symbolic sym;
  SymbolicOptions opt;
  opt.ordering = ORDER_CUSTOM;
  analyze(n, spec_.colptr.data(), spec_.rowidx.data(), opt, perm.data(), sym);
  // the postordered elimination keeps every model's columns contiguous, models in order
  std::vector<int64_t> poff(G + 1, 0);
  {
    int gcur = 0;
    for (int64_t j = 0; j < n; ++j) {
      const int g = segc[sym.perm[j]];
      if (g < gcur) throw std::runtime_error("multi: elimination order mixes models");
      while (gcur < g) poff[++gcur] = j;
    }
    while (gcur < G) poff[++gcur] = n;
  }
  std::vector<int64_t> eoff(G + 1);
  for (int g = 0; g <= G; ++g) eoff[g] = spec_.colptr[spec_.lat_off[g]];
  F_.reset(new GpuFactor(sym, max_batch, stream_));
  {  // the model of every front, so that converged (theta-set, model) pairs can be skipped
    std::vector<int> fseg(sym.nsuper);
    for (int64_t sn = 0; sn < sym.nsuper; ++sn) fseg[sn] = segc[sym.perm[sym.sn_first[sn]]];
    F_->set_front_groups(fseg);
  }
  active_.alloc((size_t)max_batch * G);

  // observation structures: contributions of A^T diag(w) A on the pattern, A^T, row pairs
  auto find = [&](int64_t row, int64_t col) -> int64_t {
    auto b = spec_.rowidx.begin() + spec_.colptr[col], e = spec_.rowidx.begin() + spec_.colptr[col + 1];
    auto it = std::lower_bound(b, e, row);
    if (it == e || *it != row) return -1;
    return it - spec_.rowidx.begin();
  };
  const auto& acp = spec_.acp;
  std::vector<int> aci(spec_.aci.size());
  for (size_t a = 0; a < aci.size(); ++a) {
    if (spec_.aci[a] < 0 || spec_.aci[a] >= n) throw std::runtime_error("multi: A column out of range");
    aci[a] = (int)spec_.aci[a];
  }
  std::vector<int64_t> opptr(nobs + 1, 0), oppos;
  std::vector<int64_t> cnt(nnz_ + 1, 0);
  for (int64_t i = 0; i < nobs; ++i) {
    const int64_t na = acp[i + 1] - acp[i];
    opptr[i + 1] = opptr[i] + na * na;
  }
  oppos.resize(opptr[nobs]);
  parallel_for(nobs, [&](int64_t i0, int64_t i1) {  // disjoint writes: the pairs of observation i
    for (int64_t i = i0; i < i1; ++i) {
      int64_t q = opptr[i];
      for (int64_t a = acp[i]; a < acp[i + 1]; ++a)
        for (int64_t c = acp[i]; c < acp[i + 1]; ++c, ++q) {
          const int64_t p = find(aci[a], aci[c]);
          if (p < 0) throw std::runtime_error("multi: pattern must contain A^T A");
          oppos[q] = p;
        }
    }
  });
  for (int64_t q = 0; q < opptr[nobs]; ++q) cnt[oppos[q] + 1]++;
  for (int64_t p = 0; p < nnz_; ++p) cnt[p + 1] += cnt[p];
  if (cnt[nnz_] >= (1LL << 31)) throw std::runtime_error("multi: too many observation contributions");
  std::vector<int> cptr(nnz_ + 1), cobs(std::max<int64_t>(cnt[nnz_], 1));
  std::vector<double> cprod(std::max<int64_t>(cnt[nnz_], 1));
  {
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (int64_t i = 0; i < nobs; ++i) {
      int64_t q = opptr[i];
      for (int64_t a = acp[i]; a < acp[i + 1]; ++a)
        for (int64_t c = acp[i]; c < acp[i + 1]; ++c, ++q) {
          const int64_t p = oppos[q];
          cobs[fill[p]] = (int)i;
          cprod[fill[p]++] = spec_.av[a] * spec_.av[c];
        }
    }
    for (int64_t p = 0; p <= nnz_; ++p) cptr[p] = (int)cnt[p];
  }
  std::vector<int64_t> atp(n + 1, 0);
  for (size_t a = 0; a < aci.size(); ++a) atp[aci[a] + 1]++;
  for (int64_t j = 0; j < n; ++j) atp[j + 1] += atp[j];
  std::vector<int> ati(std::max<size_t>(aci.size(), 1));
  std::vector<double> atv(std::max<size_t>(aci.size(), 1));
  {
    std::vector<int64_t> fill(atp.begin(), atp.end() - 1);
    for (int64_t i = 0; i < nobs; ++i)
      for (int64_t a = acp[i]; a < acp[i + 1]; ++a) {
        ati[fill[aci[a]]] = (int)i;
        atv[fill[aci[a]]++] = spec_.av[a];
      }
  }

  comp_.upload(spec_.comp, stream_);
  y_.upload(spec_.y.empty() ? std::vector<double>(1, 0.0) : spec_.y, stream_);
  if (!spec_.p1.empty()) p1_.upload(spec_.p1, stream_);
  if (!spec_.p2.empty()) p2_.upload(spec_.p2, stream_);
  qcp_.upload(spec_.colptr, stream_);
  qri_.upload(qri, stream_);
  pdiag_.upload(pdiag, stream_);
  cptr_.upload(cptr, stream_);
  cobs_.upload(cobs, stream_);
  cprod_.upload(cprod, stream_);
  opptr_.upload(opptr, stream_);
  oppos_.upload(oppos.empty() ? std::vector<int64_t>(1, 0) : oppos, stream_);
  acp_.upload(acp, stream_);
  aci_.upload(aci.empty() ? std::vector<int>(1, 0) : aci, stream_);
  av_.upload(spec_.av.empty() ? std::vector<double>(1, 0.0) : spec_.av, stream_);
  atp_.upload(atp, stream_);
  ati_.upload(ati, stream_);
  atv_.upload(atv, stream_);
  latoff_.upload(spec_.lat_off, stream_);
  obsoff_.upload(spec_.obs_off, stream_);
  poff_.upload(poff, stream_);
  eoff_.upload(eoff, stream_);
  segc_.upload(segc, stream_);
  sego_.upload(sego, stream_);
  pseg_.upload(pseg, stream_);

  const size_t B = max_batch_, BG = B * G, no = std::max<int64_t>(nobs, 1);
  const int T1 = spec_.ncomp + 1;
  coef_.alloc(BG * spec_.ncomp);
  p1s_.alloc(BG);
  x_.alloc(B * n);
  xt_.alloc(B * n);
  step_.alloc(B * n);
  tmp_n_.alloc(B * n);
  var_.alloc(B * n);
  eta_.alloc(B * no);
  logp_.alloc(B * no);
  grad_.alloc(B * no);
  w_.alloc(B * no);
  dw_.alloc(B * no);
  tmp_o_.alloc(B * no);
  sig_.alloc(B * nnz_);
  stats_.alloc(2 * BG);
  alpha_.alloc(BG);
  mdiff_.alloc(BG);
  scal_.alloc(2 * BG);   // loglik, dll
  ld_.alloc(2 * BG);     // prior, posterior log-determinants
  red_.alloc(4 * BG * T1);
  bad_.alloc(BG);
  st_.alloc(2 * BG);
  INLA_CUDA(cudaMemsetAsync(scal_.p, 0, sizeof(double) * 2 * BG, stream_));
  INLA_CUDA(cudaMemsetAsync(red_.p, 0, sizeof(double) * 4 * BG * T1, stream_));
  INLA_CUDA(cudaStreamSynchronize(stream_));
}

MultiLaplace::~MultiLaplace() = default;

void MultiLaplace::eval_lik(int B, const double* d_xsrc) {
  const int64_t nobs = spec_.nobs;
  INLA_CUDA(cudaMemsetAsync(bad_.p, 0, sizeof(int) * B * spec_.G, stream_));
  if (nobs == 0) return;
  k_spmv_a<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(nobs, (int)spec_.n, acp_.p, aci_.p, av_.p, d_xsrc, eta_.p);
  k_meval_lik<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(spec_.family, nobs, spec_.G, sego_.p, eta_.p, y_.p, p1_.p,
                                                         p2_.p, p1s_.p, logp_.p, grad_.p, w_.p, dw_.p, bad_.p);
  launches_ += 2;
}

// prior (Q + 1e-12 I, inference.rs:831-837) or posterior (Q + A^T W A) factorization of
// B theta-sets, then the per-model log-determinants and pivot gates
void MultiLaplace::factor(int B, bool posterior, bool skip) {
  const int G = spec_.G;
  F_->factor_model(spec_.ncomp, comp_.p, coef_.p, posterior ? 0.0 : 1e-12, pdiag_.p, cptr_.p, cobs_.p, cprod_.p,
                   posterior ? w_.p : nullptr, spec_.nobs, B, posterior ? 0 : B, 0.0, pseg_.p, G,
                   posterior && skip ? active_.p : nullptr);
  const size_t o = posterior ? (size_t)max_batch_ * G : 0;
  k_seg_logdet<256><<<dim3(G, B), 256, 0, stream_>>>(F_->dev_sym(), F_->d_front(), F_->front_total(), poff_.p, G,
                                                     ld_.p + o, st_.p + o);
  ++launches_;
}

void MultiLaplace::eval(int B, const double* coef, const double* p1scale, int flags, MultiOut& R) {
  if (B < 1 || B > max_batch_) throw std::runtime_error("multi: batch size out of range");
  const bool dbg = std::getenv("INLA_DEBUG") != nullptr;
  const auto tstart = std::chrono::steady_clock::now();
  std::string trace;  // active (theta-set, model) pairs after every Newton iteration
  const int G = spec_.G, T = spec_.ncomp, T1 = T + 1;
  const int64_t n = spec_.n, nobs = spec_.nobs;
  const size_t BG = (size_t)B * G, MG = (size_t)max_batch_ * G;
  R.mlik.assign(BG, NAN);
  R.ld_prior.assign(BG, NAN);
  R.ld_post.assign(BG, NAN);
  R.loglik.assign(BG, NAN);
  R.quad.assign(BG, NAN);
  R.dll.assign(BG, 0.0);
  R.status.assign(BG, LAP_OK);
  R.iters.assign(BG, 0);
  R.trP.assign(BG * T1, 0.0);
  R.trQ.assign(BG * T1, 0.0);
  R.xMx.assign(BG * T1, 0.0);
  R.zMx.assign(BG * T1, 0.0);
  INLA_CUDA(cudaMemcpyAsync(coef_.p, coef, sizeof(double) * BG * T, cudaMemcpyHostToDevice, stream_));
  std::vector<double> ones(BG, 1.0);
  INLA_CUDA(cudaMemcpyAsync(p1s_.p, p1scale ? p1scale : ones.data(), sizeof(double) * BG, cudaMemcpyHostToDevice,
                            stream_));
  const bool grad = flags & LAP_GRADIENT;
  const bool want_var = (flags & LAP_VARIANCES) || grad;
  double* d_trP = red_.p;
  double* d_trQ = red_.p + BG * T1;
  double* d_xMx = red_.p + 2 * BG * T1;
  double* d_zMx = red_.p + 3 * BG * T1;
  const unsigned GN = grid1(n);

  // ---- prior --------------------------------------------------------------------
  factor(B, false);
  if (grad) {
    F_->selinv(B);
    k_pattern_full<<<dim3(grid1(nnz_), B), 256, 0, stream_>>>(nnz_, F_->d_spos_full(), F_->d_sigma(0),
                                                              F_->front_total(), sig_.p);
    k_seg_trace<256><<<dim3(G, B), 256, 0, stream_>>>(eoff_.p, G, nnz_, T, comp_.p, sig_.p, cptr_.p, cobs_.p,
                                                      cprod_.p, nullptr, nobs, d_trP);
    launches_ += 2;
  }

  // ---- mode ---------------------------------------------------------------------
  INLA_CUDA(cudaMemsetAsync(x_.p, 0, sizeof(double) * B * n, stream_));
  std::vector<double> st(2 * BG), mdiff(BG);
  std::vector<int> bad(BG), pst(BG);
  // Newton systems after the first factorize only the pairs still iterating; a converged pair
  // keeps its last factor (its step is not taken: alpha = 0)
  static const bool no_skip = std::getenv("INLA_NO_PAIR_SKIP") != nullptr;
  bool skip_next = false;
  auto newton_system = [&](const double* d_x) {
    eval_lik(B, d_x);
    factor(B, true, skip_next && !no_skip);
    k_mnewton_rhs<<<dim3(GN, B), 256, 0, stream_>>>((int)n, T, G, segc_.p, qcp_.p, qri_.p, comp_.p, nnz_, coef_.p,
                                                    atp_.p, ati_.p, atv_.p, nobs, grad_.p, d_x, step_.p);
    F_->solve(step_.p, n, B);
    k_seg_max<256><<<dim3(G, B), 256, 0, stream_>>>(latoff_.p, G, n, step_.p, stats_.p);
    launches_ += 2;
  };
  auto fetch = [&]() {
    INLA_CUDA(cudaMemcpyAsync(st.data(), stats_.p, sizeof(double) * 2 * BG, cudaMemcpyDeviceToHost, stream_));
    INLA_CUDA(cudaMemcpyAsync(bad.data(), bad_.p, sizeof(int) * BG, cudaMemcpyDeviceToHost, stream_));
    INLA_CUDA(cudaMemcpyAsync(pst.data(), st_.p + MG, sizeof(int) * BG, cudaMemcpyDeviceToHost, stream_));
    INLA_CUDA(cudaStreamSynchronize(stream_));
  };
  std::vector<double> alpha(BG, 0.0), max_step(BG, 0.0);
  std::vector<char> active(BG, 1);
  if (spec_.family == FAM_GAUSSIAN) {
    // closed form (inference.rs:845-870): one Newton system from x = 0
    newton_system(x_.p);
    INLA_CUDA(cudaMemcpyAsync(x_.p, step_.p, sizeof(double) * B * n, cudaMemcpyDeviceToDevice, stream_));
    fetch();
    for (size_t q = 0; q < BG; ++q) {
      R.iters[q] = 1;
      if (bad[q] & 1) R.status[q] = LAP_BAD_LIKELIHOOD;
      else if (pst[q]) R.status[q] = LAP_SINGULAR_POST;
      else if (st[2 * q + 1] == 0.0) R.status[q] = LAP_NONFINITE_STEP;
    }
  } else {
    for (int it = 0; it < spec_.max_iter; ++it) {
      newton_system(x_.p);
      fetch();
      bool any = false;
      for (size_t q = 0; q < BG; ++q) {
        alpha[q] = 0.0;
        if (!active[q]) continue;
        if (bad[q] & 1) R.status[q] = LAP_BAD_LIKELIHOOD;
        else if (pst[q]) R.status[q] = LAP_SINGULAR_POST;
        else if (st[2 * q + 1] == 0.0) R.status[q] = LAP_NONFINITE_STEP;
        if (R.status[q] != LAP_OK) {
          active[q] = 0;
          continue;
        }
        max_step[q] = st[2 * q];
        alpha[q] = max_step[q] > 10.0 ? 10.0 / max_step[q] : 1.0;
        any = true;
      }
      if (!any) break;
      // backtracking while the trial objective is non-finite (inference.rs:888-914)
      std::vector<char> need(active);
      for (int bt = 0; bt < 12; ++bt) {
        INLA_CUDA(cudaMemcpyAsync(alpha_.p, alpha.data(), sizeof(double) * BG, cudaMemcpyHostToDevice, stream_));
        k_maxpy<<<dim3(GN, B), 256, 0, stream_>>>((int)n, G, segc_.p, x_.p, step_.p, alpha_.p, xt_.p);
        ++launches_;
        eval_lik(B, xt_.p);
        INLA_CUDA(cudaMemcpyAsync(bad.data(), bad_.p, sizeof(int) * BG, cudaMemcpyDeviceToHost, stream_));
        INLA_CUDA(cudaStreamSynchronize(stream_));
        bool again = false;
        for (size_t q = 0; q < BG; ++q) {
          if (!need[q]) continue;
          if (bad[q] == 0) {
            need[q] = 0;
            continue;
          }
          alpha[q] *= 0.5;
          if (alpha[q] < 1e-8) {
            R.status[q] = LAP_NONFINITE_STEP;
            active[q] = 0;
            need[q] = 0;
            alpha[q] = 0.0;
            continue;
          }
          again = true;
        }
        if (!again) break;
      }
      INLA_CUDA(cudaMemcpyAsync(alpha_.p, alpha.data(), sizeof(double) * BG, cudaMemcpyHostToDevice, stream_));
      k_maxpy<<<dim3(GN, B), 256, 0, stream_>>>((int)n, G, segc_.p, x_.p, step_.p, alpha_.p, xt_.p);
      k_seg_maxdiff<256><<<dim3(G, B), 256, 0, stream_>>>(latoff_.p, G, n, xt_.p, x_.p, mdiff_.p);
      launches_ += 2;
      INLA_CUDA(cudaMemcpyAsync(x_.p, xt_.p, sizeof(double) * B * n, cudaMemcpyDeviceToDevice, stream_));
      INLA_CUDA(cudaMemcpyAsync(mdiff.data(), mdiff_.p, sizeof(double) * BG, cudaMemcpyDeviceToHost, stream_));
      INLA_CUDA(cudaStreamSynchronize(stream_));
      bool left = false;
      size_t nleft = 0;
      for (size_t q = 0; q < BG; ++q) {
        if (!active[q]) continue;
        R.iters[q] = it + 1;
        if (mdiff[q] < spec_.tol || max_step[q] < spec_.tol) active[q] = 0;  // converged
        else left = true, ++nleft;
      }
      if (dbg) trace += " " + std::to_string(nleft);
      if (!left) break;
      if (F_->can_skip_groups()) {
        std::vector<unsigned char> act(BG);
        for (size_t q = 0; q < BG; ++q) act[q] = active[q] ? 1 : 0;
        INLA_CUDA(cudaMemcpyAsync(active_.p, act.data(), BG, cudaMemcpyHostToDevice, stream_));
        INLA_CUDA(cudaStreamSynchronize(stream_));  // `act` is released at the end of this block
        skip_next = true;
      }
    }
    for (size_t q = 0; q < BG; ++q)
      if (active[q] && R.status[q] == LAP_OK) R.status[q] = LAP_NONCONVERGED;
    // confirmation refactorization at x* (inference.rs:923-937)
    eval_lik(B, x_.p);
    factor(B, true);
  }

  // ---- marginal likelihood pieces (inference.rs:953-972) ---------------------------
  eval_lik(B, x_.p);
  if (nobs > 0) {
    k_seg_sum<256><<<dim3(G, B), 256, 0, stream_>>>(obsoff_.p, G, nobs, logp_.p, scal_.p);
    ++launches_;
  }
  k_seg_quad<256><<<dim3(G, B), 256, 0, stream_>>>(latoff_.p, G, (int)n, T, qcp_.p, qri_.p, comp_.p, nnz_, coef_.p,
                                                   nullptr, x_.p, d_xMx);
  ++launches_;
  if (spec_.family == FAM_GAUSSIAN && grad && nobs > 0) {
    k_gauss_dll_terms<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(nobs, eta_.p, y_.p, w_.p, tmp_o_.p);
    k_seg_sum<256><<<dim3(G, B), 256, 0, stream_>>>(obsoff_.p, G, nobs, tmp_o_.p, scal_.p + BG);
    launches_ += 2;
  }
  if (want_var) {
    F_->selinv(B);
    F_->extract_diag(var_.p, n, B);
    if (grad) {
      k_pattern_full<<<dim3(grid1(nnz_), B), 256, 0, stream_>>>(nnz_, F_->d_spos_full(), F_->d_sigma(0),
                                                                F_->front_total(), sig_.p);
      k_seg_trace<256><<<dim3(G, B), 256, 0, stream_>>>(eoff_.p, G, nnz_, T, comp_.p, sig_.p, cptr_.p, cobs_.p,
                                                        cprod_.p, w_.p, nobs, d_trQ);
      launches_ += 2;
      if (spec_.family != FAM_GAUSSIAN && nobs > 0) {
        // implicit term: u = A^T (dw .* v), v_i = a_i' Sigma a_i; z = Q_post^-1 u
        k_predictor_var<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(nobs, acp_.p, av_.p, oppos_.p, opptr_.p, sig_.p,
                                                                   nnz_, tmp_o_.p);
        k_mul<<<dim3(grid1(nobs), B), 256, 0, stream_>>>(nobs, tmp_o_.p, dw_.p, tmp_o_.p);
        k_spmv_at<<<dim3(GN, B), 256, 0, stream_>>>((int)n, atp_.p, ati_.p, atv_.p, nobs, tmp_o_.p, tmp_n_.p);
        F_->solve(tmp_n_.p, n, B);
        k_seg_quad<256><<<dim3(G, B), 256, 0, stream_>>>(latoff_.p, G, (int)n, T, qcp_.p, qri_.p, comp_.p, nnz_,
                                                         coef_.p, tmp_n_.p, x_.p, d_zMx);
        launches_ += 4;
      }
    }
  }
  std::vector<double> ld(2 * MG), scal(2 * BG), xmx(BG * T1);
  std::vector<int> stt(2 * MG);
  INLA_CUDA(cudaMemcpyAsync(ld.data(), ld_.p, sizeof(double) * 2 * MG, cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaMemcpyAsync(stt.data(), st_.p, sizeof(int) * 2 * MG, cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaMemcpyAsync(scal.data(), scal_.p, sizeof(double) * 2 * BG, cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaMemcpyAsync(xmx.data(), d_xMx, sizeof(double) * BG * T1, cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaMemcpyAsync(bad.data(), bad_.p, sizeof(int) * BG, cudaMemcpyDeviceToHost, stream_));
  if (grad) {
    INLA_CUDA(cudaMemcpyAsync(R.trP.data(), d_trP, sizeof(double) * BG * T1, cudaMemcpyDeviceToHost, stream_));
    INLA_CUDA(cudaMemcpyAsync(R.trQ.data(), d_trQ, sizeof(double) * BG * T1, cudaMemcpyDeviceToHost, stream_));
    if (spec_.family != FAM_GAUSSIAN)
      INLA_CUDA(cudaMemcpyAsync(R.zMx.data(), d_zMx, sizeof(double) * BG * T1, cudaMemcpyDeviceToHost, stream_));
  }
  INLA_CUDA(cudaStreamSynchronize(stream_));
  INLA_CUDA(cudaGetLastError());
  F_->check_schedule();  // a persistent factorization whose dependency wait ran out is an error
  if (dbg)
    std::fprintf(stderr, "multi eval B=%d G=%d grad=%d var=%d: %.1f ms, active after each Newton iteration:%s\n", B, G,
                 (int)grad, (int)want_var,
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tstart).count(),
                 trace.c_str());
  for (size_t q = 0; q < BG; ++q) {
    if (stt[q]) R.status[q] = LAP_SINGULAR_PRIOR;
    if (R.status[q] == LAP_OK && stt[MG + q]) R.status[q] = LAP_SINGULAR_POST;
    if (R.status[q] == LAP_OK && (bad[q] & 1)) R.status[q] = LAP_BAD_LIKELIHOOD;
    R.ld_prior[q] = ld[q];
    R.ld_post[q] = ld[MG + q];
    R.loglik[q] = nobs > 0 ? scal[q] : 0.0;
    R.dll[q] = grad && spec_.family == FAM_GAUSSIAN ? scal[BG + q] : 0.0;
    R.quad[q] = xmx[q * T1];
    for (int t = 0; t < T; ++t) R.xMx[q * T1 + t] = xmx[q * T1 + 1 + t];
    R.xMx[q * T1 + T] = 0.0;
    R.mlik[q] = R.status[q] == LAP_OK ? R.loglik[q] - 0.5 * R.quad[q] + 0.5 * R.ld_prior[q] - 0.5 * R.ld_post[q]
                                      : NAN;
  }
}

}  // namespace inla
