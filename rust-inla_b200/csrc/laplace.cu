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
#include "host_par.hpp"

namespace inla {

namespace {
inline int cdiv(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }
inline unsigned grid1(int64_t n, int threads = 256, int cap = 2048) {
  return (unsigned)std::max(1, std::min<int>(cdiv(n, threads), cap));
}
// CTAs of a multi-CTA reduction over len elements (at least one).
inline unsigned nchunks(int64_t len, int per_cta) { return (unsigned)std::max(1, cdiv(len, per_cta)); }
}  // namespace

LaplaceEngine::LaplaceEngine(const LaplaceSpec& spec, int max_batch, cudaStream_t stream)
    : spec_(spec), max_batch_(max_batch), stream_(stream) {
  if (spec_.n <= 0 || (int64_t)spec_.colptr.size() != spec_.n + 1) throw std::runtime_error("laplace: invalid pattern");
  n_ = spec_.n;
  const int64_t n0 = spec_.n;
  nnz_ = spec_.colptr[n0];
  if ((int64_t)spec_.rowidx.size() != nnz_) throw std::runtime_error("laplace: rowidx length");
  if (spec_.ncomp < 1 || spec_.ncomp + (spec_.kc > 0 ? 1 : 0) > 8)
    throw std::runtime_error("laplace: 1..8 precision components supported (1..7 with constraints)");
  if ((int64_t)spec_.comp.size() != spec_.ncomp * nnz_) throw std::runtime_error("laplace: component values length");
  const int64_t nobs = spec_.nobs;
  if (spec_.identity_a && nobs != n0) throw std::runtime_error("laplace: identity projector needs nobs == n");
  if ((int64_t)spec_.y.size() != nobs) throw std::runtime_error("laplace: y length");
  if (spec_.family < 0 || spec_.family > 3) throw std::runtime_error("laplace: unknown family");
  for (int64_t c = 0; c < n0; ++c)
    if (!std::is_sorted(spec_.rowidx.begin() + spec_.colptr[c], spec_.rowidx.begin() + spec_.colptr[c + 1]))
      throw std::runtime_error("laplace: pattern row indices must be sorted");
  nuser_ = spec_.ncomp;
  if (spec_.kc < 0) throw std::runtime_error("laplace: negative constraint count");
  if (spec_.kc > 0) augment_constraints();
  const int64_t n = spec_.n;  // n + k when bordered
  nnz_ = spec_.colptr[n];

  const auto t0 = std::chrono::steady_clock::now();
  Symbolic sym;
  SymbolicOptions opt;
  opt.ordering = border_ ? ORDER_CUSTOM : spec_.ordering;
  analyze(n, spec_.colptr.data(), spec_.rowidx.data(), opt, border_ ? border_perm_.data() : nullptr, sym);
  const auto t1 = std::chrono::steady_clock::now();
  // twice the slots: a Gaussian evaluation factorizes prior representatives and
  // posterior problems in one batch
  F_.reset(new GpuFactor(sym, 2 * max_batch, stream_));
  const auto t2 = std::chrono::steady_clock::now();
  if (std::getenv("INLA_DEBUG"))
    std::fprintf(stderr, "laplace setup: symbolic %.1f ms, device factor %.1f ms\n",
                 std::chrono::duration<double, std::milli>(t1 - t0).count(),
                 std::chrono::duration<double, std::milli>(t2 - t1).count());

  const auto t3 = std::chrono::steady_clock::now();
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
      if (spec_.aci[a] < 0 || spec_.aci[a] >= n_) throw std::runtime_error("laplace: A column out of range");
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
  parallel_for(nobs, [&](int64_t i0, int64_t i1) {  // disjoint writes: the pairs of observation i
    for (int64_t i = i0; i < i1; ++i) {
      int64_t q = opptr[i];
      for (int64_t a = acp[i]; a < acp[i + 1]; ++a)
        for (int64_t c = acp[i]; c < acp[i + 1]; ++c, ++q) {
          int64_t p = find(aci[a], aci[c]);
          if (p < 0) throw std::runtime_error("laplace: pattern must contain A^T A");
          oppos[q] = p;
        }
    }
  });
  for (int64_t q = 0; q < opptr[nobs]; ++q) cnt[oppos[q] + 1]++;
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

  const auto t4 = std::chrono::steady_clock::now();
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
  mdiff_.alloc(B);
  if (spec_.kc > 0) cres_.alloc(B * spec_.kc);
  alpha_.alloc(B);
  ldp_.alloc(B);
  bad_.alloc(B);
  stp_.alloc(B);
  INLA_CUDA(cudaStreamSynchronize(stream_));
  if (std::getenv("INLA_DEBUG"))
    std::fprintf(stderr, "laplace setup: observation tables %.1f ms, uploads and buffers %.1f ms\n",
                 std::chrono::duration<double, std::milli>(t4 - t3).count(),
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t4).count());
}

LaplaceEngine::~LaplaceEngine() = default;

// Hard constraints (constraints.rs:16-25, 275-353): C and C^T in CSR, (C C^T)^-1 for the
// projection, then the working prior Q + kappa C^T C in one of two equivalent forms.
void LaplaceEngine::augment_constraints() {
  const int64_t n = spec_.n;
  const int k = spec_.kc;
  if (k > 1024) throw std::runtime_error("laplace: at most 1024 constraint rows");
  if ((int64_t)spec_.cA.size() != (int64_t)k * n) throw std::runtime_error("laplace: constraint matrix length != k*n");
  if ((int64_t)spec_.ce.size() != k) throw std::runtime_error("laplace: constraint right-hand side length != k");
  if (spec_.cmethod < CONSTR_AUTO || spec_.cmethod > CONSTR_BORDERED)
    throw std::runtime_error("laplace: unknown constraint method");
  for (double v : spec_.cA)
    if (!std::isfinite(v)) throw std::runtime_error("laplace: non-finite constraint coefficient");
  for (double v : spec_.ce)
    if (!std::isfinite(v)) throw std::runtime_error("laplace: non-finite constraint right-hand side");
  const double* A = spec_.cA.data();
  std::vector<int64_t> crp(k + 1, 0), ctp(n + 1, 0);
  std::vector<int> cci, cta;
  std::vector<double> cv, ctv;
  int64_t pairs = 0;
  for (int r = 0; r < k; ++r) {
    for (int64_t c = 0; c < n; ++c)
      if (A[(int64_t)r * n + c] != 0.0) {
        cci.push_back((int)c);
        cv.push_back(A[(int64_t)r * n + c]);
        ctp[c + 1]++;
      }
    crp[r + 1] = (int64_t)cci.size();
    if (crp[r + 1] == crp[r]) throw std::runtime_error("laplace: singular C C^T (a constraint row is zero)");
    const int64_t len = crp[r + 1] - crp[r];
    pairs += len * len;
  }
  for (int64_t c = 0; c < n; ++c) ctp[c + 1] += ctp[c];
  cta.resize(cci.size());
  ctv.resize(cci.size());
  {
    std::vector<int64_t> fill(ctp.begin(), ctp.end() - 1);
    for (int r = 0; r < k; ++r)
      for (int64_t p = crp[r]; p < crp[r + 1]; ++p) {
        cta[fill[cci[p]]] = r;
        ctv[fill[cci[p]]++] = cv[p];
      }
  }
  // (C C^T)^-1 by Gauss-Jordan elimination with partial pivoting (solve_dense_symmetric,
  // constraints.rs:355-389, pivot threshold 1e-14); entries summed over columns in order
  std::vector<double> g((size_t)k * k), gi((size_t)k * k, 0.0);
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < k; ++b) {
      double t = 0.0;
      for (int64_t c = 0; c < n; ++c) t += A[(int64_t)a * n + c] * A[(int64_t)b * n + c];
      g[(size_t)a * k + b] = t;
    }
  for (int a = 0; a < k; ++a) gi[(size_t)a * k + a] = 1.0;
  for (int i = 0; i < k; ++i) {
    int piv = i;
    for (int r = i + 1; r < k; ++r)
      if (std::fabs(g[(size_t)r * k + i]) > std::fabs(g[(size_t)piv * k + i])) piv = r;
    if (std::fabs(g[(size_t)piv * k + i]) < 1e-14) throw std::runtime_error("laplace: singular C C^T");
    if (piv != i)
      for (int c = 0; c < k; ++c) {
        std::swap(g[(size_t)i * k + c], g[(size_t)piv * k + c]);
        std::swap(gi[(size_t)i * k + c], gi[(size_t)piv * k + c]);
      }
    const double d = g[(size_t)i * k + i];
    for (int c = 0; c < k; ++c) {
      g[(size_t)i * k + c] /= d;
      gi[(size_t)i * k + c] /= d;
    }
    for (int r = 0; r < k; ++r) {
      if (r == i) continue;
      const double f = g[(size_t)r * k + i];
      if (f == 0.0) continue;
      for (int c = 0; c < k; ++c) {
        g[(size_t)r * k + c] -= f * g[(size_t)i * k + c];
        gi[(size_t)r * k + c] -= f * gi[(size_t)i * k + c];
      }
    }
  }
  crp_.upload(crp, stream_);
  cci_.upload(cci, stream_);
  cv_.upload(cv, stream_);
  ctp_.upload(ctp, stream_);
  cta_.upload(cta, stream_);
  ctv_.upload(ctv, stream_);
  ce_.upload(spec_.ce, stream_);
  cginv_.upload(gi, stream_);
  h_crp_ = std::move(crp);
  h_cci_ = std::move(cci);
  h_cv_ = std::move(cv);
  int method = spec_.cmethod;
  if (method == CONSTR_AUTO) method = pairs <= ((int64_t)1 << 22) ? CONSTR_AUGMENTED : CONSTR_BORDERED;
  if (method == CONSTR_AUGMENTED) {
    if (pairs > ((int64_t)1 << 26))
      throw std::runtime_error("laplace: kappa C^T C would add more than 2^26 pattern entries (the augmented "
                               "method densifies every constrained block; use the bordered method)");
    augment_dense();
  } else {
    augment_bordered();
  }
}

// Q + kappa C^T C on a widened pattern (augment_precision_csc, constraints.rs:275-313):
// entry (i, j) of the appended component is kappa * sum_r C[r][i] C[r][j] with r ascending,
// present wherever some row r has both C[r][i] and C[r][j] nonzero.
void LaplaceEngine::augment_dense() {
  const int64_t n = spec_.n;
  const int k = spec_.kc;
  const auto &crp = h_crp_;
  const auto &cci = h_cci_;
  const auto &cv = h_cv_;
  std::vector<std::vector<int>> rows_of(n);  // constraint rows touching each column
  for (int r = 0; r < k; ++r)
    for (int64_t p = crp[r]; p < crp[r + 1]; ++p) rows_of[cci[p]].push_back(r);
  std::vector<int64_t> ncp(n + 1, 0);
  std::vector<int64_t> nri;
  nri.reserve(spec_.rowidx.size());
  std::vector<int> col;
  for (int64_t j = 0; j < n; ++j) {
    col.assign(spec_.rowidx.begin() + spec_.colptr[j], spec_.rowidx.begin() + spec_.colptr[j + 1]);
    for (int r : rows_of[j]) col.insert(col.end(), cci.begin() + crp[r], cci.begin() + crp[r + 1]);
    std::sort(col.begin(), col.end());
    col.erase(std::unique(col.begin(), col.end()), col.end());
    nri.insert(nri.end(), col.begin(), col.end());
    ncp[j + 1] = (int64_t)nri.size();
  }
  const int64_t nnz_old = spec_.colptr[n], nnz_new = ncp[n];
  const int T0 = spec_.ncomp;
  std::vector<double> comp((size_t)(T0 + 1) * nnz_new, 0.0);
  auto pos = [&](int64_t row, int64_t c) -> int64_t {
    auto b = nri.begin() + ncp[c], e = nri.begin() + ncp[c + 1];
    return std::lower_bound(b, e, row) - nri.begin();
  };
  for (int64_t j = 0; j < n; ++j)
    for (int64_t p = spec_.colptr[j]; p < spec_.colptr[j + 1]; ++p) {
      const int64_t q = pos(spec_.rowidx[p], j);
      for (int t = 0; t < T0; ++t) comp[(size_t)t * nnz_new + q] = spec_.comp[(size_t)t * nnz_old + p];
    }
  double* kap = comp.data() + (size_t)T0 * nnz_new;
  for (int r = 0; r < k; ++r)
    for (int64_t pj = crp[r]; pj < crp[r + 1]; ++pj)
      for (int64_t pi = crp[r]; pi < crp[r + 1]; ++pi) kap[pos(cci[pi], cci[pj])] += cv[pi] * cv[pj];
  for (int64_t p = 0; p < nnz_new; ++p) kap[p] *= kHardConstraintKappa;
  spec_.colptr = std::move(ncp);
  spec_.rowidx = std::move(nri);
  spec_.comp = std::move(comp);
  spec_.ncomp = T0 + 1;
}

// M = [[Q, C^T], [C, -I/kappa]] of order n + k: column j < n gains rows n + r for the
// constraint rows with C[r][j] != 0; border column n + r holds supp(C_r) and the diagonal.
// The appended component carries C and -1/kappa; the caller's components are zero on the
// border. Elimination order: the requested ordering of the caller's pattern with one node per
// constraint row (the latest-eliminated node of its support not yet taken) moved behind the
// border nodes.
void LaplaceEngine::augment_bordered() {
  const int64_t n = spec_.n;
  const int k = spec_.kc;
  const auto &crp = h_crp_;
  const auto &cci = h_cci_;
  const auto &cv = h_cv_;
  if (k > n) throw std::runtime_error("laplace: more constraint rows than latent nodes");
  std::vector<int64_t> perm;
  {
    Symbolic sx;
    SymbolicOptions opt;
    opt.ordering = spec_.ordering;
    analyze(n, spec_.colptr.data(), spec_.rowidx.data(), opt, nullptr, sx);
    perm = sx.perm;
  }
  std::vector<int64_t> ipos(n);
  for (int64_t i = 0; i < n; ++i) ipos[perm[i]] = i;
  std::vector<char> taken(n, 0);
  std::vector<int64_t> last(k);
  for (int r = 0; r < k; ++r) {
    int64_t best = -1;
    for (int64_t p = crp[r]; p < crp[r + 1]; ++p)
      if (!taken[cci[p]] && (best < 0 || ipos[cci[p]] > ipos[best])) best = cci[p];
    if (best < 0) throw std::runtime_error("laplace: constraint rows share their whole support");
    taken[best] = 1;
    last[r] = best;
  }
  border_perm_.clear();
  border_perm_.reserve(n + k);
  for (int64_t i = 0; i < n; ++i)
    if (!taken[perm[i]]) border_perm_.push_back(perm[i]);
  for (int r = 0; r < k; ++r) border_perm_.push_back(n + r);
  for (int r = 0; r < k; ++r) border_perm_.push_back(last[r]);

  std::vector<std::vector<std::pair<int, double>>> rows_of(n);  // (r, C[r][j]) per column
  for (int r = 0; r < k; ++r)
    for (int64_t p = crp[r]; p < crp[r + 1]; ++p) rows_of[cci[p]].push_back({r, cv[p]});
  const int64_t nm = n + k;
  std::vector<int64_t> ncp(nm + 1, 0);
  std::vector<int64_t> nri;
  std::vector<double> bval;  // the border component, aligned with nri
  std::vector<int64_t> oldpos;  // old entry of each new entry (-1: border)
  nri.reserve(spec_.rowidx.size() + 2 * h_cci_.size() + k);
  for (int64_t j = 0; j < n; ++j) {
    for (int64_t p = spec_.colptr[j]; p < spec_.colptr[j + 1]; ++p) {
      nri.push_back(spec_.rowidx[p]);
      bval.push_back(0.0);
      oldpos.push_back(p);
    }
    for (const auto& rv : rows_of[j]) {  // rows n + r > every row of column j, r ascending
      nri.push_back(n + rv.first);
      bval.push_back(rv.second);
      oldpos.push_back(-1);
    }
    ncp[j + 1] = (int64_t)nri.size();
  }
  for (int r = 0; r < k; ++r) {
    for (int64_t p = crp[r]; p < crp[r + 1]; ++p) {
      nri.push_back(cci[p]);
      bval.push_back(cv[p]);
      oldpos.push_back(-1);
    }
    nri.push_back(n + r);
    bval.push_back(-1.0 / kHardConstraintKappa);
    oldpos.push_back(-1);
    ncp[n + r + 1] = (int64_t)nri.size();
  }
  const int64_t nnz_old = spec_.colptr[n], nnz_new = ncp[nm];
  const int T0 = spec_.ncomp;
  std::vector<double> comp((size_t)(T0 + 1) * nnz_new, 0.0);
  for (int64_t q = 0; q < nnz_new; ++q) {
    if (oldpos[q] >= 0)
      for (int t = 0; t < T0; ++t) comp[(size_t)t * nnz_new + q] = spec_.comp[(size_t)t * nnz_old + oldpos[q]];
    comp[(size_t)T0 * nnz_new + q] = bval[q];
  }
  spec_.n = nm;
  spec_.colptr = std::move(ncp);
  spec_.rowidx = std::move(nri);
  spec_.comp = std::move(comp);
  spec_.ncomp = T0 + 1;
  border_ = true;
}

void LaplaceEngine::project(int B, double* d_x, bool final) {
  const int k = spec_.kc;
  if (k == 0) return;
  k_constr_resid<256><<<dim3(k, B), 256, 0, stream_>>>((int)n_, spec_.n, k, crp_.p, cci_.p, cv_.p, ce_.p, 0, 0.0,
                                                       d_x, cres_.p);
  k_constr_apply<<<dim3(grid1(n_, 256, 2 * 148), B), 256, sizeof(double) * k, stream_>>>(
      (int)n_, spec_.n, k, ctp_.p, cta_.p, ctv_.p, cginv_.p, cres_.p, d_x);
  launches_ += 2;
  if (border_) {
    k_constr_resid<256><<<dim3(k, B), 256, 0, stream_>>>((int)n_, spec_.n, k, crp_.p, cci_.p, cv_.p, ce_.p, 1,
                                                         final ? kHardConstraintKappa : 0.0, d_x, cres_.p);
    ++launches_;
  }
}

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
  const int T = spec_.ncomp;  // internal components: the caller's, then kappa C^T C when constrained
  const int T1 = T + 1;
  const int Tu = nuser_;
  std::vector<double> coef_int;
  if (T != Tu) {
    coef_int.resize((size_t)B * T);
    for (int b = 0; b < B; ++b) {
      for (int t = 0; t < Tu; ++t) coef_int[(size_t)b * T + t] = coef[(size_t)b * Tu + t];
      coef_int[(size_t)b * T + Tu] = 1.0;
    }
    coef = coef_int.data();
  }
  // prior log-det jitter: Q + 1e-12 I without constraints, Q + kappa C^T C as is with them
  // (inference.rs:831-840)
  const double jit = spec_.kc > 0 ? 0.0 : 1e-12;
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

  // ---- prior log-determinant: Q + 1e-12 I or Q + kappa C^T C (inference.rs:831-840) ----
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
    F_->factor_model(spec_.ncomp, comp_.p, coefp_.p, jit, pdiag_.p, cptr_.p, cobs_.p, cprod_.p, nullptr,
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
    k_step_stats<256><<<B, 256, 0, stream_>>>((int)n_, n, step_.p, stats_.p);
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
    F_->factor_model(spec_.ncomp, comp_.p, coefall_.p, jit, pdiag_.p, cptr_.p, cobs_.p, cprod_.p, w_.p, spec_.nobs,
                     Bp + B, Bp, 0.0);
    INLA_CUDA(cudaMemcpyAsync(ldp_.p, F_->d_logdet(), sizeof(double) * Bp, cudaMemcpyDeviceToDevice, stream_));
    INLA_CUDA(cudaMemcpyAsync(stp_.p, F_->d_status(), sizeof(int) * Bp, cudaMemcpyDeviceToDevice, stream_));
    k_newton_rhs<<<dim3(grid1(n), B), 256, 0, stream_>>>((int)n, T, qcp_.p, qri_.p, comp_.p, nnz_, coef_.p, atp,
                                                         ati_.p, atv_.p, nobs, grad_.p, x_.p, step_.p);
    F_->solve(step_.p, n, B, post0);
    k_step_stats<256><<<B, 256, 0, stream_>>>((int)n_, n, step_.p, stats_.p);
    launches_ += 2;
    INLA_CUDA(cudaMemcpyAsync(x_.p, step_.p, sizeof(double) * B * n, cudaMemcpyDeviceToDevice, stream_));
    project(B, x_.p, true);  // inference.rs:867-869
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
        project(B, xt_.p);  // inference.rs:902-904
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
      project(B, xt_.p);
      // max |x_trial - x| of the accepted (projected) point (inference.rs:917-922)
      k_max_abs_diff<256><<<B, 256, 0, stream_>>>((int)n_, n, xt_.p, x_.p, mdiff_.p);
      ++launches_;
      INLA_CUDA(cudaMemcpyAsync(x_.p, xt_.p, sizeof(double) * B * n, cudaMemcpyDeviceToDevice, stream_));
      std::vector<double> mdiff(B);
      INLA_CUDA(cudaMemcpyAsync(mdiff.data(), mdiff_.p, sizeof(double) * B, cudaMemcpyDeviceToHost, stream_));
      INLA_CUDA(cudaStreamSynchronize(stream_));
      bool left = false;
      for (int b = 0; b < B; ++b) {
        if (!active[b]) continue;
        R.iters[b] = it + 1;
        const double max_diff = mdiff[b];
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
    project(B, x_.p, true);  // inference.rs:949-951
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
  F_->check_schedule();  // a persistent factorization whose dependency wait ran out is an error
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

  // bordered: log|Q + kappa C^T C| = log|det M| + k log kappa (prior and posterior)
  const double ld_border = border_ ? spec_.kc * std::log(kHardConstraintKappa) : 0.0;
  for (int b = 0; b < B; ++b) {
    ldprior[b] += ld_border;
    ldpost[b] += ld_border;
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
  if (T != Tu) {
    // report the caller's components only: [t < Tu] and the observation term [T] -> [Tu]
    const int Tu1 = Tu + 1;
    for (auto* v : {&R.trP, &R.trQ, &R.xMx, &R.zMx}) {
      std::vector<double> c((size_t)B * Tu1);
      for (int b = 0; b < B; ++b) {
        for (int t = 0; t < Tu; ++t) c[(size_t)b * Tu1 + t] = (*v)[(size_t)b * T1 + t];
        c[(size_t)b * Tu1 + Tu] = (*v)[(size_t)b * T1 + T];
      }
      v->swap(c);
    }
  }
}

}  // namespace inla
