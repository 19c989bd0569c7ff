// scale_model_csc (crates/inla_math/src/design.rs:150-195) without the dense eigendecomposition.
//
// The reference diagonalizes the whole n x n matrix (Jacobi sweeps, O(n^3)) to get diag(R^+).
// Here R^+ comes from one sparse factorization: when the rows of U (k x n) span null(R),
//   M = [[R, U^T], [U, 0]]  has  M^-1 = [[R^+, .], [., .]],
// so the Takahashi selected inverse of M gives diag(R^+) on the GPU. M is indefinite; it is
// factorized without pivoting in an order that eliminates, per row of U, one node of its
// support after the border (the same order the bordered hard-constraint form uses), so every
// pivot before the border belongs to a positive definite block of R.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <utility>
#include <vector>

#include "capi_common.hpp"
#include "inla_b200.h"
#include "symbolic.hpp"

using namespace inla;

namespace {

void check_rc(int rc) {
  if (rc != INLA_OK) throw InlaError(rc, inla_last_error());
}

struct SolverGuard {
  inla_solver* s = nullptr;
  ~SolverGuard() { inla_solver_free(s); }
};

}  // namespace

extern "C" int inla_scale_model(int64_t n, const int64_t* colptr, const int64_t* rowidx, const double* values, int k,
                                const double* null_basis, int ordering, double* fac_out, double* scaled,
                                double* ginv_diag) {
  try {
    if (n <= 0 || !colptr || !rowidx || !values) return fail(INLA_ERR_INVALID, "scale_model: empty Q");
    if (k < -1 || (k > 0 && !null_basis) || ordering < 0 || ordering > INLA_ORDER_ND || ordering == INLA_ORDER_CUSTOM)
      return fail(INLA_ERR_INVALID, "scale_model: invalid argument");
    if (colptr[0] != 0) return fail(INLA_ERR_INVALID, "scale_model: colptr[0] must be 0");
    for (int64_t j = 0; j < n; ++j) {
      if (colptr[j + 1] < colptr[j]) return fail(INLA_ERR_INVALID, "scale_model: colptr not monotone");
      for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p)
        if (rowidx[p] < 0 || rowidx[p] >= n) return fail(INLA_ERR_INVALID, "scale_model: row index out of range");
    }
    const int64_t nnz = colptr[n];
    if (n == 1) {  // singleton component: the reference returns Q = 1 (design.rs:160-163)
      double q = 0.0;
      for (int64_t p = 0; p < nnz; ++p) q += values[p];
      if (scaled)
        for (int64_t p = 0; p < nnz; ++p) scaled[p] = p == 0 ? 1.0 : 0.0;
      if (fac_out) *fac_out = q > 0.0 ? 1.0 / q : NAN;
      if (ginv_diag) ginv_diag[0] = q > 0.0 ? 1.0 / q : 0.0;
      return INLA_OK;
    }

    double qmax = 0.0;
    std::vector<double> rowsum(n, 0.0);
    std::vector<char> active(n, 0);  // nodes with a nonzero entry; the others have ginv diagonal 0
    for (int64_t j = 0; j < n; ++j)
      for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
        const double v = values[p];
        qmax = std::max(qmax, std::fabs(v));
        rowsum[rowidx[p]] += v;
        if (v != 0.0) active[j] = active[rowidx[p]] = 1;
      }
    if (!(qmax > 0.0) || !std::isfinite(qmax)) return fail(INLA_ERR_INVALID, "scale_model: Q has no finite nonzero");

    // null-space basis, dense k x n row-major
    std::vector<double> U;
    int kk = 0;
    if (k == -1) {
      // one constant row per connected component (nonzero values) whose rows all sum to ~0
      std::vector<int64_t> comp(n, -1), stack;
      int64_t ncomp = 0;
      for (int64_t s = 0; s < n; ++s) {
        if (!active[s] || comp[s] >= 0) continue;
        comp[s] = ncomp;
        stack.assign(1, s);
        while (!stack.empty()) {
          const int64_t j = stack.back();
          stack.pop_back();
          for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
            const int64_t i = rowidx[p];
            if (values[p] != 0.0 && comp[i] < 0) {
              comp[i] = ncomp;
              stack.push_back(i);
            }
          }
        }
        ++ncomp;
      }
      std::vector<int64_t> size(ncomp, 0);
      std::vector<char> intrinsic(ncomp, 1);
      for (int64_t i = 0; i < n; ++i)
        if (comp[i] >= 0) {
          ++size[comp[i]];
          if (std::fabs(rowsum[i]) > 1e-10 * qmax) intrinsic[comp[i]] = 0;
        }
      std::vector<int> row_of(ncomp, -1);
      for (int64_t c = 0; c < ncomp; ++c)
        if (intrinsic[c]) row_of[c] = kk++;
      U.assign((size_t)kk * n, 0.0);
      for (int64_t i = 0; i < n; ++i)
        if (comp[i] >= 0 && row_of[comp[i]] >= 0)
          U[(size_t)row_of[comp[i]] * n + i] = 1.0 / std::sqrt((double)size[comp[i]]);
    } else {
      // the caller's rows, restricted to the active nodes (rows left empty are dropped)
      for (int r = 0; r < k; ++r) {
        bool any = false;
        for (int64_t i = 0; i < n; ++i) any |= active[i] && null_basis[(size_t)r * n + i] != 0.0;
        if (!any) continue;
        U.resize((size_t)(kk + 1) * n, 0.0);
        for (int64_t i = 0; i < n; ++i)
          if (active[i]) U[(size_t)kk * n + i] = null_basis[(size_t)r * n + i];
        ++kk;
      }
    }
    // every row must lie in null(R): |R u|_inf <= 1e-8 |R|_max |u|_inf
    for (int r = 0; r < kk; ++r) {
      const double* u = &U[(size_t)r * n];
      std::vector<double> ru(n, 0.0);
      double umax = 0.0;
      for (int64_t j = 0; j < n; ++j) {
        umax = std::max(umax, std::fabs(u[j]));
        for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) ru[rowidx[p]] += values[p] * u[j];
      }
      double rmax = 0.0;
      for (double v : ru) rmax = std::max(rmax, std::fabs(v));
      if (!(rmax <= 1e-8 * qmax * umax))
        return fail(INLA_ERR_INVALID, "scale_model: null-space basis row " + std::to_string(r) +
                                          " is not in the null space of Q");
    }

    // reduced system over the active nodes, bordered by the kk basis rows
    std::vector<int64_t> a(n, -1), act;
    for (int64_t i = 0; i < n; ++i)
      if (active[i]) {
        a[i] = (int64_t)act.size();
        act.push_back(i);
      }
    const int64_t na = (int64_t)act.size(), N = na + kk;
    if (kk > na) return fail(INLA_ERR_INVALID, "scale_model: more null-space rows than nodes");
    std::vector<std::vector<std::pair<int64_t, double>>> cols(N);
    for (int64_t jj = 0; jj < na; ++jj) {
      const int64_t j = act[jj];
      for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p)
        if (a[rowidx[p]] >= 0) cols[jj].push_back({a[rowidx[p]], values[p]});
      for (int r = 0; r < kk; ++r)
        if (U[(size_t)r * n + j] != 0.0) cols[jj].push_back({na + r, U[(size_t)r * n + j]});
    }
    for (int r = 0; r < kk; ++r) {
      for (int64_t jj = 0; jj < na; ++jj)
        if (U[(size_t)r * n + act[jj]] != 0.0) cols[na + r].push_back({jj, U[(size_t)r * n + act[jj]]});
      cols[na + r].push_back({na + r, 0.0});
    }
    std::vector<int64_t> mcp(N + 1, 0), mri;
    std::vector<double> mv;
    for (int64_t j = 0; j < N; ++j) {
      auto& c = cols[j];
      std::sort(c.begin(), c.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
      bool diag = false;
      for (const auto& e : c) diag |= e.first == j;
      if (!diag) c.insert(std::lower_bound(c.begin(), c.end(), std::make_pair(j, 0.0),
                                           [](const auto& x, const auto& y) { return x.first < y.first; }),
                          {j, 0.0});
      for (const auto& e : c) {
        mri.push_back(e.first);
        mv.push_back(e.second);
      }
      mcp[j + 1] = (int64_t)mri.size();
    }

    SolverGuard g;
    if (kk == 0) {
      check_rc(inla_solver_new(ordering, &g.s));
    } else {
      // fill-reducing order of R, then per basis row its latest-eliminated free supported
      // node moved behind the border
      std::vector<int64_t> perm;
      {
        std::vector<int64_t> rcp(na + 1, 0), rri;
        for (int64_t j = 0; j < na; ++j) {
          for (int64_t p = mcp[j]; p < mcp[j + 1]; ++p)
            if (mri[p] < na) rri.push_back(mri[p]);
          rcp[j + 1] = (int64_t)rri.size();
        }
        Symbolic sx;
        SymbolicOptions opt;
        opt.ordering = ordering;
        analyze(na, rcp.data(), rri.data(), opt, nullptr, sx);
        perm = sx.perm;
      }
      std::vector<int64_t> ipos(na);
      for (int64_t i = 0; i < na; ++i) ipos[perm[i]] = i;
      std::vector<char> taken(na, 0);
      std::vector<int64_t> last(kk);
      for (int r = 0; r < kk; ++r) {
        int64_t best = -1;
        for (int64_t jj = 0; jj < na; ++jj)
          if (U[(size_t)r * n + act[jj]] != 0.0 && !taken[jj] && (best < 0 || ipos[jj] > ipos[best])) best = jj;
        if (best < 0) return fail(INLA_ERR_INVALID, "scale_model: null-space rows share their whole support");
        taken[best] = 1;
        last[r] = best;
      }
      std::vector<int64_t> full;
      full.reserve(N);
      for (int64_t i = 0; i < na; ++i)
        if (!taken[perm[i]]) full.push_back(perm[i]);
      for (int r = 0; r < kk; ++r) full.push_back(na + r);
      for (int r = 0; r < kk; ++r) full.push_back(last[r]);
      check_rc(inla_solver_new(INLA_ORDER_AMD, &g.s));
      check_rc(inla_solver_set_perm(g.s, N, full.data()));
    }
    check_rc(inla_solver_factorize(g.s, N, mcp.data(), mri.data(), mv.data()));
    std::vector<double> d(N);
    check_rc(inla_solver_diag_inv(g.s, d.data()));

    // fac = exp(mean(log diag(ginv))) over the positive finite entries (design.rs:171-190)
    double log_sum = 0.0;
    int64_t count = 0;
    for (int64_t i = 0; i < n; ++i) {
      const double vi = a[i] >= 0 ? d[a[i]] : 0.0;
      if (ginv_diag) ginv_diag[i] = vi;
      if (vi > 0.0 && std::isfinite(vi)) {
        log_sum += std::log(vi);
        ++count;
      }
    }
    if (count == 0) return fail(INLA_ERR_INVALID, "scale_model: ginv has no positive diagonal");
    const double fac = std::exp(log_sum / (double)count);
    if (!(fac > 0.0) || !std::isfinite(fac)) return fail(INLA_ERR_INVALID, "scale_model: invalid scale factor");
    if (fac_out) *fac_out = fac;
    if (scaled)
      for (int64_t p = 0; p < nnz; ++p) scaled[p] = values[p] * fac;
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}
