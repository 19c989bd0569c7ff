// Theta-level INLA driver (host) over the batched Laplace engine.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>

#include "aggregate.hpp"
#include "aggregate_dev.hpp"
#include "capi_common.hpp"
#include "driver.hpp"
#include "inla_b200.h"
#include "model_select.hpp"

namespace inla {

// ---------------------------------------------------------------------------
// integration.rs restatements
// ---------------------------------------------------------------------------

// integration.rs:1-62
void ccd_design(int m, double f0, std::vector<double>& pts, std::vector<double>& w) {
  if (m < 1) throw std::runtime_error("CCD requires at least 1 factor");
  pts.assign(m, 0.0);
  for (int i = 0; i < m; ++i) {
    for (double s : {f0, -f0}) {
      std::vector<double> p(m, 0.0);
      p[i] = s;
      pts.insert(pts.end(), p.begin(), p.end());
    }
  }
  if (m >= 2 && m <= 4) {
    const double val = f0 / std::sqrt((double)m);
    for (int k = 0; k < (1 << m); ++k)
      for (int i = 0; i < m; ++i) pts.push_back(((k >> i) & 1 ? 1.0 : -1.0) * val);
  } else if (m == 5) {
    const double val = f0 / std::sqrt(5.0);
    for (int k = 0; k < 16; ++k) {
      double sp = 1.0;
      for (int i = 0; i < 4; ++i) {
        double s = (k >> i) & 1 ? 1.0 : -1.0;
        pts.push_back(s * val);
        sp *= s;
      }
      pts.push_back(sp * val);
    }
  } else if (m > 5) {
    throw std::runtime_error("CCD strategy for m > 5 is not supported");
  }
  const int ne = (int)(pts.size() / m);
  const double wv = ne > 1 ? 1.0 / ((ne - 1) * (1.0 + std::exp(-0.5 * f0 * f0) * (f0 * f0 / m - 1.0))) : 1.0;
  w.assign(ne, wv);
  w[0] = 1.0 - (ne - 1) * wv;
}

// integration.rs:163-230 (Gauss-Jordan with partial pivoting)
bool invert_symmetric_matrix(const std::vector<double>& h, int m, std::vector<double>& inv) {
  const int cols = 2 * m;
  std::vector<double> a(m * cols, 0.0);
  for (int i = 0; i < m; ++i) {
    for (int j = 0; j < m; ++j) a[i * cols + j] = h[i * m + j];
    a[i * cols + m + i] = 1.0;
  }
  for (int i = 0; i < m; ++i) {
    int mr = i;
    for (int r = i + 1; r < m; ++r)
      if (std::fabs(a[r * cols + i]) > std::fabs(a[mr * cols + i])) mr = r;
    if (std::fabs(a[mr * cols + i]) < 1e-14) return false;
    if (mr != i)
      for (int c = 0; c < cols; ++c) std::swap(a[i * cols + c], a[mr * cols + c]);
    const double piv = a[i * cols + i];
    for (int c = 0; c < cols; ++c) a[i * cols + c] /= piv;
    for (int r = 0; r < m; ++r) {
      if (r == i) continue;
      const double f = a[r * cols + i];
      if (f == 0.0) continue;
      for (int c = 0; c < cols; ++c) a[r * cols + c] -= f * a[i * cols + c];
    }
  }
  inv.assign(m * m, 0.0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) inv[i * m + j] = a[i * cols + m + j];
  return true;
}

// Cyclic Jacobi eigen-decomposition of a small symmetric matrix (row-major);
// V[i*m + j] = component i of eigenvector j. The CCD point set is invariant to
// eigenvector signs and to the order of eigenpairs.
void symmetric_eigen(const std::vector<double>& a0, int m, std::vector<double>& lambda, std::vector<double>& V) {
  std::vector<double> a = a0;
  V.assign(m * m, 0.0);
  for (int i = 0; i < m; ++i) V[i * m + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < m; ++i)
      for (int j = i + 1; j < m; ++j) off += a[i * m + j] * a[i * m + j];
    if (off < 1e-30) break;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) {
        const double apq = a[p * m + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (a[q * m + q] - a[p * m + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < m; ++k) {
          const double akp = a[k * m + p], akq = a[k * m + q];
          a[k * m + p] = c * akp - s * akq;
          a[k * m + q] = s * akp + c * akq;
        }
        for (int k = 0; k < m; ++k) {
          const double apk = a[p * m + k], aqk = a[q * m + k];
          a[p * m + k] = c * apk - s * aqk;
          a[q * m + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < m; ++k) {
          const double vkp = V[k * m + p], vkq = V[k * m + q];
          V[k * m + p] = c * vkp - s * vkq;
          V[k * m + q] = s * vkp + c * vkq;
        }
      }
  }
  lambda.resize(m);
  for (int i = 0; i < m; ++i) lambda[i] = a[i * m + i];
}

// ---------------------------------------------------------------------------
// evaluation of f = -(mlik + log prior) (inla_stats/src/hyper_opt.rs:21-47)
// ---------------------------------------------------------------------------

void InlaDriver::check_cancel() const {
  if (cancel_ && cancel_()) throw InlaError(INLA_ERR_CANCELLED, "Operation cancelled by user");
}

void InlaDriver::evaluate(int K, const double* thetas, bool want_grad, bool batched, double* f, double* grad,
                          std::vector<LaplaceOut>* keep) {
  const int T = eng_.ncomp(), m = m_;
  const int Bmax = batched ? eng_.max_batch() : 1;
  std::vector<double> coef, dcoef, p1s, dp1s, gp(m);
  for (int k0 = 0; k0 < K; k0 += Bmax) {
    check_cancel();  // before every evaluation, as evaluate_neg_log_posterior (hyper_opt.rs:21-24)
    const int Bc = std::min(Bmax, K - k0);
    coef.assign((size_t)Bc * T, 0.0);
    dcoef.assign((size_t)Bc * m * T, 0.0);
    p1s.assign(Bc, 1.0);
    dp1s.assign((size_t)Bc * m, 0.0);
    std::vector<char> ok(Bc, 1);
    for (int b = 0; b < Bc; ++b) {
      const double* th = thetas + (size_t)(k0 + b) * m;
      if (map_(th, &coef[(size_t)b * T], &dcoef[(size_t)b * m * T], &p1s[b], &dp1s[(size_t)b * m]) != 0) {
        ok[b] = 0;
        // keep the batch well-formed: reuse a harmless copy of a valid point
        for (int t = 0; t < T; ++t) coef[(size_t)b * T + t] = 1.0;
        p1s[b] = 1.0;
      }
    }
    LaplaceOut R;
    eng_.eval(Bc, coef.data(), p1s.data(), (want_grad ? LAP_GRADIENT : 0) | (keep ? LAP_VARIANCES : 0), R);
    n_evals_ += Bc;
    n_batches_ += 1;
    for (int b = 0; b < Bc; ++b) {
      const int k = k0 + b;
      const double* th = thetas + (size_t)k * m;
      const bool good = ok[b] && R.status[b] == LAP_OK && std::isfinite(R.mlik[b]);
      if (!good) {
        f[k] = 1e12;  // hyper_opt.rs:39-45: keep the search alive on a failed Laplace
        if (grad)
          for (int i = 0; i < m; ++i) grad[(size_t)k * m + i] = 0.0;
        continue;
      }
      const double lp = prior_(th, want_grad ? gp.data() : nullptr);
      f[k] = -(R.mlik[b] + lp);
      if (want_grad && grad) {
        const int T1 = T + 1;
        for (int i = 0; i < m; ++i) {
          double d = 0.0;
          for (int t = 0; t < T; ++t) {
            const double dc = dcoef[(size_t)b * m * T + (size_t)i * T + t];
            if (dc == 0.0) continue;
            d += dc * (0.5 * R.trP[(size_t)b * T1 + t] - 0.5 * R.trQ[(size_t)b * T1 + t] -
                       0.5 * R.xMx[(size_t)b * T1 + t] + 0.5 * R.zMx[(size_t)b * T1 + t]);
          }
          const double ds = dp1s[(size_t)b * m + i];
          if (ds != 0.0) d += ds / p1s[b] * (R.dll[b] - 0.5 * R.trQ[(size_t)b * T1 + T]);
          grad[(size_t)k * m + i] = -(d + gp[i]);
        }
      }
    }
    if (keep) keep->push_back(std::move(R));
  }
}

// ---------------------------------------------------------------------------
// Nelder-Mead (inla_math/src/hyper_opt.rs:15-183)
// ---------------------------------------------------------------------------

void InlaDriver::nelder_mead(std::vector<double>& x0, const FitOptions& opt, int& iters) {
  const int m = m_;
  const bool batched = opt.batched != 0;
  std::vector<std::vector<double>> v(m + 1, x0);
  std::vector<double> fv(m + 1);
  {
    std::vector<double> pts((size_t)(m + 1) * m);
    for (int i = 0; i <= m; ++i) {
      if (i > 0) v[i][i - 1] += opt.nm_step;
      std::copy(v[i].begin(), v[i].end(), pts.begin() + (size_t)i * m);
    }
    evaluate(m + 1, pts.data(), false, batched, fv.data(), nullptr);
  }
  auto f1 = [&](const std::vector<double>& t) {
    double r;
    evaluate(1, t.data(), false, false, &r, nullptr);
    return r;
  };
  iters = 0;
  for (int it = 0; it < opt.max_iter; ++it) {
    iters = it + 1;
    std::vector<int> idx(m + 1);
    for (int i = 0; i <= m; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return fv[a] < fv[b]; });
    std::vector<std::vector<double>> sv(m + 1);
    std::vector<double> sf(m + 1);
    for (int i = 0; i <= m; ++i) {
      sv[i] = v[idx[i]];
      sf[i] = fv[idx[i]];
    }
    v.swap(sv);
    fv.swap(sf);
    double mean = 0.0;
    for (double x : fv) mean += x;
    mean /= (m + 1);
    double var = 0.0;
    for (double x : fv) var += (x - mean) * (x - mean);
    var /= (m + 1);
    if (std::sqrt(var) < opt.tol) break;
    std::vector<double> cen(m, 0.0), refl(m);
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) cen[j] += v[i][j];
    for (int j = 0; j < m; ++j) cen[j] /= m;
    for (int j = 0; j < m; ++j) refl[j] = cen[j] + 1.0 * (cen[j] - v[m][j]);
    const double fr = f1(refl);
    if (fv[0] <= fr && fr < fv[m - 1]) {
      v[m] = refl;
      fv[m] = fr;
      continue;
    }
    if (fr < fv[0]) {
      std::vector<double> ex(m);
      for (int j = 0; j < m; ++j) ex[j] = cen[j] + 2.0 * (refl[j] - cen[j]);
      const double fe = f1(ex);
      if (fe < fr) {
        v[m] = ex;
        fv[m] = fe;
      } else {
        v[m] = refl;
        fv[m] = fr;
      }
      continue;
    }
    bool contract = false;
    std::vector<double> con(m);
    if (fr < fv[m]) {
      for (int j = 0; j < m; ++j) con[j] = cen[j] + 0.5 * (refl[j] - cen[j]);
      const double fc = f1(con);
      if (fc < fr) {
        v[m] = con;
        fv[m] = fc;
        contract = true;
      }
    } else {
      for (int j = 0; j < m; ++j) con[j] = cen[j] + 0.5 * (v[m][j] - cen[j]);
      const double fc = f1(con);
      if (fc < fv[m]) {
        v[m] = con;
        fv[m] = fc;
        contract = true;
      }
    }
    if (contract) continue;
    std::vector<double> pts((size_t)m * m);
    for (int i = 1; i <= m; ++i) {
      for (int j = 0; j < m; ++j) v[i][j] = v[0][j] + 0.5 * (v[i][j] - v[0][j]);
      std::copy(v[i].begin(), v[i].end(), pts.begin() + (size_t)(i - 1) * m);
    }
    evaluate(m, pts.data(), false, batched, fv.data() + 1, nullptr);
  }
  x0 = v[0];
}

// ---------------------------------------------------------------------------
// BFGS on exact adjoint gradients with a batched multi-step line search
// ---------------------------------------------------------------------------

void InlaDriver::bfgs(std::vector<double>& x, const FitOptions& opt, int& iters) {
  const int m = m_;
  const bool batched = opt.batched != 0;
  double f;
  std::vector<double> g(m), Hinv(m * m, 0.0);
  evaluate(1, x.data(), true, batched, &f, g.data());
  for (int i = 0; i < m; ++i) Hinv[i * m + i] = 1.0;
  bool scaled = false;
  static const double kAlphas[] = {1.0, 0.5, 0.25, 0.1, 0.03, 0.01};
  const int na = batched ? 6 : 1;
  iters = 0;
  for (int it = 0; it < opt.max_iter; ++it) {
    iters = it + 1;
    double gmax = 0.0;
    for (double gi : g) gmax = std::max(gmax, std::fabs(gi));
    if (gmax < opt.tol) break;
    std::vector<double> p(m, 0.0);
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) p[i] -= Hinv[i * m + j] * g[j];
    double slope = 0.0, pmax = 0.0;
    for (int i = 0; i < m; ++i) {
      slope += p[i] * g[i];
      pmax = std::max(pmax, std::fabs(p[i]));
    }
    if (slope >= 0.0) {  // not a descent direction: restart from steepest descent
      for (int i = 0; i < m * m; ++i) Hinv[i] = (i % (m + 1) == 0) ? 1.0 : 0.0;
      for (int i = 0; i < m; ++i) p[i] = -g[i];
      slope = 0.0;
      pmax = 0.0;
      for (int i = 0; i < m; ++i) {
        slope += p[i] * g[i];
        pmax = std::max(pmax, std::fabs(p[i]));
      }
    }
    const double cap = 1.0;  // theta lives on log scales: at most one unit per step
    const double base = pmax > cap ? cap / pmax : 1.0;
    bool accepted = false;
    double fa = 0.0, amax = 0.0;
    std::vector<double> xa(m), ga(m);
    double scale = base;
    for (int round = 0; round < 6 && !accepted; ++round) {
      const int K = batched ? na : 1;
      std::vector<double> pts((size_t)K * m), fk(K), gk((size_t)K * m);
      std::vector<double> al(K);
      for (int k = 0; k < K; ++k) {
        al[k] = scale * (batched ? kAlphas[k] : 1.0);
        for (int i = 0; i < m; ++i) pts[(size_t)k * m + i] = x[i] + al[k] * p[i];
      }
      evaluate(K, pts.data(), true, batched, fk.data(), gk.data());
      // best Armijo point among the candidates
      int best = -1;
      for (int k = 0; k < K; ++k) {
        if (!(fk[k] < 1e11)) continue;
        if (fk[k] <= f + 1e-4 * al[k] * slope && (best < 0 || fk[k] < fk[best])) best = k;
      }
      if (best >= 0) {
        accepted = true;
        fa = fk[best];
        amax = al[best];
        for (int i = 0; i < m; ++i) {
          xa[i] = pts[(size_t)best * m + i];
          ga[i] = gk[(size_t)best * m + i];
        }
      } else {
        scale *= batched ? 0.003 : 0.5;
      }
    }
    if (!accepted) break;
    std::vector<double> s(m), y(m);
    double sy = 0.0, yy = 0.0;
    for (int i = 0; i < m; ++i) {
      s[i] = xa[i] - x[i];
      y[i] = ga[i] - g[i];
      sy += s[i] * y[i];
      yy += y[i] * y[i];
    }
    const double fprev = f;
    x = xa;
    f = fa;
    g = ga;
    (void)amax;
    if (sy > 1e-12 * std::sqrt(yy) * 1.0) {
      if (!scaled) {
        const double gam = sy / yy;
        for (int i = 0; i < m * m; ++i) Hinv[i] = (i % (m + 1) == 0) ? gam : 0.0;
        scaled = true;
      }
      // Hinv <- (I - rho s y') Hinv (I - rho y s') + rho s s'
      const double rho = 1.0 / sy;
      std::vector<double> Hy(m, 0.0);
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) Hy[i] += Hinv[i * m + j] * y[j];
      double yHy = 0.0;
      for (int i = 0; i < m; ++i) yHy += y[i] * Hy[i];
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j)
          Hinv[i * m + j] += rho * ((1.0 + rho * yHy) * s[i] * s[j] - Hy[i] * s[j] - s[i] * Hy[j]);
    }
    if (std::fabs(fprev - f) < 1e-12 * (1.0 + std::fabs(f))) break;
  }
}

// ---------------------------------------------------------------------------
// Batched Newton: every iteration evaluates the line-search candidates
// x + a p (a = 1, 1/2, 1/4) together with their +-h stencils in one batch, so
// the accepted point comes with its exact adjoint gradient and a central-FD
// Hessian of that gradient.
// ---------------------------------------------------------------------------

void InlaDriver::eval_stencils(const std::vector<std::vector<double>>& centers, double h, std::vector<double>& f,
                               std::vector<double>& g, std::vector<double>& H, bool one_sided) {
  const int m = m_, C = (int)centers.size(), per = one_sided ? 1 + m : 1 + 2 * m;
  std::vector<double> pts;
  pts.reserve((size_t)C * per * m);
  for (const auto& c : centers) {
    pts.insert(pts.end(), c.begin(), c.end());
    for (int i = 0; i < m; ++i)
      for (double s : {1.0, -1.0}) {
        if (one_sided && s < 0) continue;
        std::vector<double> t(c);
        t[i] += s * h;
        pts.insert(pts.end(), t.begin(), t.end());
      }
  }
  const int K = C * per;
  std::vector<double> fk(K), gk((size_t)K * m);
  evaluate(K, pts.data(), true, true, fk.data(), gk.data());
  f.assign(C, 0.0);
  g.assign((size_t)C * m, 0.0);
  H.assign((size_t)C * m * m, 0.0);
  for (int c = 0; c < C; ++c) {
    const int b0 = c * per;
    f[c] = fk[b0];
    bool bad = !(fk[b0] < 1e11);
    for (int i = 0; i < m; ++i) g[(size_t)c * m + i] = gk[(size_t)b0 * m + i];
    for (int i = 0; i < m; ++i) {
      // central differences of the gradient, or forward differences from the centre
      const int kp = one_sided ? b0 + 1 + i : b0 + 1 + 2 * i, km = one_sided ? b0 : kp + 1;
      const double den = one_sided ? h : 2.0 * h;
      if (!(fk[kp] < 1e11) || !(fk[km] < 1e11)) bad = true;
      for (int j = 0; j < m; ++j)
        H[(size_t)c * m * m + i * m + j] = (gk[(size_t)kp * m + j] - gk[(size_t)km * m + j]) / den;
    }
    double* Hc = &H[(size_t)c * m * m];
    for (int i = 0; i < m; ++i)
      for (int j = i + 1; j < m; ++j) Hc[i * m + j] = Hc[j * m + i] = 0.5 * (Hc[i * m + j] + Hc[j * m + i]);
    if (bad) f[c] = 1e12;
  }
}

void InlaDriver::newton(std::vector<double>& x, const FitOptions& opt, int& iters) {
  const int m = m_;
  const double h = 1e-3;
  const bool one_sided = opt.mode_search == 3;  // m + 1 stencil points per candidate instead of 2m + 1
  std::vector<double> f1, g, H;
  eval_stencils({x}, h, f1, g, H, one_sided);
  double f = f1[0];
  double delta = 2.0;  // trust bound on max |step| (theta lives on log scales: a factor e^2 per step)
  iters = 0;
  for (int it = 0; it < opt.max_iter; ++it) {
    iters = it + 1;
    double gmax = 0.0;
    for (double gi : g) gmax = std::max(gmax, std::fabs(gi));
    if (gmax < opt.tol) break;
    // Newton direction on the |eigenvalue|-modified Hessian
    std::vector<double> lam, V;
    symmetric_eigen(H, m, lam, V);
    double lmax = 0.0;
    for (double l : lam) lmax = std::max(lmax, std::fabs(l));
    std::vector<double> p(m, 0.0);
    for (int j = 0; j < m; ++j) {
      const double l = std::max(std::fabs(lam[j]), 1e-8 * std::max(lmax, 1e-300));
      double vg = 0.0;
      for (int i = 0; i < m; ++i) vg += V[i * m + j] * g[i];
      for (int i = 0; i < m; ++i) p[i] -= V[i * m + j] * vg / l;
    }
    double pmax = 0.0, slope = 0.0;
    for (int i = 0; i < m; ++i) {
      pmax = std::max(pmax, std::fabs(p[i]));
      slope += p[i] * g[i];
    }
    const bool capped = pmax > delta;
    if (capped) {
      for (double& v : p) v *= delta / pmax;
      slope *= delta / pmax;
    }
    // Backtracking on alpha = 1, 1/2, 1/4: each candidate is one batch (its point
    // and the 2m gradient-stencil points for the next Hessian); shorter steps
    // are evaluated only when the longer one fails the sufficient-decrease test.
    static const double kA[3] = {1.0, 0.5, 0.25};
    std::vector<double> fc, gc, Hc, xc;
    int best = -1;
    for (int k = 0; k < 3 && best < 0; ++k) {
      xc = x;
      for (int i = 0; i < m; ++i) xc[i] += kA[k] * p[i];
      eval_stencils({xc}, h, fc, gc, Hc, one_sided);
      if (fc[0] < 1e11 && fc[0] <= f + 1e-4 * kA[k] * slope) best = k;
    }
    if (best < 0) {
      delta *= 0.25;
      if (delta < 1e-8) break;
      continue;
    }
    const double fprev = f;
    x = xc;
    f = fc[0];
    g.assign(gc.begin(), gc.begin() + m);
    H.assign(Hc.begin(), Hc.begin() + (size_t)m * m);
    if (std::getenv("INLA_DEBUG"))
      std::fprintf(stderr, "newton it=%d f=%.10g |g|=%.3g delta=%.3g alpha=%.3g capped=%d\n", it, f, gmax, delta,
                   kA[best], (int)capped);
    // trust radius from the agreement of the decrease with the quadratic model's prediction
    // (the ratio test of Nocedal & Wright, Numerical Optimization, 2nd ed., Alg. 4.1): grow it
    // twofold after a capped full step with ratio > 3/4, shrink it to a quarter of the step
    // taken when the ratio is below 1/4; along the |eigenvalue|-modified Newton direction the
    // predicted decrease of the step a * p (p capped by the factor sc) is -a slope (1 - a sc / 2)
    const double sc = capped ? delta / pmax : 1.0, a = kA[best];
    const double pred = -a * slope * (1.0 - 0.5 * a * sc), rho = pred > 0 ? (fprev - f) / pred : 0.0;
    if (rho > 0.75 && capped && best == 0) delta = std::min(2.0 * delta, 8.0);
    else if (rho < 0.25) delta = std::max(0.25, 0.25 * a * std::min(pmax, delta));
    else if (best > 0) delta = std::max(0.25, a * std::min(pmax, delta));
    if (std::fabs(fprev - f) < 1e-12 * (1.0 + std::fabs(f))) break;
  }
}

// ---------------------------------------------------------------------------
// Hessians
// ---------------------------------------------------------------------------

// inla_math/src/hyper_opt.rs:197-259: Hessian of g = -f, all stencil points in one batch.
void InlaDriver::fd_hessian(const std::vector<double>& mode, double h, bool batched, std::vector<double>& H) {
  const int m = m_;
  std::vector<double> pts(mode);
  auto add = [&](int i, double si, int j, double sj) {
    std::vector<double> t(mode);
    t[i] += si * h;
    if (j >= 0) t[j] += sj * h;
    pts.insert(pts.end(), t.begin(), t.end());
  };
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      if (i == j) {
        add(i, 1, -1, 0);
        add(i, -1, -1, 0);
      } else if (i < j) {
        add(i, 1, j, 1);
        add(i, 1, j, -1);
        add(i, -1, j, 1);
        add(i, -1, j, -1);
      }
    }
  const int K = (int)(pts.size() / m);
  std::vector<double> f(K);
  evaluate(K, pts.data(), false, batched, f.data(), nullptr);
  auto g = [&](int k) { return -f[k]; };
  H.assign(m * m, 0.0);
  int k = 1;
  const double g0 = g(0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) {
      if (i == j) {
        H[i * m + i] = (g(k) - 2.0 * g0 + g(k + 1)) / (h * h);
        k += 2;
      } else if (i < j) {
        const double v = (g(k) - g(k + 1) - g(k + 2) + g(k + 3)) / (4.0 * h * h);
        H[i * m + j] = H[j * m + i] = v;
        k += 4;
      }
    }
}

// Central differences of the adjoint gradient (2m points, one batch).
void InlaDriver::grad_hessian(const std::vector<double>& mode, double h, bool batched, std::vector<double>& H) {
  const int m = m_;
  std::vector<double> pts;
  for (int i = 0; i < m; ++i)
    for (double s : {1.0, -1.0}) {
      std::vector<double> t(mode);
      t[i] += s * h;
      pts.insert(pts.end(), t.begin(), t.end());
    }
  std::vector<double> f(2 * m), g((size_t)2 * m * m);
  evaluate(2 * m, pts.data(), true, batched, f.data(), g.data());
  H.assign(m * m, 0.0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j)
      H[i * m + j] = -(g[(size_t)(2 * i) * m + j] - g[(size_t)(2 * i + 1) * m + j]) / (2.0 * h);
  for (int i = 0; i < m; ++i)
    for (int j = i + 1; j < m; ++j) H[i * m + j] = H[j * m + i] = 0.5 * (H[i * m + j] + H[j * m + i]);
}

// ---------------------------------------------------------------------------
// fit without hyperparameters (inference.rs:1135-1239): one Laplace node
// ---------------------------------------------------------------------------

void InlaDriver::fit_single_node(FitResult& out) {
  const int64_t n = eng_.n();
  const int T = eng_.ncomp();
  check_cancel();
  std::vector<double> coef(T, 0.0), p1s(1, 1.0), dp1s(1, 0.0), dcoef(1, 0.0);
  if (map_(nullptr, coef.data(), dcoef.data(), &p1s[0], dp1s.data()) != 0)
    throw std::runtime_error("theta map failed at the empty theta");
  LaplaceOut R;
  eng_.eval(1, coef.data(), p1s.data(), LAP_VARIANCES, R);
  n_evals_ += 1;
  n_batches_ += 1;
  // find_latent_mode_a_with_solver(...)? : a failed mode search is the fit's error
  if (R.status[0] != LAP_OK || !std::isfinite(R.mlik[0]))
    throw InlaError((R.status[0] == LAP_SINGULAR_PRIOR || R.status[0] == LAP_SINGULAR_POST) ? INLA_ERR_SINGULAR : INLA_ERR_NONCONVERGED,
                    "Laplace mode search failed at the single node");
  std::vector<double> means(n), vars(n);
  const size_t w = sizeof(double) * n;
  INLA_CUDA(cudaMemcpyAsync(means.data(), eng_.d_x(), w, cudaMemcpyDeviceToHost, eng_.stream()));
  INLA_CUDA(cudaMemcpyAsync(vars.data(), eng_.d_var(), w, cudaMemcpyDeviceToHost, eng_.stream()));
  INLA_CUDA(cudaStreamSynchronize(eng_.stream()));
  out.mode.clear();
  out.hessian.clear();
  out.mode_iters = 0;
  out.latent_mean = means;
  out.latent_var = vars;
  const LaplaceSpec& S = eng_.spec();
  const int64_t nobs = S.identity_a ? n : S.nobs;
  out.cond_eta.resize(nobs);
  out.cond_eta_var.resize(nobs);
  {  // eta = A x* and its diagonal variance on the device (inference.rs:1142-1151)
    DBuf<double> eta_local, etav_local;
    DBuf<double>& d_eta = out.d_cond_eta ? *out.d_cond_eta : eta_local;
    DBuf<double>& d_etav = out.d_cond_eta_var ? *out.d_cond_eta_var : etav_local;
    d_eta.alloc(nobs);
    d_etav.alloc(nobs);
    DevCsrA A;
    A.rp = eng_.d_acp();
    A.ci = eng_.d_aci();
    A.v = eng_.d_av();
    dev_project_nodes(eng_.stream(), nobs, A, 1, eng_.d_x(), eng_.xstride(), eng_.d_var(), eng_.xstride(), d_eta.p,
                      d_etav.p);
    INLA_CUDA(cudaMemcpyAsync(out.cond_eta.data(), d_eta.p, sizeof(double) * nobs, cudaMemcpyDeviceToHost,
                              eng_.stream()));
    INLA_CUDA(cudaMemcpyAsync(out.cond_eta_var.data(), d_etav.p, sizeof(double) * nobs, cudaMemcpyDeviceToHost,
                              eng_.stream()));
    INLA_CUDA(cudaStreamSynchronize(eng_.stream()));
  }
  out.pred_mean = out.cond_eta;
  out.pred_var = out.cond_eta_var;
  out.mode_index = 0;
  out.p1scale_mode = p1s[0];
  out.coef_mode = coef;
  out.mlik = R.mlik[0];
  out.mlik_gaussian = R.mlik[0];  // marginal_log_lik_gaussian = marginal_log_lik (inference.rs:1224)
  out.cond_mean = std::move(means);
  out.cond_var = std::move(vars);
  out.node_theta.clear();
  out.node_weight = {1.0};  // single-node weight for the predictor / model selection / marginals
  out.node_logpost = {R.mlik[0]};
  out.n_evals = n_evals_;
  out.n_batches = n_batches_;
}

// ---------------------------------------------------------------------------
// fit (inference.rs:1116-1466)
// ---------------------------------------------------------------------------

void InlaDriver::fit(const double* theta0, const FitOptions& opt, FitResult& out) {
  auto t0 = std::chrono::steady_clock::now();
  const int m = m_;
  const int64_t n = eng_.n();
  n_evals_ = n_batches_ = 0;
  cancel_ = opt.cancel;
  if (m == 0) {
    fit_single_node(out);
    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return;
  }
  auto since = [](std::chrono::steady_clock::time_point a) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
  };
  std::vector<double> mode(theta0, theta0 + m);
  int iters = 0;
  if (opt.mode_search == 0) nelder_mead(mode, opt, iters);
  else if (opt.mode_search == 1) bfgs(mode, opt, iters);
  else newton(mode, opt, iters);  // 2: central gradient stencil, 3: forward stencil
  out.mode = mode;
  out.mode_iters = iters;
  out.phase_s[0] = since(t0);
  const auto t1 = std::chrono::steady_clock::now();

  double hh = 1e-4;  // inference.rs:1264
  for (double t : mode) hh = std::max(hh, 0.05 * std::fabs(t));
  if (opt.hessian == 0) fd_hessian(mode, hh, opt.batched != 0, out.hessian);
  else grad_hessian(mode, hh, opt.batched != 0, out.hessian);
  out.phase_s[1] = since(t1);
  const auto t2 = std::chrono::steady_clock::now();

  std::vector<double> neg(m * m), sigma;
  for (int i = 0; i < m * m; ++i) neg[i] = -out.hessian[i];
  if (!invert_symmetric_matrix(neg, m, sigma)) throw std::runtime_error("Singular Hessian matrix");
  std::vector<double> lam, V;
  symmetric_eigen(sigma, m, lam, V);

  std::vector<double> z, zw;
  if (opt.strategy == 1 && m <= 2) {
    // grid_design (integration.rs:64-156): expand until log-density drops by > 4
    auto theta_of = [&](const std::vector<double>& zz) {
      std::vector<double> th(mode);
      for (int i = 0; i < m; ++i) {
        double d = 0.0;
        for (int j = 0; j < m; ++j) d += V[i * m + j] * std::sqrt(std::fabs(lam[j])) * zz[j];
        th[i] += d;
      }
      return th;
    };
    auto logpost = [&](const std::vector<double>& zz) {
      std::vector<double> th = theta_of(zz);
      double fv;
      evaluate(1, th.data(), false, false, &fv, nullptr);
      return fv >= 1e12 ? -std::numeric_limits<double>::infinity() : -fv;
    };
    const double step = opt.f0, thr = 4.0;
    std::vector<double> c0(m, 0.0);
    const double g0 = logpost(c0);
    if (m == 1) {
      z = {0.0};
      for (int dir : {1, -1})
        for (int k = 1;; ++k) {
          std::vector<double> zz = {dir * k * step};
          if (g0 - logpost(zz) > thr) break;
          z.push_back(zz[0]);
        }
    } else {
      int lim[4] = {0, 0, 0, 0};
      const int ax[4] = {0, 0, 1, 1};
      const int sg[4] = {1, -1, 1, -1};
      for (int d = 0; d < 4; ++d)
        for (;;) {
          std::vector<double> zz(2, 0.0);
          zz[ax[d]] = sg[d] * (lim[d] + 1) * step;
          if (g0 - logpost(zz) > thr) break;
          ++lim[d];
        }
      for (int i = -lim[1]; i <= lim[0]; ++i)
        for (int j = -lim[3]; j <= lim[2]; ++j) {
          std::vector<double> zz = {i * step, j * step};
          if (g0 - logpost(zz) <= thr) z.insert(z.end(), zz.begin(), zz.end());
        }
    }
    zw.assign(z.size() / m, 1.0);
  } else {
    ccd_design(m, opt.strategy == 1 ? 2.5 : opt.f0, z, zw);
  }
  const int K = (int)zw.size();
  std::vector<double> thetas((size_t)K * m);
  for (int k = 0; k < K; ++k)
    for (int i = 0; i < m; ++i) {
      double d = 0.0;
      for (int j = 0; j < m; ++j) d += V[i * m + j] * std::sqrt(std::fabs(lam[j])) * z[(size_t)k * m + j];
      thetas[(size_t)k * m + i] = mode[i] + d;
    }

  // node evaluations (inference.rs:1306-1397): x*, Takahashi variances, log posterior. The
  // node results stay on the device for the aggregation below; the host keeps a copy for the
  // marginals of the fit.
  std::vector<double> lp(K), means((size_t)K * n), vars((size_t)K * n);
  DBuf<double> d_means, d_vars;
  d_means.alloc((size_t)K * n);
  d_vars.alloc((size_t)K * n);
  {
    const int Bmax = opt.batched ? eng_.max_batch() : 1;
    std::vector<double> fk(K);
    for (int k0 = 0; k0 < K; k0 += Bmax) {
      const int Bc = std::min(Bmax, K - k0);
      std::vector<LaplaceOut> keep;
      evaluate(Bc, thetas.data() + (size_t)k0 * m, false, true, fk.data() + k0, nullptr, &keep);
      const LaplaceOut& R = keep.back();
      const size_t w = sizeof(double) * n, pitch = sizeof(double) * eng_.xstride();
      INLA_CUDA(cudaMemcpy2DAsync(d_means.p + (size_t)k0 * n, w, eng_.d_x(), pitch, w, Bc, cudaMemcpyDeviceToDevice,
                                  eng_.stream()));
      INLA_CUDA(cudaMemcpy2DAsync(d_vars.p + (size_t)k0 * n, w, eng_.d_var(), pitch, w, Bc, cudaMemcpyDeviceToDevice,
                                  eng_.stream()));
      for (int b = 0; b < Bc; ++b) {
        const int k = k0 + b;
        if (R.status[b] != LAP_OK || fk[k] >= 1e12) {
          lp[k] = -std::numeric_limits<double>::infinity();
          INLA_CUDA(cudaMemsetAsync(d_means.p + (size_t)k * n, 0, w, eng_.stream()));
          std::vector<double> ones(n, 1.0);
          INLA_CUDA(cudaMemcpyAsync(d_vars.p + (size_t)k * n, ones.data(), w, cudaMemcpyHostToDevice, eng_.stream()));
          INLA_CUDA(cudaStreamSynchronize(eng_.stream()));  // `ones` is released at the end of this block
        } else {
          lp[k] = -fk[k];
        }
      }
    }
    INLA_CUDA(cudaMemcpyAsync(means.data(), d_means.p, sizeof(double) * K * n, cudaMemcpyDeviceToHost, eng_.stream()));
    INLA_CUDA(cudaMemcpyAsync(vars.data(), d_vars.p, sizeof(double) * K * n, cudaMemcpyDeviceToHost, eng_.stream()));
  }
  out.phase_s[2] = since(t2);  // design + node evaluations (the host copy of the node results included)
  const auto t3 = std::chrono::steady_clock::now();
  double mx = -std::numeric_limits<double>::infinity();
  for (double v : lp) mx = std::max(mx, v);
  if (!std::isfinite(mx)) throw std::runtime_error("Newton-Raphson did not converge at any integration node");
  std::vector<double> dens(K), nw(K);
  double sw = 0.0;
  for (int k = 0; k < K; ++k) {
    dens[k] = std::exp(lp[k] - mx);
    sw += zw[k] * dens[k];
  }
  for (int k = 0; k < K; ++k) nw[k] = zw[k] * dens[k] / sw;
  // mixture moments of the latent field and the linear predictor eta = A x per node with its
  // diagonal variance (inference.rs:1370-1384, 1436-1466), on the device
  {
    cudaStream_t st = eng_.stream();
    const LaplaceSpec& S = eng_.spec();
    const int64_t nobs = S.identity_a ? n : S.nobs;
    DBuf<double> d_w, d_lat, d_pred, eta_local, etav_local;
    d_w.upload(nw.data(), K, st);
    d_lat.alloc(2 * (size_t)n);
    d_pred.alloc(2 * (size_t)nobs);
    DBuf<double>& d_eta = out.d_cond_eta ? *out.d_cond_eta : eta_local;
    DBuf<double>& d_etav = out.d_cond_eta_var ? *out.d_cond_eta_var : etav_local;
    d_eta.alloc((size_t)K * nobs);
    d_etav.alloc((size_t)K * nobs);
    dev_mixture_moments(st, K, n, d_w.p, d_means.p, n, d_vars.p, n, d_lat.p, d_lat.p + n);
    DevCsrA A;
    A.rp = eng_.d_acp();
    A.ci = eng_.d_aci();
    A.v = eng_.d_av();
    dev_project_nodes(st, nobs, A, K, d_means.p, n, d_vars.p, n, d_eta.p, d_etav.p);
    dev_mixture_moments(st, K, nobs, d_w.p, d_eta.p, nobs, d_etav.p, nobs, d_pred.p, d_pred.p + nobs);
    out.latent_mean.resize(n);
    out.latent_var.resize(n);
    out.pred_mean.resize(nobs);
    out.pred_var.resize(nobs);
    out.cond_eta.resize((size_t)K * nobs);
    out.cond_eta_var.resize((size_t)K * nobs);
    INLA_CUDA(cudaMemcpyAsync(out.latent_mean.data(), d_lat.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaMemcpyAsync(out.latent_var.data(), d_lat.p + n, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaMemcpyAsync(out.pred_mean.data(), d_pred.p, sizeof(double) * nobs, cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaMemcpyAsync(out.pred_var.data(), d_pred.p + nobs, sizeof(double) * nobs, cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaMemcpyAsync(out.cond_eta.data(), d_eta.p, sizeof(double) * K * nobs, cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaMemcpyAsync(out.cond_eta_var.data(), d_etav.p, sizeof(double) * K * nobs, cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaStreamSynchronize(st));
  }
  // model-selection inputs (inference.rs:1296-1304, 1470-1485): the node nearest the mode, the
  // Gaussian-approximation mlik there, and the observations rebuilt at the mode
  {
    double best = std::numeric_limits<double>::infinity();
    for (int k = 0; k < K; ++k) {
      double s2 = 0.0;
      for (int j = 0; j < m; ++j) s2 += z[(size_t)k * m + j] * z[(size_t)k * m + j];
      if (std::sqrt(s2) < best) {
        best = std::sqrt(s2);
        out.mode_index = k;
      }
    }
    if (!mlik_gaussian(lp[out.mode_index], m, neg.data(), out.mlik_gaussian))
      out.mlik_gaussian = std::numeric_limits<double>::quiet_NaN();
    const int T = eng_.ncomp();
    std::vector<double> coef(T), dcoef((size_t)m * T), dp1s(m);
    double p1s = 1.0;
    const bool mapped = map_(mode.data(), coef.data(), dcoef.data(), &p1s, dp1s.data()) == 0;
    out.p1scale_mode = mapped ? p1s : std::numeric_limits<double>::quiet_NaN();
    if (mapped) out.coef_mode = coef;
  }
  out.mlik = mx + std::log(std::fabs(sw));
  out.cond_mean = std::move(means);
  out.cond_var = std::move(vars);
  out.node_theta = thetas;
  out.node_weight = nw;
  out.node_logpost = lp;
  out.n_evals = n_evals_;
  out.n_batches = n_batches_;
  out.phase_s[3] = since(t3);
  out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace inla
