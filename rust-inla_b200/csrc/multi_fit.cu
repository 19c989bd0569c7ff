// Lockstep INLA fit of G independent models over the multi-model engine.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>

#include "capi_common.hpp"
#include "driver.hpp"
#include "inla_b200.h"
#include "multi.hpp"

namespace inla {

void MultiDriver::evaluate(int B, const double* th, bool want_grad, bool want_var, double* f, double* grad,
                           std::vector<double>* xs, std::vector<double>* vs) {
  const int G = eng_.G(), T = eng_.ncomp(), m = m_, T1 = T + 1;
  const int64_t n = eng_.n();
  const int Bmax = eng_.max_batch();
  std::vector<double> coef, dcoef, p1s, dp1s, gp(m);
  if (xs) xs->assign((size_t)B * n, 0.0);
  if (vs) vs->assign((size_t)B * n, 0.0);
  for (int b0 = 0; b0 < B; b0 += Bmax) {
    if (cancel_ && cancel_()) throw InlaError(INLA_ERR_CANCELLED, "Operation cancelled by user");
    const int Bc = std::min(Bmax, B - b0);
    const size_t BG = (size_t)Bc * G;
    coef.assign(BG * T, 0.0);
    dcoef.assign(BG * m * T, 0.0);
    p1s.assign(BG, 1.0);
    dp1s.assign(BG * m, 0.0);
    std::vector<char> ok(BG, 1);
    for (int b = 0; b < Bc; ++b)
      for (int g = 0; g < G; ++g) {
        const size_t q = (size_t)b * G + g;
        const double* t = th + ((size_t)(b0 + b) * G + g) * m;
        if (map_(g, t, &coef[q * T], &dcoef[q * m * T], &p1s[q], &dp1s[q * m]) != 0) {
          ok[q] = 0;  // keep the batch well-formed with a harmless point
          for (int c = 0; c < T; ++c) coef[q * T + c] = 1.0;
          p1s[q] = 1.0;
        }
      }
    MultiOut R;
    eng_.eval(Bc, coef.data(), p1s.data(), (want_grad ? LAP_GRADIENT : 0) | (want_var ? LAP_VARIANCES : 0), R);
    ++n_batches_;
    n_model_evals_ += (int64_t)BG;
    if (xs)
      INLA_CUDA(cudaMemcpyAsync(xs->data() + (size_t)b0 * n, eng_.d_x(), sizeof(double) * Bc * n,
                                cudaMemcpyDeviceToHost, eng_.stream()));
    if (vs && want_var)
      INLA_CUDA(cudaMemcpyAsync(vs->data() + (size_t)b0 * n, eng_.d_var(), sizeof(double) * Bc * n,
                                cudaMemcpyDeviceToHost, eng_.stream()));
    INLA_CUDA(cudaStreamSynchronize(eng_.stream()));
    for (int b = 0; b < Bc; ++b)
      for (int g = 0; g < G; ++g) {
        const size_t q = (size_t)b * G + g, k = (size_t)(b0 + b) * G + g;
        const double* t = th + k * m;
        const bool good = ok[q] && R.status[q] == LAP_OK && std::isfinite(R.mlik[q]);
        if (!good) {
          f[k] = 1e12;  // hyper_opt.rs:39-45: keep the search alive on a failed Laplace
          if (grad)
            for (int i = 0; i < m; ++i) grad[k * m + i] = 0.0;
          continue;
        }
        const double lp = prior_(g, t, want_grad ? gp.data() : nullptr);
        f[k] = -(R.mlik[q] + lp);
        if (want_grad && grad)
          for (int i = 0; i < m; ++i) {
            double d = 0.0;
            for (int c = 0; c < T; ++c) {
              const double dc = dcoef[q * m * T + (size_t)i * T + c];
              if (dc == 0.0) continue;
              d += dc * (0.5 * R.trP[q * T1 + c] - 0.5 * R.trQ[q * T1 + c] - 0.5 * R.xMx[q * T1 + c] +
                         0.5 * R.zMx[q * T1 + c]);
            }
            const double ds = dp1s[q * m + i];
            if (ds != 0.0) d += ds / p1s[q] * (R.dll[q] - 0.5 * R.trQ[q * T1 + T]);
            grad[k * m + i] = -(d + gp[i]);
          }
      }
  }
}

void MultiDriver::fit(const double* theta0, const MultiFitOptions& opt, MultiFitResult& out) {
  const auto t0 = std::chrono::steady_clock::now();
  const int G = eng_.G(), m = m_, per = 1 + 2 * m;
  const int64_t n = eng_.n();
  const std::vector<int64_t>& lo = eng_.lat_off();
  const double h = 1e-3;  // gradient stencil of the mode search
  n_batches_ = 0;
  cancel_ = opt.cancel;
  n_model_evals_ = 0;

  // ---- mode search: InlaDriver::newton per model, all models in lockstep ----------
  // stencil points of model g around centre c: c, c +- h e_i
  std::vector<double> pts((size_t)per * G * m), fk((size_t)per * G), gk((size_t)per * G * m);
  auto stencils = [&](const std::vector<double>& centres) {
    for (int b = 0; b < per; ++b)
      for (int g = 0; g < G; ++g) {
        double* t = &pts[((size_t)b * G + g) * m];
        for (int i = 0; i < m; ++i) t[i] = centres[(size_t)g * m + i];
        if (b > 0) t[(b - 1) / 2] += ((b - 1) % 2 == 0 ? h : -h);
      }
    evaluate(per, pts.data(), true, false, fk.data(), gk.data());
  };
  // f, g, H of model g from the last stencil batch
  auto read = [&](int g, double& f, std::vector<double>& gr, std::vector<double>& H) {
    f = fk[g];
    bool bad = !(f < 1e11);
    gr.assign(gk.begin() + (size_t)g * m, gk.begin() + (size_t)(g + 1) * m);
    H.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; ++i) {
      const size_t kp = (size_t)(1 + 2 * i) * G + g, km = (size_t)(2 + 2 * i) * G + g;
      if (!(fk[kp] < 1e11) || !(fk[km] < 1e11)) bad = true;
      for (int j = 0; j < m; ++j) H[i * m + j] = (gk[kp * m + j] - gk[km * m + j]) / (2.0 * h);
    }
    for (int i = 0; i < m; ++i)
      for (int j = i + 1; j < m; ++j) H[i * m + j] = H[j * m + i] = 0.5 * (H[i * m + j] + H[j * m + i]);
    if (bad) f = 1e12;
  };
  std::vector<double> x(theta0, theta0 + (size_t)G * m), f(G), gv((size_t)G * m), Hv((size_t)G * m * m);
  std::vector<double> delta(G, 2.0), p((size_t)G * m, 0.0), slope(G, 0.0), pmax(G, 0.0), xc((size_t)G * m);
  std::vector<int> cand(G, -1), iters(G, 0);
  std::vector<char> active(G, 1), capped(G, 0);
  stencils(x);
  {
    std::vector<double> gr, H;
    for (int g = 0; g < G; ++g) {
      read(g, f[g], gr, H);
      std::copy(gr.begin(), gr.end(), gv.begin() + (size_t)g * m);
      std::copy(H.begin(), H.end(), Hv.begin() + (size_t)g * m * m);
    }
  }
  static const double kA[3] = {1.0, 0.5, 0.25};
  // start of a Newton iteration for model g: convergence test, then the direction
  auto begin_iter = [&](int g) {
    if (iters[g] >= opt.max_iter) {
      active[g] = 0;
      return;
    }
    iters[g] += 1;
    const double* gg = &gv[(size_t)g * m];
    double gmax = 0.0;
    for (int i = 0; i < m; ++i) gmax = std::max(gmax, std::fabs(gg[i]));
    if (gmax < opt.tol) {
      active[g] = 0;
      return;
    }
    std::vector<double> Hg(Hv.begin() + (size_t)g * m * m, Hv.begin() + (size_t)(g + 1) * m * m), lam, V;
    symmetric_eigen(Hg, m, lam, V);
    double lmax = 0.0;
    for (double l : lam) lmax = std::max(lmax, std::fabs(l));
    double* pg = &p[(size_t)g * m];
    for (int i = 0; i < m; ++i) pg[i] = 0.0;
    for (int j = 0; j < m; ++j) {
      const double l = std::max(std::fabs(lam[j]), 1e-8 * std::max(lmax, 1e-300));
      double vg = 0.0;
      for (int i = 0; i < m; ++i) vg += V[i * m + j] * gg[i];
      for (int i = 0; i < m; ++i) pg[i] -= V[i * m + j] * vg / l;
    }
    double pm = 0.0, sl = 0.0;
    for (int i = 0; i < m; ++i) {
      pm = std::max(pm, std::fabs(pg[i]));
      sl += pg[i] * gg[i];
    }
    capped[g] = pm > delta[g];
    if (capped[g]) {
      for (int i = 0; i < m; ++i) pg[i] *= delta[g] / pm;
      sl *= delta[g] / pm;
    }
    pmax[g] = pm;
    slope[g] = sl;
    cand[g] = 0;
  };
  for (int g = 0; g < G; ++g) begin_iter(g);
  for (int round = 0; round < 3 * opt.max_iter + 3; ++round) {
    bool any = false;
    for (int g = 0; g < G; ++g) {
      for (int i = 0; i < m; ++i)
        xc[(size_t)g * m + i] = active[g] ? x[(size_t)g * m + i] + kA[cand[g]] * p[(size_t)g * m + i]
                                          : x[(size_t)g * m + i];
      any = any || active[g];
    }
    if (!any) break;
    stencils(xc);
    std::vector<double> gr, H;
    for (int g = 0; g < G; ++g) {
      if (!active[g]) continue;
      double fc;
      read(g, fc, gr, H);
      const int k = cand[g];
      if (fc < 1e11 && fc <= f[g] + 1e-4 * kA[k] * slope[g]) {
        const double fprev = f[g];
        std::copy(xc.begin() + (size_t)g * m, xc.begin() + (size_t)(g + 1) * m, x.begin() + (size_t)g * m);
        f[g] = fc;
        std::copy(gr.begin(), gr.end(), gv.begin() + (size_t)g * m);
        std::copy(H.begin(), H.end(), Hv.begin() + (size_t)g * m * m);
        if (k == 0 && capped[g]) delta[g] = std::min(4.0 * delta[g], 8.0);
        else if (k > 0) delta[g] = std::max(0.25, kA[k] * std::min(pmax[g], delta[g]));
        if (std::fabs(fprev - fc) < 1e-12 * (1.0 + std::fabs(fc))) active[g] = 0;
        else begin_iter(g);
      } else if (k < 2) {
        cand[g] = k + 1;  // shorter step of the same direction, next round
      } else {
        delta[g] *= 0.25;
        if (delta[g] < 1e-8) active[g] = 0;
        else begin_iter(g);
      }
    }
  }

  // ---- Hessian for the CCD design (inference.rs:1260-1266) --------------------------
  out.mode = x;
  out.hessian.assign((size_t)G * m * m, 0.0);
  out.status.assign(G, 0);
  out.mode_iters = iters;
  // step per model as the single-model driver: h_g = max(1e-4, 0.05 max |theta_g|)
  std::vector<double> hstep(G);
  for (int g = 0; g < G; ++g) {
    double hh = 1e-4;
    for (int i = 0; i < m; ++i) hh = std::max(hh, 0.05 * std::fabs(x[(size_t)g * m + i]));
    hstep[g] = hh;
  }
  if (opt.hessian == 1) {  // central differences of the adjoint gradient, 2m points per model
    std::vector<double> hp((size_t)2 * m * G * m), hf((size_t)2 * m * G), hg((size_t)2 * m * G * m);
    for (int i = 0; i < m; ++i)
      for (int s = 0; s < 2; ++s)
        for (int g = 0; g < G; ++g) {
          double* t = &hp[((size_t)(2 * i + s) * G + g) * m];
          for (int j = 0; j < m; ++j) t[j] = x[(size_t)g * m + j];
          t[i] += s == 0 ? hstep[g] : -hstep[g];
        }
    evaluate(2 * m, hp.data(), true, false, hf.data(), hg.data());
    for (int g = 0; g < G; ++g) {
      double* Hg = &out.hessian[(size_t)g * m * m];
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j)
          Hg[i * m + j] = -(hg[((size_t)(2 * i) * G + g) * m + j] - hg[((size_t)(2 * i + 1) * G + g) * m + j]) /
                          (2.0 * hstep[g]);
      for (int i = 0; i < m; ++i)
        for (int j = i + 1; j < m; ++j) Hg[i * m + j] = Hg[j * m + i] = 0.5 * (Hg[i * m + j] + Hg[j * m + i]);
    }
  } else {
    // hyper_opt.rs:197-259 per model, step h_g = max(1e-4, 0.05 max |theta_g|)
    std::vector<std::vector<std::pair<int, double>>> moves{{}};
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        if (i == j) {
          moves.push_back({{i, 1.0}});
          moves.push_back({{i, -1.0}});
        } else if (i < j) {
          moves.push_back({{i, 1.0}, {j, 1.0}});
          moves.push_back({{i, 1.0}, {j, -1.0}});
          moves.push_back({{i, -1.0}, {j, 1.0}});
          moves.push_back({{i, -1.0}, {j, -1.0}});
        }
      }
    const int K = (int)moves.size();
    const std::vector<double>& hg = hstep;
    std::vector<double> hp((size_t)K * G * m), hf((size_t)K * G);
    for (int k = 0; k < K; ++k)
      for (int g = 0; g < G; ++g) {
        double* t = &hp[((size_t)k * G + g) * m];
        for (int j = 0; j < m; ++j) t[j] = x[(size_t)g * m + j];
        for (const auto& mv : moves[k]) t[mv.first] += mv.second * hg[g];
      }
    evaluate(K, hp.data(), false, false, hf.data(), nullptr);
    for (int g = 0; g < G; ++g) {
      auto val = [&](int k) { return -hf[(size_t)k * G + g]; };
      double* Hg = &out.hessian[(size_t)g * m * m];
      const double g0 = val(0), hh = hg[g];
      int k = 1;
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
          if (i == j) {
            Hg[i * m + i] = (val(k) - 2.0 * g0 + val(k + 1)) / (hh * hh);
            k += 2;
          } else if (i < j) {
            const double v = (val(k) - val(k + 1) - val(k + 2) + val(k + 3)) / (4.0 * hh * hh);
            Hg[i * m + j] = Hg[j * m + i] = v;
            k += 4;
          }
        }
    }
  }

  // ---- CCD nodes per model (inference.rs:1262-1466) ---------------------------------
  std::vector<double> z, zw;
  ccd_design(m, opt.f0, z, zw);
  const int K = (int)zw.size();
  std::vector<double> nodes((size_t)K * G * m);
  for (int g = 0; g < G; ++g) {
    std::vector<double> neg((size_t)m * m), sigma, lam, V;
    for (int i = 0; i < m * m; ++i) neg[i] = -out.hessian[(size_t)g * m * m + i];
    const bool inv = invert_symmetric_matrix(neg, m, sigma);
    if (!inv) {
      out.status[g] = 2;
      sigma.assign((size_t)m * m, 0.0);
      for (int i = 0; i < m; ++i) sigma[i * m + i] = 1.0;
    }
    symmetric_eigen(sigma, m, lam, V);
    for (int k = 0; k < K; ++k)
      for (int i = 0; i < m; ++i) {
        double d = 0.0;
        for (int j = 0; j < m; ++j) d += V[i * m + j] * std::sqrt(std::fabs(lam[j])) * z[(size_t)k * m + j];
        nodes[((size_t)k * G + g) * m + i] = x[(size_t)g * m + i] + d;
      }
  }
  std::vector<double> nf((size_t)K * G), means, vars;
  evaluate(K, nodes.data(), false, true, nf.data(), nullptr, &means, &vars);
  out.latent_mean.assign(n, 0.0);
  out.latent_var.assign(n, 0.0);
  const MultiSpec& S = eng_.spec();
  out.pred_mean.assign(S.nobs, 0.0);
  out.pred_var.assign(S.nobs, 0.0);
  out.K = K;
  out.cond_eta.assign((size_t)K * S.nobs, 0.0);
  out.cond_eta_var.assign((size_t)K * S.nobs, 0.0);
  out.node_weight.assign((size_t)G * K, 0.0);
  out.p1scale_mode.assign(G, NAN);
  out.logpost_mode.assign(G, NAN);
  {  // the node with the smallest |z| (inference.rs:1296-1304), shared by every model
    double best = std::numeric_limits<double>::infinity();
    for (int k = 0; k < K; ++k) {
      double s2 = 0.0;
      for (int j = 0; j < m; ++j) s2 += z[(size_t)k * m + j] * z[(size_t)k * m + j];
      if (std::sqrt(s2) < best) {
        best = std::sqrt(s2);
        out.mode_index = k;
      }
    }
  }
  out.mlik.assign(G, NAN);
  for (int g = 0; g < G; ++g) {
    std::vector<double> lp(K);
    double mx = -std::numeric_limits<double>::infinity();
    for (int k = 0; k < K; ++k) {
      const double fv = nf[(size_t)k * G + g];
      lp[k] = fv >= 1e12 ? -std::numeric_limits<double>::infinity() : -fv;
      mx = std::max(mx, lp[k]);
    }
    if (!std::isfinite(mx)) {
      out.status[g] = 1;
      continue;
    }
    std::vector<double> nw(K);
    double sw = 0.0;
    for (int k = 0; k < K; ++k) sw += zw[k] * std::exp(lp[k] - mx);
    for (int k = 0; k < K; ++k) nw[k] = zw[k] * std::exp(lp[k] - mx) / sw;
    for (int64_t i = lo[g]; i < lo[g + 1]; ++i) {
      double mi = 0.0;
      for (int k = 0; k < K; ++k)
        if (std::isfinite(lp[k])) mi += nw[k] * means[(size_t)k * n + i];
      double vi = 0.0;
      for (int k = 0; k < K; ++k) {
        if (!std::isfinite(lp[k])) continue;
        const double d = means[(size_t)k * n + i] - mi;
        vi += nw[k] * (vars[(size_t)k * n + i] + d * d);
      }
      out.latent_mean[i] = mi;
      out.latent_var[i] = vi;
    }
    // linear predictor of the model's observations (inference.rs:1370-1384, 1451-1466):
    // per node eta_k = A x_k and sum_j A_ij^2 var_kj as matvec_csc / predictor_variances_diag
    // sum them, then the same mixture
    std::vector<double> eta(K), ev(K);
    for (int64_t r = S.obs_off[g]; r < S.obs_off[g + 1]; ++r) {
      for (int k = 0; k < K; ++k) {
        double e = 0.0, s2 = 0.0;
        for (int64_t p = S.acp[r]; p < S.acp[r + 1]; ++p) {
          const double a = S.av[p], xv = means[(size_t)k * n + S.aci[p]];
          if (xv != 0.0) e += a * xv;
          s2 += a * a * vars[(size_t)k * n + S.aci[p]];
        }
        eta[k] = e;
        ev[k] = s2;
        out.cond_eta[(size_t)k * S.nobs + r] = e;
        out.cond_eta_var[(size_t)k * S.nobs + r] = s2;
      }
      double mi = 0.0;
      for (int k = 0; k < K; ++k)
        if (std::isfinite(lp[k])) mi += nw[k] * eta[k];
      double vi = 0.0;
      for (int k = 0; k < K; ++k) {
        if (!std::isfinite(lp[k])) continue;
        const double d = eta[k] - mi;
        vi += nw[k] * (ev[k] + d * d);
      }
      out.pred_mean[r] = mi;
      out.pred_var[r] = vi;
    }
    out.mlik[g] = mx + std::log(std::fabs(sw));
    for (int k = 0; k < K; ++k) out.node_weight[(size_t)g * K + k] = std::isfinite(lp[k]) ? nw[k] : 0.0;
    out.logpost_mode[g] = lp[out.mode_index];
    {  // observations rebuilt at the model's mode (inference.rs:1478-1485)
      const int T = eng_.ncomp();
      std::vector<double> coef(T), dcoef((size_t)m * T), dp1s(m);
      double p1s = 1.0;
      if (map_(g, &out.mode[(size_t)g * m], coef.data(), dcoef.data(), &p1s, dp1s.data()) == 0)
        out.p1scale_mode[g] = p1s;
    }
  }
  out.n_batches = n_batches_;
  out.n_model_evals = n_model_evals_;
  out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace inla
