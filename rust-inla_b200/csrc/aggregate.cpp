#include "aggregate.hpp"

#include <algorithm>
#include <vector>

#include "host_par.hpp"

namespace inla {

void mixture_moments(int K, int64_t len, const double* w, const double* cmean, const double* cvar, double* mean,
                     double* var) {
  parallel_for(len, [&](int64_t i0, int64_t i1) {
    for (int64_t i = i0; i < i1; ++i) {
      double mi = 0.0;
      for (int k = 0; k < K; ++k) mi += w[k] * cmean[(size_t)k * len + i];
      double vi = 0.0;
      for (int k = 0; k < K; ++k) {
        const double d = cmean[(size_t)k * len + i] - mi;
        vi += w[k] * (cvar[(size_t)k * len + i] + d * d);
      }
      mean[i] = mi;
      var[i] = vi;
    }
  });
}

void project_nodes(int64_t nobs, int64_t n, const int64_t* acp, const int64_t* aci, const double* av, int K,
                   const double* cmean, const double* cvar, double* eta, double* eta_var) {
  if (!acp) {
    std::copy(cmean, cmean + (size_t)K * n, eta);
    std::copy(cvar, cvar + (size_t)K * n, eta_var);
    return;
  }
  parallel_for(
      nobs,
      [&](int64_t r0, int64_t r1) {
        for (int k = 0; k < K; ++k) {
          const double* x = cmean + (size_t)k * n;
          const double* v = cvar + (size_t)k * n;
          for (int64_t r = r0; r < r1; ++r) {
            double e = 0.0, s = 0.0;
            for (int64_t p = acp[r]; p < acp[r + 1]; ++p) {
              const double a = av[p], xv = x[aci[p]];
              if (xv != 0.0) e += a * xv;
              s += a * a * v[aci[p]];
            }
            eta[(size_t)k * nobs + r] = e;
            eta_var[(size_t)k * nobs + r] = s;
          }
        }
      },
      2048);
}

void predictor_moments(int64_t nobs, int64_t n, const int64_t* acp, const int64_t* aci, const double* av, int K,
                       const double* w, const double* cmean, const double* cvar, double* mean, double* var) {
  if (!acp) {
    mixture_moments(K, n, w, cmean, cvar, mean, var);
    return;
  }
  std::vector<double> eta((size_t)K * nobs), ev((size_t)K * nobs);
  project_nodes(nobs, n, acp, aci, av, K, cmean, cvar, eta.data(), ev.data());
  mixture_moments(K, nobs, w, eta.data(), ev.data(), mean, var);
}

}  // namespace inla
