#include "aggregate.hpp"

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

void predictor_moments(int64_t nobs, int64_t n, const int64_t* acp, const int64_t* aci, const double* av, int K,
                       const double* w, const double* cmean, const double* cvar, double* mean, double* var) {
  if (!acp) {
    mixture_moments(K, n, w, cmean, cvar, mean, var);
    return;
  }
  parallel_for(
      nobs,
      [&](int64_t r0, int64_t r1) {
        std::vector<double> eta(K), ev(K);
        for (int64_t r = r0; r < r1; ++r) {
          for (int k = 0; k < K; ++k) {
            const double* x = cmean + (size_t)k * n;
            const double* v = cvar + (size_t)k * n;
            double e = 0.0, s = 0.0;
            for (int64_t p = acp[r]; p < acp[r + 1]; ++p) {
              const double a = av[p], xv = x[aci[p]];
              if (xv != 0.0) e += a * xv;
              s += a * a * v[aci[p]];
            }
            eta[k] = e;
            ev[k] = s;
          }
          double mi = 0.0;
          for (int k = 0; k < K; ++k) mi += w[k] * eta[k];
          double vi = 0.0;
          for (int k = 0; k < K; ++k) {
            const double d = eta[k] - mi;
            vi += w[k] * (ev[k] + d * d);
          }
          mean[r] = mi;
          var[r] = vi;
        }
      },
      2048);
}

}  // namespace inla
