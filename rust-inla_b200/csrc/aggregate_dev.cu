// Device post-node aggregation (see aggregate_dev.hpp).
#include "aggregate_dev.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

#include "likelihood.cuh"
#include "model_select_core.cuh"

namespace inla {

namespace {

constexpr int kAggNT = 256;
constexpr int kRedNT = 1024;

inline int agg_blocks(int64_t len) { return (int)std::min<int64_t>((len + kAggNT - 1) / kAggNT, 4096); }

// One node per blockIdx.y, observations grid-strided. The multiply-adds are kept apart
// (__dmul_rn / __dadd_rn) so the sums equal the host's term by term.
__global__ void __launch_bounds__(kAggNT) k_project_nodes(int64_t nobs, const int64_t* __restrict__ rp,
                                                         const int* __restrict__ ci, const double* __restrict__ av,
                                                         const double* __restrict__ cmean, int64_t ldm,
                                                         const double* __restrict__ cvar, int64_t ldv,
                                                         double* __restrict__ eta, double* __restrict__ eta_var) {
  const int k = blockIdx.y;
  const double* x = cmean + (int64_t)k * ldm;
  const double* v = cvar + (int64_t)k * ldv;
  double* e_out = eta + (int64_t)k * nobs;
  double* v_out = eta_var + (int64_t)k * nobs;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nobs; i += (int64_t)gridDim.x * blockDim.x) {
    if (!rp) {
      e_out[i] = x[i];
      v_out[i] = v[i];
      continue;
    }
    double e = 0.0, s = 0.0;
    for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
      const double a = av[p], xv = x[ci[p]];
      if (xv != 0.0) e = __dadd_rn(e, __dmul_rn(a, xv));
      s = __dadd_rn(s, __dmul_rn(__dmul_rn(a, a), v[ci[p]]));
    }
    e_out[i] = e;
    v_out[i] = s;
  }
}

__global__ void __launch_bounds__(kAggNT) k_mixture(int K, int64_t len, const double* __restrict__ w,
                                                   const double* __restrict__ cmean, int64_t ldm,
                                                   const double* __restrict__ cvar, int64_t ldv,
                                                   double* __restrict__ mean, double* __restrict__ var) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    double mi = 0.0;
    for (int k = 0; k < K; ++k) mi = __dadd_rn(mi, __dmul_rn(w[k], cmean[(int64_t)k * ldm + i]));
    double vi = 0.0;
    for (int k = 0; k < K; ++k) {
      const double d = __dadd_rn(cmean[(int64_t)k * ldm + i], -mi);
      vi = __dadd_rn(vi, __dmul_rn(w[k], __dadd_rn(cvar[(int64_t)k * ldv + i], __dmul_rn(d, d))));
    }
    mean[i] = mi;
    var[i] = vi;
  }
}

__device__ __forceinline__ double obs_q1(const DevObs& o, int64_t i) { return (o.p1 ? o.p1[i] : 1.0) * o.p1scale; }
__device__ __forceinline__ double obs_q2(const DevObs& o, int64_t i) { return o.p2 ? o.p2[i] : 1.0; }

// log p(y_i | eta_ki) for every (node, observation); ok = 0 where the reference returns Err
__global__ void __launch_bounds__(kAggNT) k_ms_loglik(DevObs o, const double* __restrict__ eta,
                                                     double* __restrict__ ll, unsigned char* __restrict__ ok) {
  const int k = blockIdx.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < o.nobs; i += (int64_t)gridDim.x * blockDim.x) {
    double lp, g, h, dw;
    const int64_t q = (int64_t)k * o.nobs + i;
    const bool good = d_eval_lik(o.family, eta[q], o.y[i], obs_q1(o, i), obs_q2(o, i), lp, g, h, dw) == 0;
    ok[q] = good;
    ll[q] = good ? lp : NAN;
  }
}

// Fixed-order block sum: thread t adds entries t, t + NT, ... in order, then a tree.
template <int NT>
__device__ double block_sum(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

template <int NT>
__device__ int block_min(int v, int* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = min(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  const int r = red[0];
  __syncthreads();
  return r;
}

// DIC pieces (compute_dic, model_selection.rs:101-150): one CTA per node, the node's
// log-likelihood sum and its first failing observation (INT_MAX when none).
__global__ void __launch_bounds__(kRedNT) k_ms_dic_nodes(int64_t nobs, const double* __restrict__ ll,
                                                        const unsigned char* __restrict__ ok,
                                                        double* __restrict__ node_sum, int* __restrict__ node_bad) {
  __shared__ double red[kRedNT];
  __shared__ int ired[kRedNT];
  const int k = blockIdx.x;
  double s = 0.0;
  int bad = 0x7fffffff;
  for (int64_t i = threadIdx.x; i < nobs; i += kRedNT) {
    const int64_t q = (int64_t)k * nobs + i;
    if (ok[q]) s += ll[q];
    else bad = min(bad, (int)i);
  }
  s = block_sum<kRedNT>(s, red);
  bad = block_min<kRedNT>(bad, ired);
  if (threadIdx.x == 0) {
    node_sum[k] = s;
    node_bad[k] = bad;
  }
}

// WAIC per observation (compute_waic, model_selection.rs:152-211): lppd_i, the variance term
// and a code (1 failed likelihood, 2 non-finite predictive density).
__global__ void __launch_bounds__(kAggNT) k_ms_waic_obs(int64_t nobs, int K, const double* __restrict__ w,
                                                       const double* __restrict__ ll,
                                                       const unsigned char* __restrict__ ok,
                                                       double* __restrict__ lppd, double* __restrict__ pw,
                                                       int* __restrict__ bad) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nobs; i += (int64_t)gridDim.x * blockDim.x) {
    int code = 0;
    double mx = -INFINITY;
    for (int k = 0; k < K; ++k) {
      if (!ok[(int64_t)k * nobs + i]) {
        code = 1;
        break;
      }
      mx = fmax(mx, ll[(int64_t)k * nobs + i]);
    }
    double l_i = 0.0, p_i = 0.0;
    if (code == 0) {
      double sum_w_exp = 0.0, mean_ll = 0.0;
      for (int k = 0; k < K; ++k) {
        const double l = ll[(int64_t)k * nobs + i];
        sum_w_exp += w[k] * exp(l - mx);
        mean_ll += w[k] * l;
      }
      if (!(isfinite(sum_w_exp) && sum_w_exp > 0.0)) {
        code = 2;
      } else {
        l_i = mx + log(sum_w_exp);
        for (int k = 0; k < K; ++k) {
          const double d = ll[(int64_t)k * nobs + i] - mean_ll;
          p_i += w[k] * d * d;
        }
      }
    }
    lppd[i] = l_i;
    pw[i] = p_i;
    bad[i] = code;
  }
}

// One CTA: fixed-order sums of lppd_i and pw_i, and the first observation with a code.
__global__ void __launch_bounds__(kRedNT) k_ms_waic_sum(int64_t nobs, const double* __restrict__ lppd,
                                                       const double* __restrict__ pw, const int* __restrict__ bad,
                                                       double* __restrict__ out2, int* __restrict__ first_bad) {
  __shared__ double red[kRedNT];
  __shared__ int ired[kRedNT];
  double a = 0.0, b = 0.0;
  int fb = 0x7fffffff;
  for (int64_t i = threadIdx.x; i < nobs; i += kRedNT) {
    a += lppd[i];
    b += pw[i];
    if (bad[i]) fb = min(fb, (int)i);
  }
  a = block_sum<kRedNT>(a, red);
  b = block_sum<kRedNT>(b, red);
  fb = block_min<kRedNT>(fb, ired);
  if (threadIdx.x == 0) {
    out2[0] = a;
    out2[1] = b;
    *first_bad = fb;
  }
}

__global__ void __launch_bounds__(kAggNT) k_ms_cpo(DevObs o, int K, const double* __restrict__ w,
                                                  const double* __restrict__ eta, const double* __restrict__ ev,
                                                  double* __restrict__ cpo, double* __restrict__ pit,
                                                  int* __restrict__ failed) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < o.nobs; i += (int64_t)gridDim.x * blockDim.x) {
    double c, p;
    const bool good = ms_cpo_pit_obs(o.family, o.y[i], obs_q1(o, i), obs_q2(o, i), K, w, eta + i, ev + i, o.nobs, c, p);
    cpo[i] = c;
    pit[i] = p;
    failed[i] = good ? 0 : 1;
  }
}

__global__ void __launch_bounds__(kRedNT) k_int_sum(int64_t len, const int* __restrict__ v, int* __restrict__ out) {
  __shared__ double red[kRedNT];
  double a = 0.0;  // counts below 2^53 are exact in a double
  for (int64_t i = threadIdx.x; i < len; i += kRedNT) a += v[i];
  a = block_sum<kRedNT>(a, red);
  if (threadIdx.x == 0) *out = (int)a;
}

}  // namespace

void dev_project_nodes(cudaStream_t st, int64_t nobs, const DevCsrA& A, int K, const double* cmean, int64_t ldm,
                       const double* cvar, int64_t ldv, double* eta, double* eta_var) {
  if (K < 1 || nobs < 1) return;
  k_project_nodes<<<dim3(agg_blocks(nobs), K), kAggNT, 0, st>>>(nobs, A.rp, A.ci, A.v, cmean, ldm, cvar, ldv, eta,
                                                                eta_var);
  INLA_CUDA(cudaGetLastError());
}

void dev_mixture_moments(cudaStream_t st, int K, int64_t len, const double* d_w, const double* cmean, int64_t ldm,
                         const double* cvar, int64_t ldv, double* mean, double* var) {
  if (K < 1 || len < 1) return;
  k_mixture<<<agg_blocks(len), kAggNT, 0, st>>>(K, len, d_w, cmean, ldm, cvar, ldv, mean, var);
  INLA_CUDA(cudaGetLastError());
}

std::string dev_model_selection(cudaStream_t st, const DevObs& obs, int K, const double* w, int mode_index,
                                const double* d_eta, const double* d_eta_var, int what, AggScratch& sc,
                                ModelSelection& out) {
  const int64_t n = obs.nobs;
  if (K < 1 || mode_index < 0 || mode_index >= K) return "model selection: invalid node count or mode index";
  out = ModelSelection();
  const double NaN = std::numeric_limits<double>::quiet_NaN();
  sc.w.upload(w, K, st);
  if (n == 0) {  // nothing to sum: every criterion is its empty-sum value
    if (what & MS_DIC) out.mean_deviance = out.dic_p_eff = out.dic = 0.0;
    if (what & MS_WAIC) out.lppd = out.waic_p_eff = out.waic = 0.0;
    INLA_CUDA(cudaStreamSynchronize(st));
    return std::string();
  }
  if (what & (MS_DIC | MS_WAIC)) {
    sc.ll.alloc((size_t)K * n);
    sc.ok.alloc((size_t)K * n);
    k_ms_loglik<<<dim3(agg_blocks(n), K), kAggNT, 0, st>>>(obs, d_eta, sc.ll.p, sc.ok.p);
    INLA_CUDA(cudaGetLastError());
    if (what & MS_DIC) {
      sc.red.alloc(K);
      sc.nodebad.alloc(K);
      k_ms_dic_nodes<<<K, kRedNT, 0, st>>>(n, sc.ll.p, sc.ok.p, sc.red.p, sc.nodebad.p);
      INLA_CUDA(cudaGetLastError());
      std::vector<double> sums(K);
      std::vector<int> bad(K);
      INLA_CUDA(cudaMemcpyAsync(sums.data(), sc.red.p, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
      INLA_CUDA(cudaMemcpyAsync(bad.data(), sc.nodebad.p, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
      INLA_CUDA(cudaStreamSynchronize(st));
      for (int k = 0; k < K; ++k)  // node-major like the reference: the first node with a failure
        if (bad[k] != 0x7fffffff) return "DIC: likelihood evaluation failed at observation " + std::to_string(bad[k]);
      double mean_dev = 0.0;
      for (int k = 0; k < K; ++k) mean_dev += w[k] * (-2.0 * sums[k]);
      out.mean_deviance = mean_dev;
      out.dic_p_eff = mean_dev - (-2.0 * sums[mode_index]);
      out.dic = mean_dev + out.dic_p_eff;
    }
    if (what & MS_WAIC) {
      sc.lppd.alloc(n);
      sc.pw.alloc(n);
      sc.bad.alloc(n);
      sc.red.alloc(std::max(K, 2));
      sc.ired.alloc(1);
      k_ms_waic_obs<<<agg_blocks(n), kAggNT, 0, st>>>(n, K, sc.w.p, sc.ll.p, sc.ok.p, sc.lppd.p, sc.pw.p, sc.bad.p);
      k_ms_waic_sum<<<1, kRedNT, 0, st>>>(n, sc.lppd.p, sc.pw.p, sc.bad.p, sc.red.p, sc.ired.p);
      INLA_CUDA(cudaGetLastError());
      double s2[2];
      int fb = 0;
      INLA_CUDA(cudaMemcpyAsync(s2, sc.red.p, sizeof(s2), cudaMemcpyDeviceToHost, st));
      INLA_CUDA(cudaMemcpyAsync(&fb, sc.ired.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      INLA_CUDA(cudaStreamSynchronize(st));
      if (fb != 0x7fffffff) {
        int code = 0;
        INLA_CUDA(cudaMemcpy(&code, sc.bad.p + fb, sizeof(int), cudaMemcpyDeviceToHost));
        if (code == 1) return "WAIC: likelihood evaluation failed at observation " + std::to_string(fb);
        return "WAIC: non-finite predictive density at obs " + std::to_string(fb);
      }
      out.lppd = s2[0];
      out.waic_p_eff = s2[1];
      out.waic = -2.0 * (s2[0] - s2[1]);
    }
  }
  if (what & MS_CPO) {
    sc.cpo.alloc(n);
    sc.pit.alloc(n);
    sc.bad.alloc(n);
    sc.ired.alloc(1);
    k_ms_cpo<<<agg_blocks(n), kAggNT, 0, st>>>(obs, K, sc.w.p, d_eta, d_eta_var, sc.cpo.p, sc.pit.p, sc.bad.p);
    k_int_sum<<<1, kRedNT, 0, st>>>(n, sc.bad.p, sc.ired.p);
    INLA_CUDA(cudaGetLastError());
    out.cpo.assign(n, NaN);
    out.pit.assign(n, NaN);
    int nf = 0;
    INLA_CUDA(cudaMemcpyAsync(out.cpo.data(), sc.cpo.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaMemcpyAsync(out.pit.data(), sc.pit.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaMemcpyAsync(&nf, sc.ired.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    INLA_CUDA(cudaStreamSynchronize(st));
    out.cpo_failures = nf;
  }
  return std::string();
}

}  // namespace inla
