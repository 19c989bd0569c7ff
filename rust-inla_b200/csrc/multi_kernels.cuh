// Kernels of the multi-model Laplace engine: G independent latent models held as
// one block-diagonal field (model g owns latent columns [lat_off[g], lat_off[g+1])
// and observations [obs_off[g], obs_off[g+1])), B theta-sets, coefficients and
// likelihood scales per (theta-set, model). Per-model reductions run one CTA per
// (model, theta-set) over the model's contiguous range in a fixed order, so every
// result is deterministic and independent of the other models.
#pragma once
#include "devsym.hpp"
#include "laplace_kernels.cuh"

namespace inla {
namespace {

// rhs[b][j] = (A^T g_b)_j - sum_p (sum_t coef[b][seg(j)][t] comp[t][p]) x_b[row p]
__global__ void k_mnewton_rhs(int n, int ncomp, int G, const int* __restrict__ segc, const int64_t* __restrict__ qcp,
                              const int* __restrict__ qri, const double* __restrict__ comp, int64_t nnz,
                              const double* __restrict__ coef, const int64_t* __restrict__ atp,
                              const int* __restrict__ ati, const double* __restrict__ atv, int64_t nobs,
                              const double* __restrict__ g, const double* __restrict__ x, double* __restrict__ rhs) {
  const int b = blockIdx.y;
  const double* xb = x + (int64_t)b * n;
  const double* gb = g + (int64_t)b * nobs;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double* cb = coef + ((int64_t)b * G + segc[j]) * ncomp;
    double s = 0.0;
    for (int64_t a = atp[j]; a < atp[j + 1]; ++a) s += atv[a] * gb[ati[a]];
    double qx = 0.0;
    for (int64_t p = qcp[j]; p < qcp[j + 1]; ++p) {
      double v = 0.0;
      for (int t = 0; t < ncomp; ++t) v += cb[t] * comp[(int64_t)t * nnz + p];
      qx += v * xb[qri[p]];
    }
    rhs[(int64_t)b * n + j] = s - qx;
  }
}

// x_trial = x + alpha[b][seg(j)] step
__global__ void k_maxpy(int n, int G, const int* __restrict__ segc, const double* __restrict__ x,
                        const double* __restrict__ step, const double* __restrict__ alpha, double* __restrict__ xt) {
  const int b = blockIdx.y;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int64_t o = (int64_t)b * n + j;
    xt[o] = x[o] + alpha[(int64_t)b * G + segc[j]] * step[o];
  }
}

// Likelihood terms (inference.rs:170-311) with the family scale p1scale[b][seg] and
// failure flags per (theta-set, model): bit 0 invalid evaluation, bit 1 non-finite log p.
__global__ void k_meval_lik(int fam, int64_t nobs, int G, const int* __restrict__ sego,
                            const double* __restrict__ eta, const double* __restrict__ y,
                            const double* __restrict__ p1, const double* __restrict__ p2,
                            const double* __restrict__ p1scale, double* __restrict__ logp, double* __restrict__ grad,
                            double* __restrict__ w, double* __restrict__ dw, int* __restrict__ bad) {
  const int b = blockIdx.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nobs; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = (int64_t)b * nobs + i;
    const int sg = sego[i];
    const double sc = p1scale ? p1scale[(int64_t)b * G + sg] : 1.0;
    double lp = 0, gr = 0, h = 0, d = 0;
    int flag = 0;
    if (d_eval_lik(fam, eta[o], y[i], (p1 ? p1[i] : 1.0) * sc, p2 ? p2[i] : 1.0, lp, gr, h, d)) {
      flag = 1;
      lp = NAN;
    } else if (!isfinite(lp)) {
      flag = 2;
    }
    logp[o] = lp;
    grad[o] = gr;
    w[o] = -h;
    if (dw) dw[o] = d;
    if (flag) atomicOr(bad + (int64_t)b * G + sg, flag);
  }
}

// d loglik / d log p1scale of the Gaussian family per observation: 1/2 - w (y - eta)^2 / 2
__global__ void k_gauss_dll_terms(int64_t nobs, const double* __restrict__ eta, const double* __restrict__ y,
                                  const double* __restrict__ w, double* __restrict__ out) {
  const int b = blockIdx.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nobs; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = (int64_t)b * nobs + i;
    const double r = y[i] - eta[o];
    out[o] = 0.5 - 0.5 * w[o] * r * r;
  }
}

// out[b][g] = {max |v| over the model's range, all finite ? 1 : 0}
template <int NT>
__global__ void __launch_bounds__(NT) k_seg_max(const int64_t* __restrict__ off, int G, int64_t stride,
                                               const double* __restrict__ v, double* __restrict__ out) {
  __shared__ double red[NT];
  const int g = blockIdx.x, b = blockIdx.y;
  const double* vb = v + (int64_t)b * stride;
  double mx = 0.0, fin = 1.0;
  for (int64_t j = off[g] + threadIdx.x; j < off[g + 1]; j += NT) {
    const double s = vb[j];
    if (!isfinite(s)) fin = 0.0;
    else mx = fmax(mx, fabs(s));
  }
  mx = block_max<NT>(mx, red);
  fin = -block_max<NT>(-fin, red);
  if (threadIdx.x == 0) {
    out[2 * ((int64_t)b * G + g)] = mx;
    out[2 * ((int64_t)b * G + g) + 1] = fin;
  }
}

// out[b][g] = max |a - c| over the model's range
template <int NT>
__global__ void __launch_bounds__(NT) k_seg_maxdiff(const int64_t* __restrict__ off, int G, int64_t stride,
                                                   const double* __restrict__ a, const double* __restrict__ c,
                                                   double* __restrict__ out) {
  __shared__ double red[NT];
  const int g = blockIdx.x, b = blockIdx.y;
  double mx = 0.0;
  for (int64_t j = off[g] + threadIdx.x; j < off[g + 1]; j += NT)
    mx = fmax(mx, fabs(a[(int64_t)b * stride + j] - c[(int64_t)b * stride + j]));
  mx = block_max<NT>(mx, red);
  if (threadIdx.x == 0) out[(int64_t)b * G + g] = mx;
}

// out[b][g] = sum of v over the model's range
template <int NT>
__global__ void __launch_bounds__(NT) k_seg_sum(const int64_t* __restrict__ off, int G, int64_t stride,
                                               const double* __restrict__ v, double* __restrict__ out) {
  __shared__ double red[NT];
  const int g = blockIdx.x, b = blockIdx.y;
  double s = 0.0;
  for (int64_t j = off[g] + threadIdx.x; j < off[g + 1]; j += NT) s += v[(int64_t)b * stride + j];
  s = block_sum<NT>(s, red);
  if (threadIdx.x == 0) out[(int64_t)b * G + g] = s;
}

// log|Q_bg| = sum of log|D_j| over the model's pivots (permuted columns
// [poff[g], poff[g+1])) and the pivot gate of sparse_ldlt.rs:104-149 per model.
template <int NT>
__global__ void __launch_bounds__(NT) k_seg_logdet(DevSym S, const double* __restrict__ F, int64_t fstride,
                                                  const int64_t* __restrict__ poff, int G, double* __restrict__ ld,
                                                  int* __restrict__ st) {
  __shared__ double red[NT];
  const int g = blockIdx.x, b = blockIdx.y;
  const double* Fb = F + (int64_t)b * fstride;
  double acc = 0.0, sing = 0.0, nonfin = 0.0;
  for (int64_t j = poff[g] + threadIdx.x; j < poff[g + 1]; j += NT) {
    const double d = Fb[S.dpos[j]];
    const double ad = fabs(d);
    if (!isfinite(d)) nonfin = 1.0;
    else if (ad < 1e-14) sing = 1.0;
    acc += log(ad);
  }
  acc = block_sum<NT>(acc, red);
  sing = block_max<NT>(sing, red);
  nonfin = block_max<NT>(nonfin, red);
  if (threadIdx.x == 0) {
    ld[(int64_t)b * G + g] = acc;
    st[(int64_t)b * G + g] = (sing > 0.0 ? kStatusSingular : 0) | (nonfin > 0.0 ? kStatusNotFinite : 0);
  }
}

// Per-model quadratic forms over the model's columns: out[b][g][0] = x^T Q x with the
// model's coefficients, out[b][g][1 + t] = x^T M_t x; with z != nullptr the bilinear forms
// z^T M_t x go to out[b][g][t] (no total).
template <int NT>
__global__ void __launch_bounds__(NT) k_seg_quad(const int64_t* __restrict__ off, int G, int n, int ncomp,
                                                const int64_t* __restrict__ qcp, const int* __restrict__ qri,
                                                const double* __restrict__ comp, int64_t nnz,
                                                const double* __restrict__ coef, const double* __restrict__ z,
                                                const double* __restrict__ x, double* __restrict__ out) {
  __shared__ double red[NT];
  const int g = blockIdx.x, b = blockIdx.y;
  const double* xb = x + (int64_t)b * n;
  const double* zb = z ? z + (int64_t)b * n : xb;
  double acc[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) acc[t] = 0.0;
  for (int64_t j = off[g] + threadIdx.x; j < off[g + 1]; j += NT) {
    const double zj = zb[j];
    for (int64_t p = qcp[j]; p < qcp[j + 1]; ++p) {
      const double zx = zj * xb[qri[p]];
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (t < ncomp) acc[t] += comp[(int64_t)t * nnz + p] * zx;
    }
  }
  const int T1 = ncomp + 1;
  double* ob = out + ((int64_t)b * G + g) * T1;
  const double* cb = coef + ((int64_t)b * G + g) * ncomp;
  double total = 0.0;
  for (int t = 0; t < ncomp && t < 8; ++t) {
    const double s = block_sum<NT>(acc[t], red);
    if (z) {
      if (threadIdx.x == 0) ob[t] = s;
    } else {
      if (threadIdx.x == 0) ob[1 + t] = s;
      total += cb[t] * s;
    }
  }
  if (!z && threadIdx.x == 0) ob[0] = total;
}

// Per-model trace contractions of Sigma on the full pattern (entries [eoff[g], eoff[g+1])):
// out[b][g][t] = tr(Sigma M_t), out[b][g][ncomp] = tr(Sigma A^T diag(w2) A) (if w2).
template <int NT>
__global__ void __launch_bounds__(NT) k_seg_trace(const int64_t* __restrict__ eoff, int G, int64_t nnz, int ncomp,
                                                 const double* __restrict__ comp, const double* __restrict__ sigma,
                                                 const int* __restrict__ cptr, const int* __restrict__ cobs,
                                                 const double* __restrict__ cprod, const double* __restrict__ w2,
                                                 int64_t nobs, double* __restrict__ out) {
  __shared__ double red[NT];
  const int g = blockIdx.x, b = blockIdx.y;
  const double* sb = sigma + (int64_t)b * nnz;
  double acc[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) acc[t] = 0.0;
  for (int64_t p = eoff[g] + threadIdx.x; p < eoff[g + 1]; p += NT) {
    const double sv = sb[p];
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (t < ncomp) acc[t] += sv * comp[(int64_t)t * nnz + p];
    if (w2) {
      double a = 0.0;
      for (int q = cptr[p]; q < cptr[p + 1]; ++q) a += w2[(int64_t)b * nobs + cobs[q]] * cprod[q];
      acc[8] += sv * a;
    }
  }
  const int T1 = ncomp + 1;
  double* ob = out + ((int64_t)b * G + g) * T1;
  for (int t = 0; t < ncomp && t < 8; ++t) {
    const double s = block_sum<NT>(acc[t], red);
    if (threadIdx.x == 0) ob[t] = s;
  }
  const double s = block_sum<NT>(acc[8], red);
  if (threadIdx.x == 0) ob[ncomp] = w2 ? s : 0.0;
}

}  // namespace
}  // namespace inla
