// CUDA kernels of the batched Laplace step (sm_100a, FP64): eta = A x,
// likelihood Eval1D (value, gradient, Fisher/observed Hessian), the Newton
// right-hand side A^T g - Q x, the log-likelihood / quadratic-form
// reductions of the marginal likelihood and the trace contractions of the
// adjoint. One problem (theta-point) per blockIdx.y; every reduction uses a
// fixed tree, so results are run-to-run bit-identical.
//
// Reference:
//   likelihoods            crates/inla_stats/src/inference.rs:170-311, 1641-1664
//   Newton system          crates/inla_math/src/ldlt.rs:373-453, design.rs:52-139
//   mlik                   crates/inla_stats/src/inference.rs:953-972
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "likelihood.cuh"

namespace inla {
namespace {  // each including translation unit gets its own copies of the kernels

// eta[b][i] = sum_a A[i, col] x[b][col]  (A in CSR; acp == nullptr => identity)
__global__ void k_spmv_a(int64_t nobs, int n, const int64_t* __restrict__ acp, const int* __restrict__ aci,
                         const double* __restrict__ av, const double* __restrict__ x, double* __restrict__ eta) {
  const int b = blockIdx.y;
  const double* xb = x + (int64_t)b * n;
  double* eb = eta + (int64_t)b * nobs;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nobs; i += (int64_t)gridDim.x * blockDim.x) {
    if (!acp) {
      eb[i] = xb[i];
      continue;
    }
    double s = 0.0;
    for (int64_t a = acp[i]; a < acp[i + 1]; ++a) s += av[a] * xb[aci[a]];
    eb[i] = s;
  }
}

// logp/grad/w(=-hess)/dw per observation; bad[b] |= 1 on an invalid evaluation,
// 2 on a non-finite log-likelihood.
__global__ void k_eval_lik(int fam, int64_t nobs, const double* __restrict__ eta, const double* __restrict__ y,
                           const double* __restrict__ p1, const double* __restrict__ p2,
                           const double* __restrict__ p1scale, double* __restrict__ logp, double* __restrict__ grad,
                           double* __restrict__ w, double* __restrict__ dw, int* __restrict__ bad) {
  const int b = blockIdx.y;
  const double sc = p1scale ? p1scale[b] : 1.0;
  int flag = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nobs; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t o = (int64_t)b * nobs + i;
    double lp = 0, g = 0, h = 0, d = 0;
    const double q1 = (p1 ? p1[i] : 1.0) * sc;
    if (d_eval_lik(fam, eta[o], y[i], q1, p2 ? p2[i] : 1.0, lp, g, h, d)) {
      flag |= 1;
      lp = NAN;
    } else if (!isfinite(lp)) {
      flag |= 2;
    }
    logp[o] = lp;
    grad[o] = g;
    w[o] = -h;
    if (dw) dw[o] = d;
  }
  if (flag) atomicOr(bad + b, flag);
}

// rhs[b][j] = sum_a A[a, j] g[b][a] - (Q x)[b][j]; Q values = sum_t coef[b][t] comp[t][p]
// on the full symmetric pattern (column j of Q = row j). A^T in CSR (atp, ati, atv).
__global__ void k_newton_rhs(int n, int ncomp, const int64_t* __restrict__ qcp, const int* __restrict__ qri,
                             const double* __restrict__ comp, int64_t nnz, const double* __restrict__ coef,
                             const int64_t* __restrict__ atp, const int* __restrict__ ati,
                             const double* __restrict__ atv, int64_t nobs, const double* __restrict__ g,
                             const double* __restrict__ x, double* __restrict__ rhs) {
  const int b = blockIdx.y;
  const double* xb = x + (int64_t)b * n;
  const double* gb = g + (int64_t)b * nobs;
  const double* cb = coef + (int64_t)b * ncomp;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double s = 0.0;
    if (atp) {
      for (int64_t a = atp[j]; a < atp[j + 1]; ++a) s += atv[a] * gb[ati[a]];
    } else {
      s = gb[j];
    }
    double qx = 0.0;
    for (int64_t p = qcp[j]; p < qcp[j + 1]; ++p) {
      double v = 0.0;
      for (int t = 0; t < ncomp; ++t) v += cb[t] * comp[(int64_t)t * nnz + p];
      qx += v * xb[qri[p]];
    }
    rhs[(int64_t)b * n + j] = s - qx;
  }
}

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

// Newton update with the reference's step cap: x_trial = x + alpha step.
__global__ void k_axpy_trial(int n, const double* __restrict__ x, const double* __restrict__ step,
                             const double* __restrict__ alpha, double* __restrict__ xt) {
  const int b = blockIdx.y;
  const double a = alpha[b];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const int64_t o = (int64_t)b * n + j;
    xt[o] = x[o] + a * step[o];
  }
}

// Per-problem block reductions (one CTA per problem, fixed tree).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}
template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
  red[threadIdx.x] = v;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  double r = red[0];
  __syncthreads();
  return r;
}

// Multi-CTA reductions with a fixed summation order. A kernel launched on a
// grid (nchunk, B) of 256-thread CTAs reduces NQ per-thread values over its
// CTA (fixed tree), stores them at part[((b * nchunk) + chunk) * NQ + q], and the
// CTA that takes the last ticket of problem b adds the partials in chunk
// order and writes out[b * ostride + q] for q < nlo and, when has_last,
// v[NQ - 1] to out[b * ostride + last_off]; it then resets the ticket.
constexpr int kRedChunk = 2048;  // elements per CTA (256 threads x 8)
__device__ __forceinline__ double block_sum256(double v, double* red) { return block_sum<256>(v, red); }

template <int NQ>
__device__ __forceinline__ void grid_reduce_store(const double (&v)[NQ], int nlo, bool has_last, double* part,
                                                  unsigned* ticket, double* out, int64_t ostride, int last_off) {
  __shared__ double red[256];
  __shared__ bool last;
  const int b = blockIdx.y, nch = gridDim.x;
  double* pb = part + ((int64_t)b * nch) * NQ;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    if (q < nlo || (has_last && q == NQ - 1)) {
      const double sq = block_sum256(v[q], red);
      if (threadIdx.x == 0) pb[(int64_t)blockIdx.x * NQ + q] = sq;
    }
  }
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(&ticket[b], 1u) == (unsigned)(nch - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    if (q < nlo || (has_last && q == NQ - 1)) {
      double a = 0.0;
      for (int c = threadIdx.x; c < nch; c += 256) a += __ldcg(pb + (int64_t)c * NQ + q);
      const double sq = block_sum256(a, red);
      if (threadIdx.x == 0) out[(int64_t)b * ostride + (q < nlo ? q : last_off)] = sq;
    }
  }
  if (threadIdx.x == 0) ticket[b] = 0u;
}

// sum_i v[b][i] -> out[b]
__global__ void __launch_bounds__(256) k_row_sum_g(int64_t len, const double* __restrict__ v, double* part,
                                                   unsigned* ticket, double* __restrict__ out) {
  const int b = blockIdx.y;
  double a[1] = {0.0};
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int64_t i = (int64_t)blockIdx.x * kRedChunk + threadIdx.x + 256 * u;
    if (i < len) a[0] += v[(int64_t)b * len + i];
  }
  grid_reduce_store<1>(a, 1, false, part, ticket, out, 1, 0);
}

// d loglik / d log(scale) for Gaussian precision scaling: sum_i (1/2 - w_i r_i^2 / 2)
__global__ void __launch_bounds__(256) k_gauss_dll_g(int64_t nobs, const double* __restrict__ eta,
                                                     const double* __restrict__ y, const double* __restrict__ w,
                                                     double* part, unsigned* ticket, double* __restrict__ out) {
  const int b = blockIdx.y;
  double a[1] = {0.0};
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int64_t i = (int64_t)blockIdx.x * kRedChunk + threadIdx.x + 256 * u;
    if (i < nobs) {
      const double r = eta[(int64_t)b * nobs + i] - y[i];
      a[0] += 0.5 - 0.5 * w[(int64_t)b * nobs + i] * r * r;
    }
  }
  grid_reduce_store<1>(a, 1, false, part, ticket, out, 1, 0);
}

// x^T M_t x (t < ncomp) and x^T Q x = sum_t coef_t x^T M_t x, columns in chunks of
// kColChunk: out[b][0] = x^T Q x, out[b][1+t] = x^T M_t x. With z != nullptr the
// bilinear forms z^T M_t x go to out[b][t] (no total).
constexpr int kColChunk = 1024;  // 256 threads x 4 columns
__global__ void __launch_bounds__(256) k_quad_forms_g(int n, int ncomp, const int64_t* __restrict__ qcp,
                                                      const int* __restrict__ qri, const double* __restrict__ comp,
                                                      int64_t nnz, const double* __restrict__ coef,
                                                      const double* __restrict__ z, const double* __restrict__ x,
                                                      double* part, unsigned* ticket, double* __restrict__ out) {
  const int b = blockIdx.y;
  const double* xb = x + (int64_t)b * n;
  const double* zb = z ? z + (int64_t)b * n : xb;
  double acc[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) acc[t] = 0.0;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int j = blockIdx.x * kColChunk + threadIdx.x + 256 * u;
    if (j >= n) continue;
    const double zj = zb[j];
    for (int64_t p = qcp[j]; p < qcp[j + 1]; ++p) {
      const double zx = zj * xb[qri[p]];
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (t < ncomp) acc[t] += comp[(int64_t)t * nnz + p] * zx;
    }
  }
  const int nc = ncomp < 8 ? ncomp : 8;
  if (z) {
    grid_reduce_store<9>(acc, nc, false, part, ticket, out, ncomp + 1, 0);
  } else {
#pragma unroll
    for (int t = 0; t < 8; ++t)
      if (t < nc) acc[8] += coef[(int64_t)b * ncomp + t] * acc[t];
    grid_reduce_store<9>(acc, nc, true, part, ticket, out + 1, ncomp + 1, -1);
  }
}

// Trace contractions of a selected inverse given on the full pattern (both
// triangles): out[b][t] = sum_p sigma[b][p] comp[t][p] (= tr(Sigma M_t)) and
// out[b][ncomp] = sum_p sigma[b][p] sum_q w2[b][obs_q] prod_q (= tr(Sigma A^T diag(w2) A)).
__global__ void __launch_bounds__(256) k_trace_contract_g(int64_t nnz, int ncomp, const double* __restrict__ comp,
                                                          const double* __restrict__ sigma,
                                                          const int* __restrict__ cptr, const int* __restrict__ cobs,
                                                          const double* __restrict__ cprod,
                                                          const double* __restrict__ w2, int64_t nobs, double* part,
                                                          unsigned* ticket, double* __restrict__ out) {
  const int b = blockIdx.y;
  const double* sb = sigma + (int64_t)b * nnz;
  double acc[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) acc[t] = 0.0;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int64_t p = (int64_t)blockIdx.x * kRedChunk + threadIdx.x + 256 * u;
    if (p >= nnz) continue;
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
  const int nc = ncomp < 8 ? ncomp : 8;
  grid_reduce_store<9>(acc, nc, true, part, ticket, out, ncomp + 1, ncomp);
}

// out[b] = {max|step|, all finite ? 1 : 0}
template <int NT>
__global__ void __launch_bounds__(NT) k_step_stats(int n, int64_t stride, const double* __restrict__ step,
                                                  double* __restrict__ out) {
  __shared__ double red[NT];
  const int b = blockIdx.x;
  double mx = 0.0, fin = 1.0;
  for (int j = threadIdx.x; j < n; j += NT) {
    double s = step[(int64_t)b * stride + j];
    if (!isfinite(s)) fin = 0.0;
    else mx = fmax(mx, fabs(s));
  }
  mx = block_max<NT>(mx, red);
  fin = -block_max<NT>(-fin, red);
  if (threadIdx.x == 0) {
    out[2 * b] = mx;
    out[2 * b + 1] = fin;
  }
}

// max |a - b| over the first n entries per problem (Newton convergence on the accepted,
// projected trial point)
template <int NT>
__global__ void __launch_bounds__(NT) k_max_abs_diff(int n, int64_t stride, const double* __restrict__ a,
                                                    const double* __restrict__ c, double* __restrict__ out) {
  __shared__ double red[NT];
  const int b = blockIdx.x;
  double mx = 0.0;
  for (int j = threadIdx.x; j < n; j += NT)
    mx = fmax(mx, fabs(a[(int64_t)b * stride + j] - c[(int64_t)b * stride + j]));
  mx = block_max<NT>(mx, red);
  if (threadIdx.x == 0) out[b] = mx;
}

// Constraint residual r[b][a] = (C x_b)_a - e_a, one CTA per (row a, problem b), fixed
// summation order (constraints.rs:324-333). C in CSR: rows of ConstraintSpec.a without zeros.
// With set_border it instead sets the border entry x[b][n + a] = border * (C x_b)_a of a
// bordered system: border = kappa gives the multiplier kappa C x (M x = [Q x + kappa C^T C x;
// 0]), border = 0 clears it.
template <int NT>
__global__ void __launch_bounds__(NT) k_constr_resid(int n, int64_t stride, int k, const int64_t* __restrict__ crp,
                                                    const int* __restrict__ cci, const double* __restrict__ cv,
                                                    const double* __restrict__ ce, int set_border, double border,
                                                    double* __restrict__ x, double* __restrict__ r) {
  __shared__ double red[NT];
  const int a = blockIdx.x, b = blockIdx.y;
  double* xb = x + (int64_t)b * stride;
  double s = 0.0;
  for (int64_t p = crp[a] + threadIdx.x; p < crp[a + 1]; p += NT) s += cv[p] * xb[cci[p]];
  s = block_sum<NT>(s, red);
  if (threadIdx.x == 0) {
    if (set_border) xb[n + a] = border * s;
    else r[(int64_t)b * k + a] = s - ce[a];
  }
}

// x_b <- x_b - C^T lambda_b, lambda_b = (C C^T)^-1 r_b (constraints.rs:343-351). Every CTA
// forms lambda_b in shared memory (k doubles) from the precomputed inverse; C^T in CSR.
__global__ void k_constr_apply(int n, int64_t stride, int k, const int64_t* __restrict__ ctp,
                               const int* __restrict__ cta, const double* __restrict__ ctv,
                               const double* __restrict__ ginv, const double* __restrict__ r,
                               double* __restrict__ x) {
  extern __shared__ double lam[];
  const int b = blockIdx.y;
  const double* rb = r + (int64_t)b * k;
  for (int a = threadIdx.x; a < k; a += blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < k; ++j) s += ginv[(int64_t)a * k + j] * rb[j];
    lam[a] = s;
  }
  __syncthreads();
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double corr = 0.0;
    for (int64_t p = ctp[c]; p < ctp[c + 1]; ++p) corr += ctv[p] * lam[cta[p]];
    x[(int64_t)b * stride + c] -= corr;
  }
}

// Mirror lower-entry values onto the upper entries of the full pattern:
// out[b][p] = buf[b][spos_full[p]] (spos_full maps every entry to its lower twin).
__global__ void k_pattern_full(int64_t nnz, const int64_t* __restrict__ spos_full, const double* __restrict__ buf,
                               int64_t fstride, double* __restrict__ out) {
  const int b = blockIdx.y;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x)
    out[(int64_t)b * nnz + p] = buf[(int64_t)b * fstride + spos_full[p]];
}

// Exact predictor variances v_i = a_i^T Sigma a_i from Sigma on the pattern
// (A row pairs -> pattern positions in opos).
__global__ void k_predictor_var(int64_t nobs, const int64_t* __restrict__ acp, const double* __restrict__ av,
                                const int64_t* __restrict__ oppos, const int64_t* __restrict__ opptr,
                                const double* __restrict__ sigma, int64_t nnz, double* __restrict__ v) {
  const int b = blockIdx.y;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nobs; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a0 = acp[i], na = acp[i + 1] - a0;
    double s = 0.0;
    int64_t q = opptr[i];
    for (int64_t a = 0; a < na; ++a)
      for (int64_t c = 0; c < na; ++c, ++q) s += av[a0 + a] * av[a0 + c] * sigma[(int64_t)b * nnz + oppos[q]];
    v[(int64_t)b * nobs + i] = s;
  }
}

}  // namespace
}  // namespace inla
