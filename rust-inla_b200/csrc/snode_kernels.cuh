// CUDA kernels (sm_100a, FP64) for the multifrontal supernodal LDL^T, its
// triangular solves, the log-determinant and the supernodal Takahashi
// selected inverse.
//
// Storage ("front layout"): supernode s owns a dense m_s x m_s column-major
// block at offset fptr[s] inside one buffer per problem. Its first k_s
// columns are the L panel (unit-lower L below the diagonal, D on the
// diagonal); the trailing r_s x r_s lower block holds the Schur-complement
// update that the parent pulls (factorization), or Sigma restricted to the
// supernode's below-rows (selected inversion). Children are always
// assembled by the parent in a fixed order (deterministic, no atomics).
//
// Reference recurrences being computed:
//   LDL^T without pivoting, D gate |D| < 1e-14 or non-finite => Singular
//       (crates/inla_math/src/sparse_ldlt.rs:104-149)
//   log|Q| = sum log|D_i|            (crates/inla_math/src/ldlt.rs:65-67)
//   Takahashi: S_ij = -sum_{l>j} L_lj S_li (i>j), S_jj = 1/D_j - sum_{l>j} L_lj S_lj
//                                      (crates/inla_math/src/sparse_ldlt.rs:366-432)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dense_ldlt.cuh"
#include "devsym.hpp"

namespace inla {
// Internal linkage: every translation unit that launches these kernels owns
// its own copy (no cross-file kernel symbols).
namespace {

__device__ __forceinline__ int sn_k(const DevSym& S, int s) { return S.first[s + 1] - S.first[s]; }
__device__ __forceinline__ int sn_m(const DevSym& S, int s) { return S.rowptr[s + 1] - S.rowptr[s]; }

// ---------------------------------------------------------------------------
// value fill: every panel entry written exactly once (value or zero)
// ---------------------------------------------------------------------------

// The compact panel numbering (entry e of supernode s at lptr[s] + col * m + row)
// is cut into chunks of kFillChunk entries, one CTA each; csn[c] is the
// supernode holding the first entry of chunk c (csn[nchunks] = ns - 1). Within
// its front the entry sits at fptr[s] + (e - lptr[s]) (panel columns first).
constexpr int kFillChunk = 2048;  // 256 threads x 8 entries

__device__ __forceinline__ int fill_find(const DevSym& S, int lo, int hi, int64_t e) {
  // largest s in [lo, hi] with lptr[s] <= e
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (S.lptr[mid] <= e) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// vals: [B][nnz] full-CSC values; pmap: compact panel index -> input entry or -1.
__global__ void __launch_bounds__(256) k_fill_panels(DevSym S, const int* __restrict__ csn, int64_t ntot,
                                                     const int* __restrict__ pmap, const double* __restrict__ vals,
                                                     int64_t vstride, double* __restrict__ F, int64_t fstride) {
  const int b = blockIdx.y;
  const int lo = csn[blockIdx.x], hi = csn[blockIdx.x + 1];
  const double* v = vals + (int64_t)b * vstride;
  double* Fb = F + (int64_t)b * fstride;
  int src[8];
  int64_t dst[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int64_t e = (int64_t)blockIdx.x * kFillChunk + threadIdx.x + 256 * u;
    src[u] = -1;
    dst[u] = -1;
    if (e < ntot) {
      const int s = fill_find(S, lo, hi, e);
      src[u] = pmap[e];
      dst[u] = S.fptr[s] + (e - S.lptr[s]);
    }
  }
#pragma unroll
  for (int u = 0; u < 8; ++u)
    if (dst[u] >= 0) Fb[dst[u]] = src[u] >= 0 ? v[src[u]] : 0.0;
}

// Component model: value(p) = sum_t coef[b][t] * comp[t][p] + sum_q w[b][obs_q] * prod_q
// over the observation contributions of entry p (A^T diag(w) A on the pattern).
// diag_add is added on diagonal entries (pdiag[p] != 0), e.g. the 1e-12 jitter of
// the prior log-determinant (inference.rs:831-837). Problems [0, nprior) are prior
// precisions (diag_add, no observation term); problems [nprior, B) add
// diag_add_post and take their weights from w + (b - nprior) * wstride (if w).
// One thread per panel entry fills it for all B problems, so the entry's pattern
// data is read once. With pseg (independent models held block-diagonally) the
// coefficients are per model: coef[(b * nseg + pseg[p]) * ncomp + t].
constexpr int kFillModelChunk = 512;  // 256 threads x 2 entries
__global__ void __launch_bounds__(256) k_fill_panels_model(DevSym S, const int* __restrict__ csn, int64_t ntot,
                                                           const int* __restrict__ pmap, int ncomp,
                                                           const double* __restrict__ comp, int64_t nnz,
                                                           const double* __restrict__ coef, double diag_add,
                                                           const unsigned char* __restrict__ pdiag,
                                                           const int* __restrict__ cptr, const int* __restrict__ cobs,
                                                           const double* __restrict__ cprod,
                                                           const double* __restrict__ w, int64_t wstride, int B,
                                                           int nprior, double diag_add_post,
                                                           const int* __restrict__ pseg, int nseg,
                                                           double* __restrict__ F, int64_t fstride,
                                                           const int* __restrict__ fseg = nullptr,
                                                           const unsigned char* __restrict__ active = nullptr) {
  const int lo = csn[blockIdx.x], hi = csn[blockIdx.x + 1];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int64_t e = (int64_t)blockIdx.x * kFillModelChunk + threadIdx.x + 256 * u;
    if (e >= ntot) continue;
    const int s = fill_find(S, lo, hi, e);
    const int p = pmap[e];
    const int64_t dst = S.fptr[s] + (e - S.lptr[s]);
    // with `active` ([B][nseg]), the fronts of inactive (problem, model) pairs keep their
    // last factor: they are neither filled nor factorized
    const int fs = active ? fseg[s] : 0;
    if (p < 0) {
      for (int b = 0; b < B; ++b)
        if (!active || active[(int64_t)b * nseg + fs]) F[(int64_t)b * fstride + dst] = 0.0;
      continue;
    }
    double cv[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) cv[t] = t < ncomp ? comp[(int64_t)t * nnz + p] : 0.0;
    const bool isdiag = pdiag[p] != 0;
    const int q0 = cptr[p], q1 = cptr[p + 1];
    const int sg = pseg ? pseg[p] : 0;
    for (int b = 0; b < B; ++b) {
      if (active && !active[(int64_t)b * nseg + fs]) continue;
      const double* cb = coef + ((int64_t)b * nseg + sg) * ncomp;
      double v = isdiag ? (b < nprior ? diag_add : diag_add_post) : 0.0;
#pragma unroll
      for (int t = 0; t < 8; ++t)
        if (t < ncomp) v += cb[t] * cv[t];
      if (w && b >= nprior) {
        const double* wb = w + (int64_t)(b - nprior) * wstride;
        double acc = 0.0;
        // design.rs:100-115: observations with a zero or non-finite weight are skipped
        for (int q = q0; q < q1; ++q) {
          const double wq = wb[cobs[q]];
          if (wq != 0.0 && isfinite(wq)) acc += wq * cprod[q];
        }
        v += acc;
      }
      F[(int64_t)b * fstride + dst] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// small fronts: whole front in shared memory, one CTA per (supernode, problem)
// ---------------------------------------------------------------------------

// Shared memory of k_factor_small for fronts of up to m rows (bytes).
__host__ __device__ constexpr int small_factor_smem(int m) {
  return (m * dense_ld(m) + 16 * dense_uld(m) + kDenseScratch) * 8;
}

// One CTA per (front, problem): the front in shared memory (leading dimension
// dense_ld(m)), the children's updates added in fixed order, then the blocked
// partial LDL^T of the k pivot columns (cta_ldlt).
template <int NT>
__device__ __forceinline__ void factor_small_body(const DevSym& S, int s, int b, double* __restrict__ F,
                                                  int64_t fstride, double* sm) {
  if (front_skipped(S, s, b)) return;
  double* Fb = F + (int64_t)b * fstride;
  const int k = sn_k(S, s), m = sn_m(S, s);
  const int lda = dense_ld(m), uld = dense_uld(m);
  double* A = sm;
  double* U = A + m * lda;
  double* ws = U + 16 * uld;
  int* rs = reinterpret_cast<int*>(U);  // child relative indices (U is free until the factorization)
  double* Fs = Fb + S.fptr[s];
  const int mm = m * m;
  for (int e = threadIdx.x; e < mm; e += NT) {
    const int col = e / m, row = e - col * m;
    if (col < k) cp_async8(&A[row + col * lda], Fs + e);
    else A[row + col * lda] = 0.0;
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  for (int q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
    const int c = S.child_list[q];
    const int kc = sn_k(S, c), mc = sn_m(S, c), rc = mc - kc;
    const double* Uc = Fb + S.fptr[c] + (int64_t)kc * mc + kc;
    const int* relc = S.relx + S.rowptr[c] + kc;
    for (int t = threadIdx.x; t < rc; t += NT) rs[t] = relc[t];
    __syncthreads();
    const int rr = rc * rc;
    int e = threadIdx.x;
    for (; e + 3 * NT < rr; e += 4 * NT) {
      double v[4];
      int dst[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int ee = e + u * NT;
        const int jj = ee / rc, ii = ee - jj * rc;
        const bool ok = ii >= jj;
        v[u] = ok ? Uc[ii + (int64_t)jj * mc] : 0.0;
        dst[u] = ok ? rs[ii] + rs[jj] * lda : -1;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (dst[u] >= 0) A[dst[u]] += v[u];
    }
    for (; e < rr; e += NT) {
      const int jj = e / rc, ii = e - jj * rc;
      if (ii >= jj) A[rs[ii] + rs[jj] * lda] += Uc[ii + (int64_t)jj * mc];
    }
    __syncthreads();
  }
  cta_ldlt<false>(A, lda, m, k, nullptr, 0, U, uld, ws);
  for (int e = threadIdx.x; e < mm; e += NT) {
    const int col = e / m, row = e - col * m;
    if (col < k || row >= col) Fs[e] = A[row + col * lda];
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_factor_small(DevSym S, const int* __restrict__ list,
                                                     double* __restrict__ F, int64_t fstride) {
  extern __shared__ double sm[];
  factor_small_body<NT>(S, list[blockIdx.x], blockIdx.y, F, fstride, sm);
}

// ---------------------------------------------------------------------------
// tiny fronts (m <= kTinyM rows): one warp per (front, problem), kTinyWarps fronts
// per CTA. The front is staged in the warp's shared-memory slice (column-major,
// leading dimension kTinyLd), the children's updates are added in fixed order,
// then the k pivot steps run right-looking with lane i owning row i:
//   u_i = A[i][t], A[i][t] = u_i / d_t (i > t), A[i][j] -= (u_i / d_t) u_j for t < j <= i,
// leaving unit L below the diagonal, D on it and the Schur complement in the
// trailing block -- the layout k_factor_small leaves. Fronts this small give a
// CTA-wide blocked factorization almost nothing to share among its warps.
// ---------------------------------------------------------------------------
constexpr int kTinyM = 32;
constexpr int kTinyWarps = 4;
constexpr int kTinyLd = kTinyM + 1;

// One warp: front s of problem b in the warp's shared slices A [kTinyM x kTinyLd], U [kTinyM]
// and R [kTinyM] (ints). Only warp-level synchronization inside.
__device__ __forceinline__ void factor_tiny_warp(const DevSym& S, int s, int b, double* __restrict__ F,
                                                 int64_t fstride, double* A, double* U, int* R) {
  if (front_skipped(S, s, b)) return;
  const int lane = threadIdx.x & 31;
  double* Fb = F + (int64_t)b * fstride;
  const int k = sn_k(S, s), m = sn_m(S, s);
  double* Fs = Fb + S.fptr[s];
  const int mm = m * m;
  for (int e = lane; e < mm; e += 32) {
    const int col = e / m, row = e - col * m;
    A[row + col * kTinyLd] = col < k ? Fs[e] : 0.0;
  }
  __syncwarp();
  for (int q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
    const int c = S.child_list[q];
    const int kc = sn_k(S, c), mc = sn_m(S, c), rc = mc - kc;
    const double* Uc = Fb + S.fptr[c] + (int64_t)kc * mc + kc;
    if (lane < rc) R[lane] = S.relx[S.rowptr[c] + kc + lane];
    __syncwarp();
    for (int e = lane; e < rc * rc; e += 32) {
      const int jj = e / rc, ii = e - jj * rc;
      if (ii >= jj) A[R[ii] + R[jj] * kTinyLd] += Uc[ii + (int64_t)jj * mc];
    }
    __syncwarp();
  }
  for (int t = 0; t < k; ++t) {
    const double d = A[t + t * kTinyLd];
    const bool below = lane > t && lane < m;
    const double u = below ? A[lane + t * kTinyLd] : 0.0;
    U[lane] = u;
    __syncwarp();
    if (below) {
      const double l = u / d;
      A[lane + t * kTinyLd] = l;
      for (int j = t + 1; j <= lane; ++j) A[lane + j * kTinyLd] -= l * U[j];
    }
    __syncwarp();
  }
  for (int e = lane; e < mm; e += 32) {
    const int col = e / m, row = e - col * m;
    if (col < k || row >= col) Fs[e] = A[row + col * kTinyLd];
  }
}

__global__ void __launch_bounds__(32 * kTinyWarps) k_factor_tiny(DevSym S, const int* __restrict__ list, int nlist,
                                                                 double* __restrict__ F, int64_t fstride) {
  __shared__ double sA[kTinyWarps][kTinyM * kTinyLd];
  __shared__ double sU[kTinyWarps][kTinyM];
  __shared__ int sR[kTinyWarps][kTinyM];
  const int warp = threadIdx.x >> 5;
  const int idx = blockIdx.x * kTinyWarps + warp;
  if (idx >= nlist) return;  // the whole warp leaves; only warp-level synchronization follows
  factor_tiny_warp(S, list[idx], blockIdx.y, F, fstride, sA[warp], sU[warp], sR[warp]);
}

// ---------------------------------------------------------------------------
// large fronts: blocked right-looking partial LDL^T in global memory
// ---------------------------------------------------------------------------

constexpr int kNB = 32;       // block-column width

// Unblocked LDL^T of the diagonal block [j0, j0+w) of every listed front.
__global__ void k_diag_large(DevSym S, const int* __restrict__ list, int j0, double* __restrict__ F,
                             int64_t fstride) {
  __shared__ double sm[kNB * kNB];
  const int s = list[blockIdx.x], b = blockIdx.y;
  const int k = sn_k(S, s), m = sn_m(S, s);
  if (j0 >= k) return;
  const int w = min(kNB, k - j0);
  double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* D0 = Fs + j0 + (int64_t)j0 * m;
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    int c = e / w, r = e - c * w;
    sm[r + c * kNB] = D0[r + (int64_t)c * m];
  }
  __syncthreads();
  for (int j = 0; j < w; ++j) {
    const double dinv = 1.0 / sm[j + j * kNB];
    const int ww = w - j - 1;
    for (int e = threadIdx.x; e < ww * ww; e += blockDim.x) {
      int tt = e / ww, ii = e - tt * ww;
      if (ii >= tt) sm[(j + 1 + ii) + (j + 1 + tt) * kNB] -= sm[j + 1 + ii + j * kNB] * sm[j + 1 + tt + j * kNB] * dinv;
    }
    __syncthreads();
    for (int i = j + 1 + threadIdx.x; i < w; i += blockDim.x) sm[i + j * kNB] *= dinv;
    __syncthreads();
  }
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    int c = e / w, r = e - c * w;
    if (r >= c) D0[r + (int64_t)c * m] = sm[r + c * kNB];
  }
}

// Rows below the diagonal block: L_i = F_i L11^-T D^-1 (one thread per row).
constexpr int kTrsmRows = 128;
__global__ void __launch_bounds__(kTrsmRows) k_trsm_large(DevSym S, const int* __restrict__ list, int j0,
                                                          double* __restrict__ F, int64_t fstride) {
  __shared__ double dl[kNB * kNB];  // dl[t*kNB+u] = d_u * L_tu (u < t)
  __shared__ double dinv[kNB];
  const int s = list[blockIdx.x], b = blockIdx.y;
  const int k = sn_k(S, s), m = sn_m(S, s);
  if (j0 >= k) return;
  const int w = min(kNB, k - j0);
  const int r0 = j0 + w + blockIdx.z * kTrsmRows;
  if (r0 >= m) return;
  double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  const double* D0 = Fs + j0 + (int64_t)j0 * m;
  for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
    int t = e / w, u = e - t * w;
    dl[t * kNB + u] = (u < t) ? D0[u + (int64_t)u * m] * D0[t + (int64_t)u * m] : 0.0;
  }
  for (int t = threadIdx.x; t < w; t += blockDim.x) dinv[t] = 1.0 / D0[t + (int64_t)t * m];
  __syncthreads();
  const int i = r0 + threadIdx.x;
  if (i >= m) return;
  double x[kNB];
  double* Fi = Fs + i + (int64_t)j0 * m;
#pragma unroll
  for (int t = 0; t < kNB; ++t) {
    if (t < w) {
      double y = Fi[(int64_t)t * m];
#pragma unroll
      for (int u = 0; u < kNB; ++u)
        if (u < t) y -= x[u] * dl[t * kNB + u];
      x[t] = y * dinv[t];
      Fi[(int64_t)t * m] = x[t];
    }
  }
}

// Trailing update F[i,j] -= sum_t L[i,t] d_t L[j,t] over the block [j0,j0+w),
// for the lower triangle of the trailing region [c, m), 64x64 tiles, FP64
// tensor-core tiles (mma.sync m8n8k4).
constexpr int kUT = 64;
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(128) k_update_large(DevSym S, const int* __restrict__ list, int j0,
                                                     double* __restrict__ F, int64_t fstride) {
  __shared__ double As[kNB][kUT + 1];  // As[t][i] = L[I0+i, j0+t]
  __shared__ double Bs[kNB][kUT + 1];  // Bs[t][j] = d_t L[J0+j, j0+t]
  const int s = list[blockIdx.x], b = blockIdx.y;
  const int k = sn_k(S, s), m = sn_m(S, s);
  if (j0 >= k) return;
  const int w = min(kNB, k - j0);
  const int c = j0 + w;
  const int T = m - c;
  if (T <= 0) return;
  const int nt = (T + kUT - 1) / kUT;
  const int tile = blockIdx.z;
  if (tile >= nt * (nt + 1) / 2) return;
  // tile -> (I,J), I >= J, column-major over the lower triangle of tiles
  int J = 0, rem = tile;
  while (rem >= nt - J) { rem -= nt - J; ++J; }
  const int I = J + rem;
  const int I0 = c + I * kUT, J0 = c + J * kUT;
  double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  const double* Lb = Fs + (int64_t)j0 * m;
  for (int e = threadIdx.x; e < kNB * kUT; e += blockDim.x) {
    int t = e / kUT, i = e - t * kUT;
    double a = 0.0, bb = 0.0;
    if (t < w) {
      if (I0 + i < m) a = Lb[I0 + i + (int64_t)t * m];
      if (J0 + i < m) bb = Lb[J0 + i + (int64_t)t * m] * Lb[j0 + t + (int64_t)t * m];
    }
    As[t][i] = a;
    Bs[t][i] = bb;
  }
  __syncthreads();
  // 4 warps, each a 32x32 quadrant made of 4x4 mma tiles of 8x8
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wi = (warp & 1) * 32, wj = (warp >> 1) * 32;
  const int g = lane >> 2, tg = lane & 3;
  double acc[4][4][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int bq = 0; bq < 4; ++bq) acc[a][bq][0] = acc[a][bq][1] = 0.0;
#pragma unroll
  for (int t0 = 0; t0 < kNB; t0 += 4) {
    double af[4], bf[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) af[a] = As[t0 + tg][wi + a * 8 + g];
#pragma unroll
    for (int bq = 0; bq < 4; ++bq) bf[bq] = Bs[t0 + tg][wj + bq * 8 + g];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int bq = 0; bq < 4; ++bq) dmma_8x8x4(acc[a][bq][0], acc[a][bq][1], af[a], bf[bq]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int bq = 0; bq < 4; ++bq)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = I0 + wi + a * 8 + g;
        const int j = J0 + wj + bq * 8 + tg * 2 + h;
        if (i < m && j < m && i >= j) Fs[i + (int64_t)j * m] -= acc[a][bq][h];
      }
}

// ---------------------------------------------------------------------------
// log-determinant + singularity gate (one CTA per problem, fixed reduction tree)
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT) k_logdet(DevSym S, const double* __restrict__ F, int64_t fstride,
                                               double* __restrict__ logdet, int* __restrict__ status) {
  __shared__ double red[NT];
  __shared__ int bad[NT];
  const int b = blockIdx.x;
  const double* Fb = F + (int64_t)b * fstride;
  double acc = 0.0;
  int flag = 0;
  for (int j = threadIdx.x; j < S.n; j += NT) {
    double d = Fb[S.dpos[j]];
    double ad = fabs(d);
    if (!isfinite(d)) flag |= kStatusNotFinite;
    else if (ad < 1e-14) flag |= kStatusSingular;
    acc += log(ad);
  }
  red[threadIdx.x] = acc;
  bad[threadIdx.x] = flag;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[threadIdx.x] += red[threadIdx.x + o];
      bad[threadIdx.x] |= bad[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    logdet[b] = red[0];
    status[b] = bad[0];
  }
}

// log|Q_b| = sum_j log|d_j| and the status word, over chunks of kLogdetChunk
// pivots per CTA. Each CTA writes its partial; the CTA that takes the last
// ticket of problem b adds the partials in chunk order (deterministic), writes
// the result and resets the ticket for the next launch.
constexpr int kLogdetChunk = 2048;  // 256 threads x 8 pivots
__global__ void __launch_bounds__(256) k_logdet_chunks(DevSym S, const double* __restrict__ F, int64_t fstride,
                                                       double* __restrict__ part, int* __restrict__ pflag,
                                                       unsigned* __restrict__ ticket, double* __restrict__ logdet,
                                                       int* __restrict__ status,
                                                       const int* __restrict__ sched_err = nullptr) {
  __shared__ double red[256];
  __shared__ int bad[256];
  __shared__ bool last;
  const int b = blockIdx.y, nch = gridDim.x;
  const double* Fb = F + (int64_t)b * fstride;
  double dv[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int j = blockIdx.x * kLogdetChunk + threadIdx.x + 256 * u;
    dv[u] = j < S.n ? Fb[S.dpos[j]] : 1.0;
  }
  double acc = 0.0;
  int flag = 0;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const double ad = fabs(dv[u]);
    if (!isfinite(dv[u])) flag |= kStatusNotFinite;
    else if (ad < 1e-14) flag |= kStatusSingular;
    acc += log(ad);
  }
  red[threadIdx.x] = acc;
  bad[threadIdx.x] = flag;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[threadIdx.x] += red[threadIdx.x + o];
      bad[threadIdx.x] |= bad[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[(int64_t)b * nch + blockIdx.x] = red[0];
    pflag[(int64_t)b * nch + blockIdx.x] = bad[0];
    __threadfence();
    last = atomicAdd(&ticket[b], 1u) == (unsigned)(nch - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double a2 = 0.0;
  int f2 = 0;
  for (int c = threadIdx.x; c < nch; c += 256) {
    a2 += __ldcg(part + (int64_t)b * nch + c);
    f2 |= __ldcg(pflag + (int64_t)b * nch + c);
  }
  red[threadIdx.x] = a2;
  bad[threadIdx.x] = f2;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red[threadIdx.x] += red[threadIdx.x + o];
      bad[threadIdx.x] |= bad[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    logdet[b] = red[0];
    status[b] = bad[0] | ((sched_err && __ldcg(sched_err) != 0) ? kStatusSchedule : 0);
    ticket[b] = 0u;
  }
}

// ---------------------------------------------------------------------------
// triangular solves: forward (bottom-up levels) then backward (top-down)
// xp: [B][n] permuted working vector; ub: [B][sum r] child update vectors
// ---------------------------------------------------------------------------

__global__ void k_permute_in(int n, const int* __restrict__ perm, const double* __restrict__ x,
                             int64_t xstride, double* __restrict__ xp) {
  const int b = blockIdx.y;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    xp[(int64_t)b * n + j] = x[(int64_t)b * xstride + perm[j]];
}
__global__ void k_permute_out(int n, const int* __restrict__ perm, const double* __restrict__ xp,
                              double* __restrict__ x, int64_t xstride) {
  const int b = blockIdx.y;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x)
    x[(int64_t)b * xstride + perm[j]] = xp[(int64_t)b * n + j];
}

template <int NT>
__global__ void __launch_bounds__(NT) k_fwd(DevSym S, const int* __restrict__ list, const double* __restrict__ F,
                                            int64_t fstride, double* __restrict__ xp, double* __restrict__ ub,
                                            int64_t ustride) {
  extern __shared__ double y[];
  const int s = list[blockIdx.x], b = blockIdx.y;
  const int k = sn_k(S, s), m = sn_m(S, s), f = S.first[s];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* xb = xp + (int64_t)b * S.n;
  double* ubb = ub + (int64_t)b * ustride;
  for (int t = threadIdx.x; t < m; t += NT) y[t] = t < k ? xb[f + t] : 0.0;
  __syncthreads();
  for (int q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
    const int c = S.child_list[q];
    const int kc = sn_k(S, c), rc = sn_m(S, c) - kc;
    const int* relc = S.relx + S.rowptr[c] + kc;
    const double* uc = ubb + S.uoff[c];
    for (int t = threadIdx.x; t < rc; t += NT) y[relc[t]] += uc[t];
    __syncthreads();
  }
  for (int j = 0; j < k; ++j) {
    const double yj = y[j];
    const double* Lj = Fs + (int64_t)j * m;
    for (int i = j + 1 + threadIdx.x; i < m; i += NT) y[i] -= Lj[i] * yj;
    __syncthreads();
  }
  for (int t = threadIdx.x; t < m; t += NT) {
    if (t < k) xb[f + t] = y[t] / Fs[t + (int64_t)t * m];
    else ubb[S.uoff[s] + t - k] = y[t];
  }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_bwd(DevSym S, const int* __restrict__ list, const double* __restrict__ F,
                                            int64_t fstride, double* __restrict__ xp) {
  extern __shared__ double x[];
  const int s = list[blockIdx.x], b = blockIdx.y;
  const int k = sn_k(S, s), m = sn_m(S, s), f = S.first[s];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* xb = xp + (int64_t)b * S.n;
  const int* R = S.rows + S.rowptr[s];
  for (int t = threadIdx.x; t < m; t += NT) x[t] = xb[R[t]];
  __syncthreads();
  // x_j -= sum_{i>=k} L_ij x_i for j < k (one warp per column)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = warp; j < k; j += NT / 32) {
    const double* Lj = Fs + (int64_t)j * m;
    double acc = 0.0;
    for (int i = k + lane; i < m; i += 32) acc += Lj[i] * x[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) x[j] -= acc;
  }
  __syncthreads();
  for (int i = k - 1; i > 0; --i) {
    const double xi = x[i];
    for (int j = threadIdx.x; j < i; j += NT) x[j] -= Fs[i + (int64_t)j * m] * xi;
    __syncthreads();
  }
  for (int t = threadIdx.x; t < k; t += NT) xb[f + t] = x[t];
}

// ---------------------------------------------------------------------------
// selected inverse (supernodal Takahashi), top-down levels
// L: factored fronts; Sg: Sigma fronts (same layout)
// ---------------------------------------------------------------------------

// Gather Sigma restricted to the below-rows of s from the parent's Sigma front.
__device__ __forceinline__ double parent_sigma(const double* Sp, int mp, int pi, int pj) {
  return pi >= pj ? Sp[pi + (int64_t)pj * mp] : Sp[pj + (int64_t)pi * mp];
}

// Shared memory of k_selinv_small for fronts of up to m rows and k pivots (bytes).
__host__ __device__ constexpr int small_selinv_smem(int m, int k) {
  return ((m + k) * dense_ld(m) + 16 * dense_uld(m) + 2 * 16 * kLamLd + 64 + 16) * 8;
}

// Selected inverse of a small front, one CTA per (front, problem): Sigma is kept
// with both triangles in shared memory (Sigma_RR gathered from the parent),
// and the pivot columns are processed in 16-column blocks J from right to
// left, A = rows after J:
//   G = Sigma_AA L_AJ,  X = -G L_JJ^-1 = Sigma_AJ,  P = L_AJ^T X,
//   Sigma_JJ = L_JJ^-T (D_J^-1 L_JJ^-1 - P)
// (the block form of the Takahashi recurrence, crates/inla_math/src/sparse_ldlt.rs:366-432),
// with tensor-core tiles for the products and L_JJ^-1 formed by one warp
// while the others compute G.
template <int NT>
__global__ void __launch_bounds__(NT, 4) k_selinv_small(DevSym S, const int* __restrict__ list,
                                                     const double* __restrict__ F, double* __restrict__ Sg,
                                                     int64_t fstride) {
  extern __shared__ double smem[];
  const int s = list[blockIdx.x], b = blockIdx.y;
  const int k = sn_k(S, s), m = sn_m(S, s), r = m - k;
  const int ld = dense_ld(m), uld = dense_uld(m);
  double* Sm = smem;               // Sigma, both triangles: Sm[i + j*ld]
  double* Lp = Sm + m * ld;        // L panel: Lp[i + c*ld], c < k
  double* Xb = Lp + k * ld;        // [16][uld]: G rows of A
  double* lam = Xb + 16 * uld;     // L_JJ^-1 (ld kLamLd)
  double* Pm = lam + 16 * kLamLd;  // P, then M = D^-1 L^-1 - P
  double* xbuf = Pm + 16 * kLamLd; // warp scratch
  double* dv = xbuf + 64;          // 1 / d_j of the block
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* Ss = Sg + (int64_t)b * fstride + S.fptr[s];
  for (int e = threadIdx.x; e < m * k; e += NT) {
    const int c = e / m, i = e - c * m;
    cp_async8(&Lp[i + c * ld], Fs + e);
  }
  cp_async_commit();
  if (r > 0) {
    const int p = S.parent[s];
    const int mp = sn_m(S, p);
    const double* Sp = Sg + (int64_t)b * fstride + S.fptr[p];
    const int* rel = S.relx + S.rowptr[s] + k;
    const int rr = r * r;
    int e = threadIdx.x;
    for (; e + 3 * NT < rr; e += 4 * NT) {
      double v[4];
      int ia[4], ja[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int ee = e + u * NT;
        const int jj = ee / r, ii = ee - jj * r;
        ia[u] = ii >= jj ? ii : -1;
        ja[u] = jj;
        v[u] = ii >= jj ? parent_sigma(Sp, mp, rel[ii], rel[jj]) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (ia[u] >= 0) {
          Sm[(k + ia[u]) + (k + ja[u]) * ld] = v[u];
          Sm[(k + ja[u]) + (k + ia[u]) * ld] = v[u];
        }
    }
    for (; e < rr; e += NT) {
      const int jj = e / r, ii = e - jj * r;
      if (ii < jj) continue;
      const double v = parent_sigma(Sp, mp, rel[ii], rel[jj]);
      Sm[(k + ii) + (k + jj) * ld] = v;
      Sm[(k + jj) + (k + ii) * ld] = v;
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = NT / 32;
  const int g = lane >> 2, tg = lane & 3;
  const int nblk = (k + 15) / 16;
  for (int bi = nblk - 1; bi >= 0; --bi) {
    const int j0 = bi * 16, j1 = min(k, j0 + 16), w = j1 - j0, na = m - j1;
    const int T = (na + 7) >> 3;
    if (warp == 0) {
      warp_trinv16(Lp + j0 + j0 * ld, ld, w, lam, xbuf);
      if (lane < 16) dv[lane] = lane < w ? 1.0 / Lp[(j0 + lane) * (ld + 1)] : 0.0;
    } else {
      // G = Sigma_AA L_AJ: 8 rows x 16 columns per task, K = na split in two chains
      for (int task = warp - 1; task < T; task += nw - 1) {
        const int i = j1 + 8 * task + g;
        double c[2][2][2] = {};
        for (int kk = 0; kk < na; kk += 8) {
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            const int l = j1 + kk + 4 * hh + tg;
            const double a = (i < m && l < m) ? Sm[i + l * ld] : 0.0;
#pragma unroll
            for (int ct = 0; ct < 2; ++ct) {
              const int t = ct * 8 + g;
              const double bb = (l < m && t < w) ? Lp[l + (j0 + t) * ld] : 0.0;
              dmma884(c[hh][ct][0], c[hh][ct][1], a, bb);
            }
          }
        }
#pragma unroll
        for (int ct = 0; ct < 2; ++ct)
#pragma unroll
          for (int h2 = 0; h2 < 2; ++h2) Xb[(ct * 8 + 2 * tg + h2) * uld + 8 * task + g] = c[0][ct][h2] + c[1][ct][h2];
      }
    }
    __syncthreads();
    // X = -G L_JJ^-1 -> Sigma_AJ (both triangles)
    for (int task = warp; task < T; task += nw) {
      double c[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int kk = 0; kk < 16; kk += 4) {
        const double a = Xb[(kk + tg) * uld + 8 * task + g];
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) dmma884(c[ct][0], c[ct][1], a, lam[(kk + tg) + (ct * 8 + g) * kLamLd]);
      }
      const int i = j1 + 8 * task + g;
#pragma unroll
      for (int ct = 0; ct < 2; ++ct)
#pragma unroll
        for (int h2 = 0; h2 < 2; ++h2) {
          const int t = ct * 8 + 2 * tg + h2;
          if (i < m && t < w) {
            Sm[i + (j0 + t) * ld] = -c[ct][h2];
            Sm[(j0 + t) + i * ld] = -c[ct][h2];
          }
        }
    }
    __syncthreads();
    // P[j][i] = sum_{l in A} L[l, j0+j] X[l, i]  (4 tiles, K = na in two chains)
    for (int task = warp; task < 4; task += nw) {
      const int jt = task >> 1, it = task & 1;
      double c[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
      for (int kk = 0; kk < na; kk += 8) {
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const int l = j1 + kk + 4 * hh + tg;
          const double a = (l < m) ? Lp[l + (j0 + jt * 8 + g) * ld] : 0.0;
          const double bb = (l < m) ? Sm[l + (j0 + it * 8 + g) * ld] : 0.0;
          dmma884(c[hh][0], c[hh][1], a, bb);
        }
      }
#pragma unroll
      for (int h2 = 0; h2 < 2; ++h2) Pm[(jt * 8 + g) + (it * 8 + 2 * tg + h2) * kLamLd] = c[0][h2] + c[1][h2];
    }
    __syncthreads();
    // M = D^-1 L_JJ^-1 - P
    for (int e = threadIdx.x; e < 256; e += NT) {
      const int rr2 = e & 15, cc = e >> 4;
      Pm[rr2 + cc * kLamLd] = (rr2 < w && cc < w) ? lam[rr2 + cc * kLamLd] * dv[rr2] - Pm[rr2 + cc * kLamLd] : 0.0;
    }
    __syncthreads();
    // Sigma_JJ = L_JJ^-T M
    for (int task = warp; task < 4; task += nw) {
      const int jt = task >> 1, it = task & 1;
      double c0 = 0.0, c1 = 0.0;
#pragma unroll
      for (int kk = 0; kk < 16; kk += 4)
        dmma884(c0, c1, lam[(kk + tg) + (jt * 8 + g) * kLamLd], Pm[(kk + tg) + (it * 8 + g) * kLamLd]);
      const int rr2 = jt * 8 + g;
#pragma unroll
      for (int h2 = 0; h2 < 2; ++h2) {
        const int cc = it * 8 + 2 * tg + h2;
        const double v = h2 ? c1 : c0;
        if (rr2 < w && cc < w && rr2 >= cc) {
          Sm[(j0 + rr2) + (j0 + cc) * ld] = v;
          Sm[(j0 + cc) + (j0 + rr2) * ld] = v;
        }
      }
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < m * m; e += NT) {
    const int col = e / m, row = e - col * m;
    if (row >= col) Ss[e] = Sm[row + col * ld];
  }
}

// Selected inverse of tiny fronts (m <= kTinyM), one warp per (front, problem), the
// Takahashi recurrence of sparse_ldlt.rs:376-432 restricted to the front: for the pivot
// columns j from right to left, lane i > j forms S_ij = -sum_{l > j} L_lj S_li, then
// S_jj = 1/d_j - sum_{l > j} L_lj S_lj (a fixed shuffle tree), with Sigma kept with both
// triangles in the warp's shared slice and Sigma of the below-rows gathered from the parent.
constexpr int kTinySiWarps = 2;  // two 32 x 33 slices per warp: 33.8 KB of static shared memory
__global__ void __launch_bounds__(32 * kTinySiWarps) k_selinv_tiny(DevSym S, const int* __restrict__ list, int nlist,
                                                                  const double* __restrict__ F,
                                                                  double* __restrict__ Sg, int64_t fstride) {
  __shared__ double sS[kTinySiWarps][kTinyM * kTinyLd];
  __shared__ double sL[kTinySiWarps][kTinyM * kTinyLd];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int idx = blockIdx.x * kTinySiWarps + warp;
  if (idx >= nlist) return;  // the whole warp leaves; only warp-level synchronization follows
  const int s = list[idx], b = blockIdx.y;
  const int k = sn_k(S, s), m = sn_m(S, s), r = m - k;
  double* Sm = sS[warp];
  double* L = sL[warp];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* Ss = Sg + (int64_t)b * fstride + S.fptr[s];
  for (int e = lane; e < m * k; e += 32) {
    const int c = e / m, i = e - c * m;
    L[i + c * kTinyLd] = Fs[e];
  }
  if (r > 0) {
    const int p = S.parent[s];
    const int mp = sn_m(S, p);
    const double* Sp = Sg + (int64_t)b * fstride + S.fptr[p];
    const int* rel = S.relx + S.rowptr[s] + k;
    for (int e = lane; e < r * r; e += 32) {
      const int jj = e / r, ii = e - jj * r;
      if (ii < jj) continue;
      const double v = parent_sigma(Sp, mp, rel[ii], rel[jj]);
      Sm[(k + ii) + (k + jj) * kTinyLd] = v;
      Sm[(k + jj) + (k + ii) * kTinyLd] = v;
    }
  }
  __syncwarp();
  for (int j = k - 1; j >= 0; --j) {
    const bool mine = lane > j && lane < m;
    double acc = 0.0;
    if (mine)
      for (int l = j + 1; l < m; ++l) acc += L[l + j * kTinyLd] * Sm[l + lane * kTinyLd];
    __syncwarp();
    if (mine) {
      Sm[lane + j * kTinyLd] = -acc;
      Sm[j + lane * kTinyLd] = -acc;
    }
    __syncwarp();
    double t = mine ? L[lane + j * kTinyLd] * Sm[lane + j * kTinyLd] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) Sm[j + j * kTinyLd] = 1.0 / L[j + j * kTinyLd] - t;
    __syncwarp();
  }
  for (int e = lane; e < m * m; e += 32) {
    const int col = e / m, row = e - col * m;
    if (row >= col) Ss[e] = Sm[row + col * kTinyLd];
  }
}

// diag(Q^-1) in original order
__global__ void k_extract_diag(DevSym S, const double* __restrict__ Sg, int64_t fstride, double* __restrict__ out,
                               int64_t ostride) {
  const int b = blockIdx.y;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < S.n; j += gridDim.x * blockDim.x)
    out[(int64_t)b * ostride + S.perm[j]] = Sg[(int64_t)b * fstride + S.dpos[j]];
}

// Sigma (or L) values back on the lower entries of the input pattern:
// out[b][p] = buf[b][spos[p]] for lower entries, 0 for upper entries.
__global__ void k_pattern_values(int64_t nnz, const int64_t* __restrict__ spos, const double* __restrict__ buf,
                                 int64_t fstride, double* __restrict__ out) {
  const int b = blockIdx.y;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
    int64_t q = spos[p];
    out[(int64_t)b * nnz + p] = q >= 0 ? buf[(int64_t)b * fstride + q] : 0.0;
  }
}

}  // namespace
}  // namespace inla
