// Large-front kernels (fronts with more than 96 rows), 64-column blocks.
//
// Factorization, per block J = [j0, j0+w) of a front (right-looking):
//   k_gather8   extend-add of the children's updates (once per level);
//   k_panel64   every CTA factors the w x w diagonal block with the blocked
//               dense routine (cta_ldlt, which also forms L_JJ^-1); CTA 0
//               stores the factored block (dcache) and L_JJ^-1 (the inverse-
//               block cache, reused by the selected inverse); each CTA forms
//               its 64 rows L_i = F_i L_JJ^-T D_J^-1 as one tensor-core GEMM;
//   update      F[i,j] -= sum_{t in J} L_it d_t L_jt on 64x64 tiles of the lower
//               trailing matrix (tensor-core tiles, operands staged with cp.async;
//               update64w8_body in snode_persist.cuh, launched as k_update64w8).
// Selected inverse, per block J from right to left (A = rows after J):
//   k_si_step64 G = Sigma[A,A] L[A,J] per 64-row tile of A (the K range split over
//               several CTAs where the launch would leave SMs idle), X = -G L_JJ^-1
//               (cached inverse block), Sigma[A,J] = X, and the tile's partial
//               P = L[I,J]^T X[I,J];
//   k_si_diag64 Sigma_JJ = L_JJ^-T (D^-1 L_JJ^-1 - P), P the fixed-order sum of
//               the partials: the closed form of the in-block Takahashi
//   recurrence S_ij = -P_ji - sum_{l in J, l>j} L_lj S_li,
//   S_jj = 1/d_j - P_jj - sum_{l in J, l>j} L_lj S_lj.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dense_ldlt.cuh"
#include "devsym.hpp"

namespace inla {
namespace {

constexpr int kB64 = 64;         // block-column width
constexpr int kPanelRows = 64;   // rows per panel GEMM sub-block
constexpr int kLd64 = dense_ld(kB64);
constexpr int kULd64 = dense_uld(kB64);
constexpr int kPanelSmem = (2 * kB64 * kLd64 + 16 * kULd64 + kDenseScratch) * 8;
constexpr int kSiGemmSmem = 3 * 64 * kLd64 * 8;  // three stage buffers
constexpr int kSiDiagSmem = 3 * kB64 * (kB64 + 1) * 8;

__device__ __forceinline__ int lg_k(const DevSym& S, int s) { return S.first[s + 1] - S.first[s]; }
__device__ __forceinline__ int lg_m(const DevSym& S, int s) { return S.rowptr[s + 1] - S.rowptr[s]; }

__device__ __forceinline__ void mma884(double& c0, double& c1, double a, double b) { dmma884(c0, c1, a, b); }

__device__ __forceinline__ const double* linv_block(const DevSym& S, const double* linv, int b, int s, int blk) {
  return linv + (int64_t)b * S.lstride + ((int64_t)S.lbo[s] + blk) * (kB64 * kB64);
}

// Extend-add of the children's updates into parent columns [c0, c1) (gcols
// columns per CTA, at most kGatherCols, fewer when the slice would not fit;
// grng[gptr[s] + z * nchildren + q] = the child's source columns whose parent
// column falls in chunk z, from a host table): the
// column slice is assembled in shared memory (panel columns start from the
// filled values, update columns from zero), every child adds its entries in
// fixed order (targets are distinct within one child), and the slice's lower
// part is written back once. Work per child is flattened over (source column,
// row) pairs with eight independent loads in flight per thread.
constexpr int kGatherCols = 8;
// Chunk z of front s, problem b (any block size; gsl: [gcols][m] doubles of shared memory).
__device__ __forceinline__ void gather8_body(const DevSym& S, int s, int b, int z, double* __restrict__ F,
                                             int64_t fstride, int gcols, const int64_t* __restrict__ gptr,
                                             const int2* __restrict__ grng, double* gsl) {
  if (front_skipped(S, s, b)) return;
  const int k = lg_k(S, s), m = lg_m(S, s);
  const int c0 = z * gcols;
  if (c0 >= m) return;
  const int c1 = min(c0 + gcols, m), nc = c1 - c0;
  double* Fb = F + (int64_t)b * fstride;
  double* Fs = Fb + S.fptr[s];
  for (int e = threadIdx.x; e < nc * m; e += blockDim.x) {
    const int cc = e / m, row = e - cc * m, col = c0 + cc;
    if (col < k && row >= col) cp_async8(&gsl[e], Fs + row + (int64_t)col * m);
    else gsl[e] = 0.0;
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const int q0 = S.child_ptr[s], nch = S.child_ptr[s + 1] - q0;
  // source-column range of every child for this chunk (host table, no search)
  const int2* rng = grng + gptr[s] + (int64_t)z * nch;
  for (int qi = 0; qi < nch; ++qi) {
    const int c = S.child_list[q0 + qi];
    const int kc = lg_k(S, c), mc = lg_m(S, c), rc = mc - kc;
    const double* __restrict__ Uc = Fb + S.fptr[c] + (int64_t)kc * mc + kc;
    const int* __restrict__ relc = S.relx + S.rowptr[c] + kc;
    const int2 lh = rng[qi];
    const int lo = lh.x, hi = lh.y;
    const int total = (hi - lo) * rc;
    for (int e0 = 0; e0 < total; e0 += 8 * (int)blockDim.x) {
      double v[8];
      int dst[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + threadIdx.x + u * blockDim.x;
        dst[u] = -1;
        v[u] = 0.0;
        if (e < total) {
          const int jj = lo + e / rc, ii = e - (e / rc) * rc;
          if (ii >= jj) {
            v[u] = Uc[ii + (int64_t)jj * mc];
            dst[u] = (relc[jj] - c0) * m + relc[ii];
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (dst[u] >= 0) gsl[dst[u]] += v[u];
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nc * m; e += blockDim.x) {
    const int cc = e / m, row = e - cc * m, col = c0 + cc;
    if (row >= col) Fs[row + (int64_t)col * m] = gsl[e];
  }
}

__global__ void __launch_bounds__(256) k_gather8(DevSym S, const int* __restrict__ list, double* __restrict__ F,
                                                 int64_t fstride, int gcols, const int64_t* __restrict__ gptr,
                                                 const int2* __restrict__ grng) {
  extern __shared__ double gsl[];  // [gcols][m] column slice
  gather8_body(S, list[blockIdx.x], blockIdx.y, blockIdx.z, F, fstride, gcols, gptr, grng, gsl);
}

// Sigma restricted to the below-rows of s, gathered from the parent's Sigma
// front into the trailing block (lower triangle), columns [c0, c1) of it.
__device__ __forceinline__ void si_gather8_body(const DevSym& S, int s, int b, int z, double* __restrict__ Sg,
                                                int64_t fstride) {
  const int k = lg_k(S, s), m = lg_m(S, s), r = m - k;
  if (r == 0) return;
  const int c0 = z * kGatherCols;
  if (c0 >= r) return;
  const int c1 = min(c0 + kGatherCols, r);
  const int p = S.parent[s];
  const int mp = lg_m(S, p);
  const double* __restrict__ Sp = Sg + (int64_t)b * fstride + S.fptr[p];
  double* Ss = Sg + (int64_t)b * fstride + S.fptr[s];
  const int* __restrict__ rel = S.relx + S.rowptr[s] + k;
  const int total = (c1 - c0) * r;
  int e = threadIdx.x;
  for (; e + 3 * (int)blockDim.x < total; e += 4 * blockDim.x) {
    double v[4];
    int64_t dst[4];
    bool ok[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int ee = e + u * blockDim.x;
      const int jj = c0 + ee / r, ii = ee - (ee / r) * r;
      ok[u] = ii >= jj;
      const int pi = ok[u] ? rel[ii] : 0, pj = ok[u] ? rel[jj] : 0;
      v[u] = ok[u] ? (pi >= pj ? Sp[pi + (int64_t)pj * mp] : Sp[pj + (int64_t)pi * mp]) : 0.0;
      dst[u] = (k + ii) + (int64_t)(k + jj) * m;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (ok[u]) Ss[dst[u]] = v[u];
  }
  for (; e < total; e += blockDim.x) {
    const int jj = c0 + e / r, ii = e - (e / r) * r;
    if (ii < jj) continue;
    const int pi = rel[ii], pj = rel[jj];
    Ss[(k + ii) + (int64_t)(k + jj) * m] = pi >= pj ? Sp[pi + (int64_t)pj * mp] : Sp[pj + (int64_t)pi * mp];
  }
}

__global__ void __launch_bounds__(256) k_si_gather8(DevSym S, const int* __restrict__ list, double* __restrict__ Sg,
                                                    int64_t fstride) {
  si_gather8_body(S, list[blockIdx.x], blockIdx.y, blockIdx.z, Sg, fstride);
}

// The factored diagonal block goes to dcache[(list index, problem)] (written by
// CTA 0): the other CTAs of this launch still read the unfactored block from
// the front, so it is copied into the front by the trailing update (tile 0) of the same step.
// Each CTA: blocked LDL^T + inverse of the diagonal block, then the rows
// [r0, r0 + rpc) (rpc a multiple of 64) in 64-row sub-blocks, each
// X = F_rows (L_JJ^-T D^-1) as one tensor-core GEMM. The row sub-blocks are
// staged in the diagonal block's buffer once it is no longer needed, which
// keeps the CTA at 84 KB of shared memory (two CTAs per SM).
// Block J = [j0, j0 + 64) of front s, problem b, row CTA z (256 threads). dc: this front's and
// problem's slot of the factored-diagonal-block cache (written when z == 0).
__device__ __forceinline__ void panel64_body(const DevSym& S, int s, int b, int z, int j0, int rpc,
                                             double* __restrict__ F, int64_t fstride, double* __restrict__ dc,
                                             double* __restrict__ linv, double* smem64) {
  constexpr int ld = kLd64;  if (front_skipped(S, s, b)) return;

  double* Ds = smem64;         // [64 cols][ld]: diagonal block, factored in place; then row sub-blocks
  double* Li = Ds + kB64 * ld; // L_JJ^-1, then Bm[u + t*ld] = Li[t][u] / d_t
  double* U = Li + kB64 * ld;  // [16][kULd64] scratch of cta_ldlt, then 1 / d_t
  double* ws = U + 16 * kULd64;
  const int k = lg_k(S, s), m = lg_m(S, s);
  if (j0 >= k) return;
  const int w = min(kB64, k - j0);
  const int r0 = j0 + w + z * rpc;
  if (z > 0 && r0 >= m) return;
  const int r1 = min(m, r0 + rpc);
  double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  const double* D0 = Fs + j0 + (int64_t)j0 * m;
  for (int e = threadIdx.x; e < kB64 * kB64; e += blockDim.x) {
    const int c = e >> 6, r = e & 63;
    if (r < w && c < w && r >= c) cp_async8(&Ds[r + c * ld], D0 + r + (int64_t)c * m);
    else Ds[r + c * ld] = 0.0;
    Li[r + c * ld] = 0.0;
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  cta_ldlt<true>(Ds, ld, w, w, Li, ld, U, kULd64, ws);
  if (z == 0) {
    double* lc = const_cast<double*>(linv_block(S, linv, b, s, j0 / kB64));
    for (int e = threadIdx.x; e < kB64 * kB64; e += blockDim.x) {
      const int c = e >> 6, r = e & 63;
      dc[e] = (r < w && c < w) ? Ds[r + c * ld] : 0.0;
      lc[e] = Li[r + c * ld];  // zero outside the w x w lower triangle
    }
  }
  if (r0 >= r1) return;
  double* dinv = U;
  if (threadIdx.x < kB64) dinv[threadIdx.x] = threadIdx.x < w ? 1.0 / Ds[threadIdx.x * (ld + 1)] : 0.0;
  __syncthreads();
  double bv[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int e = threadIdx.x + 256 * q, u = e & 63, t = e >> 6;
    bv[q] = Li[t + u * ld] * dinv[t];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int e = threadIdx.x + 256 * q, u = e & 63, t = e >> 6;
    Li[u + t * ld] = bv[q];
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;
  const int g = lane >> 2, tg = lane & 3;
  const int wk = (w + 3) & ~3;
  double* Fa = Ds;  // row sub-block: Fa[t*ld + r] = F[rb + r, j0 + t]
  for (int rb = r0; rb < r1; rb += kPanelRows) {
    const int rows = min(kPanelRows, r1 - rb);
    __syncthreads();  // previous sub-block (or the diagonal block) fully consumed
    for (int e = threadIdx.x; e < kB64 * kPanelRows; e += blockDim.x) {
      const int c = e >> 6, r = e & 63;
      if (r < rows && c < w) cp_async8(&Fa[c * ld + r], Fs + (rb + r) + (int64_t)(j0 + c) * m);
      else Fa[c * ld + r] = 0.0;
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    // X (64 x 64) = Fa (64 x w) * Bm (w x 64); warp tile 32 x 16
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q) acc[a][q][0] = acc[a][q][1] = 0.0;
#pragma unroll 4
    for (int kk = 0; kk < wk; kk += 4) {
      double af[4], bf[2];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = Fa[(kk + tg) * ld + wr + a * 8 + g];
#pragma unroll
      for (int q = 0; q < 2; ++q) bf[q] = Li[(kk + tg) + (wc + q * 8 + g) * ld];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 2; ++q) mma884(acc[a][q][0], acc[a][q][1], af[a], bf[q]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wr + a * 8 + g, t = wc + q * 8 + tg * 2 + h;
          if (r < rows && t < w) Fs[(rb + r) + (int64_t)(j0 + t) * m] = acc[a][q][h];
        }
  }
}

__global__ void __launch_bounds__(256) k_panel64(DevSym S, const int* __restrict__ list, int j0, int rpc,
                                                 double* __restrict__ F, int64_t fstride,
                                                 double* __restrict__ dcache, double* __restrict__ linv) {
  extern __shared__ double smem64[];
  double* dc = dcache + ((int64_t)blockIdx.x * gridDim.y + blockIdx.y) * (kB64 * kB64);
  panel64_body(S, list[blockIdx.x], blockIdx.y, blockIdx.z, j0, rpc, F, fstride, dc, linv, smem64);
}

// Rows of a 64-column block from this step's factored diagonal block (dcache:
// L_JJ with D on the diagonal, written by k_panel64 launched with rpc = 0;
// linv: L_JJ^-1): X = F_rows L_JJ^-T D^-1 for the 64 rows of CTA z, one
// tensor-core GEMM. Used when many fronts x problems share a step, where a
// factorization per row CTA would be redundant work.
constexpr int kRowsSmem = (2 * kB64 * kLd64 + kB64) * 8;
// Row block z of block J of front s, problem b (256 threads); dc as in panel64_body.
__device__ __forceinline__ void rows64_body(const DevSym& S, int s, int b, int z, int j0, double* __restrict__ F,
                                            int64_t fstride, const double* __restrict__ dc,
                                            const double* __restrict__ linv, double* smr) {
  if (front_skipped(S, s, b)) return;
  constexpr int ld = kLd64;
  double* Bm = smr;               // Bm[u + t*ld] = L_JJ^-1[t][u] / d_t
  double* Fa = Bm + kB64 * ld;    // Fa[t*ld + r] = F[r0 + r, j0 + t]
  double* dinv = Fa + kB64 * ld;  // [kB64]
  const int k = lg_k(S, s), m = lg_m(S, s);
  if (j0 >= k) return;
  const int w = min(kB64, k - j0);
  const int r0 = j0 + w + z * kPanelRows;
  if (r0 >= m) return;
  const int rows = min(kPanelRows, m - r0);
  double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  for (int e = threadIdx.x; e < kB64 * kPanelRows; e += blockDim.x) {
    const int c = e >> 6, r = e & 63;
    if (r < rows && c < w) cp_async8(&Fa[c * ld + r], Fs + (r0 + r) + (int64_t)(j0 + c) * m);
    else Fa[c * ld + r] = 0.0;
  }
  cp_async_commit();
  const double* lc = linv_block(S, linv, b, s, j0 / kB64);
  if (threadIdx.x < kB64) dinv[threadIdx.x] = threadIdx.x < w ? 1.0 / dc[threadIdx.x * (kB64 + 1)] : 0.0;
  __syncthreads();
  double lv[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) lv[q] = lc[threadIdx.x + 256 * q];  // L_JJ^-1 column-major: (t, u) at t + 64 u
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    const int e = threadIdx.x + 256 * q, t = e & 63, u = e >> 6;
    Bm[u + t * ld] = lv[q] * dinv[t];
  }
  cp_async_wait<0>();
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;
  const int g = lane >> 2, tg = lane & 3;
  const int wk = (wr >= rows || wc >= w) ? 0 : (w + 3) & ~3;
  double acc[4][2][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 2; ++q) acc[a][q][0] = acc[a][q][1] = 0.0;
#pragma unroll 4
  for (int kk = 0; kk < wk; kk += 4) {
    double af[4], bf[2];
#pragma unroll
    for (int a = 0; a < 4; ++a) af[a] = Fa[(kk + tg) * ld + wr + a * 8 + g];
#pragma unroll
    for (int q = 0; q < 2; ++q) bf[q] = Bm[(kk + tg) + (wc + q * 8 + g) * ld];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q) mma884(acc[a][q][0], acc[a][q][1], af[a], bf[q]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = wr + a * 8 + g, t = wc + q * 8 + tg * 2 + h;
        if (r < rows && t < w) Fs[(r0 + r) + (int64_t)(j0 + t) * m] = acc[a][q][h];
      }
}

__global__ void __launch_bounds__(256) k_rows64(DevSym S, const int* __restrict__ list, int j0,
                                                double* __restrict__ F, int64_t fstride,
                                                const double* __restrict__ dcache, const double* __restrict__ linv) {
  extern __shared__ double smr[];
  const double* dc = dcache + ((int64_t)blockIdx.x * gridDim.y + blockIdx.y) * (kB64 * kB64);
  rows64_body(S, list[blockIdx.x], blockIdx.y, blockIdx.z, j0, F, fstride, dc, linv, smr);
}

constexpr int kUT64 = 64;

// ---------------------------------------------------------------------------
// triangular sweeps in 32-column blocks: the diagonal block is solved by one
// warp with shuffles, the rows below it are updated by the whole CTA
// (two barriers per block instead of one per column)
// ---------------------------------------------------------------------------

// Forward sweep of front s, problem b (NT threads; y: m + 2 + 32 * 33 doubles of shared memory).
template <int NT>
__device__ __forceinline__ void fwd32_body(const DevSym& S, int s, int b, const double* __restrict__ F,
                                           int64_t fstride, double* __restrict__ xp, double* __restrict__ ub,
                                           int64_t ustride, double* y) {
  const int k = lg_k(S, s), m = lg_m(S, s), f = S.first[s];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* xb = xp + (int64_t)b * S.n;
  double* ubb = ub + (int64_t)b * ustride;
  for (int t = threadIdx.x; t < m; t += NT) y[t] = t < k ? xb[f + t] : 0.0;
  __syncthreads();
  for (int q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
    const int c = S.child_list[q];
    const int kc = lg_k(S, c), rc = lg_m(S, c) - kc;
    const int* relc = S.relx + S.rowptr[c] + kc;
    const double* uc = ubb + S.uoff[c];
    for (int t = threadIdx.x; t < rc; t += NT) y[relc[t]] += uc[t];
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* Ls = y + ((m + 1) & ~1);  // [32][33] strictly lower part of the block's diagonal tile
  for (int jb = 0; jb < k; jb += 32) {
    const int wb = min(32, k - jb);
    for (int e = threadIdx.x; e < 32 * 32; e += NT) {
      const int r = e & 31, c = e >> 5;
      Ls[r * 33 + c] = (c < r && r < wb) ? Fs[(jb + r) + (int64_t)(jb + c) * m] : 0.0;
    }
    __syncthreads();
    if (warp == 0) {
      double yi = lane < wb ? y[jb + lane] : 0.0;
#pragma unroll 8
      for (int j = 0; j < 32; ++j) {
        const double yj = __shfl_sync(0xffffffffu, yi, j);
        yi -= Ls[lane * 33 + j] * yj;
      }
      if (lane < wb) y[jb + lane] = yi;
    }
    __syncthreads();
    for (int r = jb + wb + threadIdx.x; r < m; r += NT) {
      // all (up to 32) loads of the row issued together, four partial sums
      double a[4] = {0.0, 0.0, 0.0, 0.0};
      const double* Lr = Fs + r + (int64_t)jb * m;
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (j < wb) a[j & 3] += Lr[(int64_t)j * m] * y[jb + j];
      y[r] -= (a[0] + a[1]) + (a[2] + a[3]);
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < m; t += NT) {
    if (t < k) xb[f + t] = y[t] / Fs[t + (int64_t)t * m];
    else ubb[S.uoff[s] + t - k] = y[t];
  }
}

template <int NT>
__global__ void __launch_bounds__(NT, 8) k_fwd32(DevSym S, const int* __restrict__ list, const double* __restrict__ F,
                                              int64_t fstride, double* __restrict__ xp, double* __restrict__ ub,
                                              int64_t ustride) {
  extern __shared__ double y[];
  fwd32_body<NT>(S, list[blockIdx.x], blockIdx.y, F, fstride, xp, ub, ustride, y);
}

// Backward sweep of front s, problem b (NT threads; x: m + 2 + 32 * 33 doubles of shared memory).
template <int NT>
__device__ __forceinline__ void bwd32_body(const DevSym& S, int s, int b, const double* __restrict__ F,
                                           int64_t fstride, double* __restrict__ xp, double* x) {
  const int k = lg_k(S, s), m = lg_m(S, s), f = S.first[s];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* xb = xp + (int64_t)b * S.n;
  const int* R = S.rows + S.rowptr[s];
  for (int t = threadIdx.x; t < m; t += NT) x[t] = xb[R[t]];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* Ls = x + ((m + 1) & ~1);  // [32][33] strictly lower part of the block's diagonal tile
  const int nblk = (k + 31) / 32;
  for (int bi = nblk - 1; bi >= 0; --bi) {
    const int jb = bi * 32, wb = min(32, k - jb), i0 = jb + wb;
    // x_j -= sum_{i >= i0} L_ij x_i for the block's columns (warp per column)
    for (int j = jb + warp; j < jb + wb; j += NT / 32) {
      const double* Lj = Fs + (int64_t)j * m;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      int i = i0 + lane;
      for (; i + 96 < m; i += 128) {
        a0 += Lj[i] * x[i];
        a1 += Lj[i + 32] * x[i + 32];
        a2 += Lj[i + 64] * x[i + 64];
        a3 += Lj[i + 96] * x[i + 96];
      }
      for (; i < m; i += 32) a0 += Lj[i] * x[i];
      double acc = (a0 + a1) + (a2 + a3);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) x[j] -= acc;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * 32; e += NT) {
      const int r = e & 31, c = e >> 5;
      Ls[r * 33 + c] = (c < r && r < wb) ? Fs[(jb + r) + (int64_t)(jb + c) * m] : 0.0;
    }
    __syncthreads();
    if (warp == 0) {
      // lane j holds x_{jb+j}; unit upper L_JJ^T solved from the last row up
      double xj = lane < wb ? x[jb + lane] : 0.0;
#pragma unroll 8
      for (int i = 31; i >= 0; --i) {
        const double xi = __shfl_sync(0xffffffffu, xj, i);
        xj -= Ls[i * 33 + lane] * xi;
      }
      if (lane < wb) x[jb + lane] = xj;
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < k; t += NT) xb[f + t] = x[t];
}

template <int NT>
__global__ void __launch_bounds__(NT, 8) k_bwd32(DevSym S, const int* __restrict__ list, const double* __restrict__ F,
                                              int64_t fstride, double* __restrict__ xp) {
  extern __shared__ double x[];
  bwd32_body<NT>(S, list[blockIdx.x], blockIdx.y, F, fstride, xp, x);
}

// Sweeps of the large fronts (those with cached 64 x 64 inverse blocks), 64-column blocks:
// the diagonal block is applied as a product with its cached inverse L_JJ^-1 (no sequential
// substitution chain), and the rows below (forward) or the column sums (backward) are spread
// over the CTA. NT threads; NT / 64 threads share one row of the inverse-block product (their
// partial sums are combined by shuffles in a fixed order). Shared memory: m + 2 doubles.
template <int NT>
__device__ __forceinline__ double inv_block_dot(const double* __restrict__ lc, const double* v, int wb, bool trans) {
  constexpr int kP = NT / 64;
  const int r = threadIdx.x / kP, q = threadIdx.x % kP;
  double acc = 0.0;
  if (r < wb) {
    if (!trans) {  // (L^-1 v)_r = sum_{c <= r} L^-1[r][c] v_c
      for (int c = q; c <= r; c += kP) acc += lc[r + 64 * c] * v[c];
    } else {  // (L^-T v)_r = sum_{c >= r} L^-1[c][r] v_c
      for (int c = r + q; c < wb; c += kP) acc += lc[c + 64 * r] * v[c];
    }
  }
#pragma unroll
  for (int o = 1; o < kP; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  return acc;
}

// Forward sweep of large front s, problem b (NT = 256 threads). kDeep: two rows per pass and
// 32 loads per row instead of one row and 16 (more loads in flight, more registers); the
// result is the same either way.
template <int NT, bool kDeep = true>
__device__ __forceinline__ void fwd64_body(const DevSym& S, int s, int b, const double* __restrict__ F,
                                           int64_t fstride, const double* __restrict__ linv,
                                           double* __restrict__ xp, double* __restrict__ ub, int64_t ustride,
                                           double* y) {
  static_assert(NT % 64 == 0 && NT / 64 <= 32, "whole rows of the inverse-block product per warp");
  const int k = lg_k(S, s), m = lg_m(S, s), f = S.first[s];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* xb = xp + (int64_t)b * S.n;
  double* ubb = ub + (int64_t)b * ustride;
  for (int t = threadIdx.x; t < m; t += NT) y[t] = t < k ? xb[f + t] : 0.0;
  __syncthreads();
  for (int q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
    const int c = S.child_list[q];
    const int kc = lg_k(S, c), rc = lg_m(S, c) - kc;
    const int* relc = S.relx + S.rowptr[c] + kc;
    const double* uc = ubb + S.uoff[c];
    for (int t = threadIdx.x; t < rc; t += NT) y[relc[t]] += uc[t];
    __syncthreads();
  }
  const int nblk = (k + kB64 - 1) / kB64;
  for (int bi = 0; bi < nblk; ++bi) {
    const int jb = bi * kB64, wb = min(kB64, k - jb);
    const double v = inv_block_dot<NT>(linv_block(S, linv, b, s, bi), y + jb, wb, false);
    __syncthreads();  // every read of y_J is done
    if (threadIdx.x % (NT / 64) == 0 && threadIdx.x / (NT / 64) < wb) y[jb + threadIdx.x / (NT / 64)] = v;
    __syncthreads();
    // rows below: one thread per row (kDeep: two rows per pass, 32 loads of each in flight;
    // otherwise one row, 16 loads: the panel streams from DRAM, so the loads in flight set the
    // rate), eight partial sums per row in column order
    for (int r = jb + wb + threadIdx.x; r < m; r += (kDeep ? 2 : 1) * NT) {
      const int r2 = r + NT;
      const bool two = kDeep && r2 < m;
      double a[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      double c[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      const double* Lr = Fs + r + (int64_t)jb * m;
      constexpr int kJ = kDeep ? 32 : 16;  // loads of a row per pass
      for (int j0 = 0; j0 < wb; j0 += kJ) {
        double la[kJ], lb[kDeep ? kJ : 1];
#pragma unroll
        for (int u = 0; u < kJ; ++u) {
          const bool ok = j0 + u < wb;
          la[u] = ok ? Lr[(int64_t)(j0 + u) * m] : 0.0;
          if (kDeep) lb[kDeep ? u : 0] = ok && two ? Lr[(int64_t)(j0 + u) * m + NT] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kJ; ++u) {
          const double yj = j0 + u < wb ? y[jb + j0 + u] : 0.0;
          a[u & 7] += la[u] * yj;
          if (kDeep) c[u & 7] += lb[kDeep ? u : 0] * yj;
        }
      }
      y[r] -= ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
      if (two) y[r2] -= ((c[0] + c[1]) + (c[2] + c[3])) + ((c[4] + c[5]) + (c[6] + c[7]));
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < m; t += NT) {
    if (t < k) xb[f + t] = y[t] / Fs[t + (int64_t)t * m];
    else ubb[S.uoff[s] + t - k] = y[t];
  }
}

// kDeep: the register-hungry form (one CTA per SM) for launches with few CTAs; the other
// (two CTAs per SM) for wide levels. Both give the same result.
template <int NT, bool kDeep>
__global__ void __launch_bounds__(NT, kDeep ? 1 : 2) k_fwd64(DevSym S, const int* __restrict__ list,
                                                             const double* __restrict__ F, int64_t fstride,
                                                             const double* __restrict__ linv,
                                                             double* __restrict__ xp, double* __restrict__ ub,
                                                             int64_t ustride) {
  extern __shared__ double y[];
  fwd64_body<NT, kDeep>(S, list[blockIdx.x], blockIdx.y, F, fstride, linv, xp, ub, ustride, y);
}

// Backward sweep of large front s, problem b (NT = 256 threads). kDeep: four rows per pass
// instead of two (more loads in flight); every lane still visits its rows in increasing
// order, so the result is the same either way.
template <int NT, bool kDeep = true>
__device__ __forceinline__ void bwd64_body(const DevSym& S, int s, int b, const double* __restrict__ F,
                                           int64_t fstride, const double* __restrict__ linv,
                                           double* __restrict__ xp, double* x) {
  const int k = lg_k(S, s), m = lg_m(S, s), f = S.first[s];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* xb = xp + (int64_t)b * S.n;
  const int* R = S.rows + S.rowptr[s];
  for (int t = threadIdx.x; t < m; t += NT) x[t] = xb[R[t]];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nblk = (k + kB64 - 1) / kB64;
  for (int bi = nblk - 1; bi >= 0; --bi) {
    const int jb = bi * kB64, wb = min(kB64, k - jb), i0 = jb + wb;
    // x_j -= sum_{i >= i0} L_ij x_i for the block's columns: warp w takes the columns
    // j = jb + w + (NT / 32) c, all of them at once (lane l: rows i0 + l + 32 t, four rows per
    // pass), so that every lane keeps kR * kC loads in flight; a butterfly per column at the end
    {
      constexpr int kW = NT / 32, kC = 64 / kW;  // columns per warp
      double acc[kC];
#pragma unroll
      for (int c = 0; c < kC; ++c) acc[c] = 0.0;
      constexpr int kR = kDeep ? 4 : 2;  // rows per lane and pass
      for (int i = i0 + lane; i < m; i += 32 * kR) {
        double lv[kR][kC], xv[kR];
#pragma unroll
        for (int t = 0; t < kR; ++t) {
          const int it = i + 32 * t;
          xv[t] = it < m ? x[it] : 0.0;
#pragma unroll
          for (int c = 0; c < kC; ++c) {
            const int j = warp + kW * c;
            lv[t][c] = (it < m && j < wb) ? Fs[it + (int64_t)(jb + j) * m] : 0.0;
          }
        }
#pragma unroll
        for (int t = 0; t < kR; ++t)
#pragma unroll
          for (int c = 0; c < kC; ++c) acc[c] += lv[t][c] * xv[t];
      }
#pragma unroll
      for (int c = 0; c < kC; ++c) {
        double v = acc[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        const int j = warp + kW * c;
        if (lane == 0 && j < wb) x[jb + j] -= v;
      }
    }
    __syncthreads();
    const double v = inv_block_dot<NT>(linv_block(S, linv, b, s, bi), x + jb, wb, true);
    __syncthreads();
    if (threadIdx.x % (NT / 64) == 0 && threadIdx.x / (NT / 64) < wb) x[jb + threadIdx.x / (NT / 64)] = v;
    __syncthreads();
  }
  for (int t = threadIdx.x; t < k; t += NT) xb[f + t] = x[t];
}

template <int NT, bool kDeep>
__global__ void __launch_bounds__(NT, kDeep ? 1 : 2) k_bwd64(DevSym S, const int* __restrict__ list,
                                                             const double* __restrict__ F, int64_t fstride,
                                                             const double* __restrict__ linv,
                                                             double* __restrict__ xp) {
  extern __shared__ double x[];
  bwd64_body<NT, kDeep>(S, list[blockIdx.x], blockIdx.y, F, fstride, linv, xp, x);
}

// Sweeps of fronts with m <= 32 rows (one 32-column block): one warp per (front,
// problem), kTinySweepWarps per CTA. Lane t holds entry t of the front's vector; the
// arithmetic follows k_fwd32 / k_bwd32 step for step (sequential shuffle chain on the
// diagonal block, the same four partial sums for the rows below, the same xor tree
// for the column sums), so the results equal theirs.
constexpr int kTinySweepWarps = 8;

// One warp: forward sweep of tiny front s, problem b (y: 32 doubles of shared memory).
__device__ __forceinline__ void fwd_tiny_warp(const DevSym& S, int s, int b, const double* __restrict__ F,
                                              int64_t fstride, double* __restrict__ xp, double* __restrict__ ub,
                                              int64_t ustride, double* y) {
  const int lane = threadIdx.x & 31;
  const int k = lg_k(S, s), m = lg_m(S, s), f = S.first[s];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* xb = xp + (int64_t)b * S.n;
  double* ubb = ub + (int64_t)b * ustride;
  y[lane] = lane < k ? xb[f + lane] : 0.0;
  __syncwarp();
  for (int q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
    const int c = S.child_list[q];
    const int kc = lg_k(S, c), rc = lg_m(S, c) - kc;
    if (lane < rc) y[S.relx[S.rowptr[c] + kc + lane]] += ubb[S.uoff[c] + lane];
    __syncwarp();
  }
  double yi = y[lane];
  {  // diagonal block: unit lower L_JJ
    double yd = lane < k ? yi : 0.0;
    for (int j = 0; j < k; ++j) {
      const double yj = __shfl_sync(0xffffffffu, yd, j);
      if (lane > j && lane < k) yd -= Fs[lane + (int64_t)j * m] * yj;
    }
    if (lane < k) yi = yd;
    y[lane] = yi;
  }
  __syncwarp();
  if (lane >= k && lane < m) {  // rows below the block
    double a[4] = {0.0, 0.0, 0.0, 0.0};
    const double* Lr = Fs + lane;
    for (int j = 0; j < k; ++j) a[j & 3] += Lr[(int64_t)j * m] * y[j];
    yi -= (a[0] + a[1]) + (a[2] + a[3]);
  }
  if (lane < k) xb[f + lane] = yi / Fs[lane + (int64_t)lane * m];
  else if (lane < m) ubb[S.uoff[s] + lane - k] = yi;
}

__global__ void __launch_bounds__(32 * kTinySweepWarps) k_fwd_tiny(DevSym S, const int* __restrict__ list, int nlist,
                                                                   const double* __restrict__ F, int64_t fstride,
                                                                   double* __restrict__ xp, double* __restrict__ ub,
                                                                   int64_t ustride) {
  __shared__ double sy[kTinySweepWarps][32];
  const int warp = threadIdx.x >> 5;
  const int idx = blockIdx.x * kTinySweepWarps + warp;
  if (idx >= nlist) return;  // the whole warp leaves; only warp-level synchronization follows
  fwd_tiny_warp(S, list[idx], blockIdx.y, F, fstride, xp, ub, ustride, sy[warp]);
}

// One warp: backward sweep of tiny front s, problem b (registers and shuffles only).
__device__ __forceinline__ void bwd_tiny_warp(const DevSym& S, int s, int b, const double* __restrict__ F,
                                              int64_t fstride, double* __restrict__ xp) {
  const int lane = threadIdx.x & 31;
  const int k = lg_k(S, s), m = lg_m(S, s), f = S.first[s];
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* xb = xp + (int64_t)b * S.n;
  double xl = lane < m ? xb[S.rows[S.rowptr[s] + lane]] : 0.0;
  // x_j -= sum_{i >= k} L_ij x_i for the block's columns: as in k_bwd32, lane l holds the
  // term of row k + l and the butterfly total of lane 0 is used
  const int ri = k + lane;
  const double xs = __shfl_sync(0xffffffffu, xl, ri & 31);
  for (int j = 0; j < k; ++j) {
    double acc = ri < m ? Fs[ri + (int64_t)j * m] * xs : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    acc = __shfl_sync(0xffffffffu, acc, 0);
    if (lane == j) xl -= acc;
  }
  // unit upper L_JJ^T from the last row up
  for (int i = k - 1; i >= 0; --i) {
    const double xi = __shfl_sync(0xffffffffu, xl, i);
    if (lane < i) xl -= Fs[i + (int64_t)lane * m] * xi;
  }
  if (lane < k) xb[f + lane] = xl;
}

__global__ void __launch_bounds__(32 * kTinySweepWarps) k_bwd_tiny(DevSym S, const int* __restrict__ list, int nlist,
                                                                   const double* __restrict__ F, int64_t fstride,
                                                                   double* __restrict__ xp) {
  const int warp = threadIdx.x >> 5;
  const int idx = blockIdx.x * kTinySweepWarps + warp;
  if (idx >= nlist) return;  // the whole warp leaves; only warp-level synchronization follows
  bwd_tiny_warp(S, list[idx], blockIdx.y, F, fstride, xp);
}

// ---------------------------------------------------------------------------
// selected inverse
// ---------------------------------------------------------------------------

// Sigma[row, col] of a front stored as its lower triangle (column-major, ld m)
__device__ __forceinline__ double sig_lower(const double* Ss, int m, int row, int col) {
  return row >= col ? Ss[row + (int64_t)col * m] : Ss[col + (int64_t)row * m];
}

constexpr int kSiT = 64;  // rows of A per CTA

// Split of the K loop of G = Sigma[I,A] L[A,J]: a front whose A spans at least
// kSiSplitMinChunks chunks of 32 rows has its K range cut into pieces of kSiChunksPerSplit
// chunks, one CTA each, when the launch allows it (the host allows it where one CTA per row
// tile would leave SMs idle). The pieces are summed in a fixed order, so a given launch shape
// always gives the same result; split and unsplit steps differ by rounding only.
constexpr int kSiChunksPerSplit = 4;
constexpr int kSiSplitMinChunks = 8;
__host__ __device__ inline int si_nsplit(int nch, bool allow) {
  return (allow && nch >= kSiSplitMinChunks) ? (nch + kSiChunksPerSplit - 1) / kSiChunksPerSplit : 1;
}

// Sigma_JJ = L^-T (D^-1 L^-1 - P), L = L_JJ unit lower, P = L[A,J]^T Sigma[A,J]
// (the closed form of the in-block Takahashi recurrence), with L^-1 from the
// inverse-block cache and the product as a tensor-core GEMM. Block jb of front s, problem b
// (256 threads); pp_front: the tiles' partial P blocks (tile z at pp_front + z * 4096), read
// through L2 because other CTAs of the same launch wrote them.
__device__ __forceinline__ void si_diag64_body(const DevSym& S, int s, int b, int jb, const double* __restrict__ F,
                                               double* __restrict__ Sg, int64_t fstride,
                                               const double* __restrict__ pp_front,
                                               const double* __restrict__ linv, double* smem64) {
  constexpr int ld = kB64 + 1;
  double* Pm = smem64;            // P, then M = D^-1 L^-1 - P  (Pm[r + c*ld] = entry (r, c))
  double* Ld = Pm + kB64 * ld;    // L_JJ with D on the diagonal
  double* Li = Ld + kB64 * ld;    // L_JJ^-1
  const int k = lg_k(S, s), m = lg_m(S, s);
  const int nblk = (k + kB64 - 1) / kB64;
  if (jb >= nblk) return;
  const int bi = nblk - 1 - jb;
  const int j0 = bi * kB64, j1 = min(k, j0 + kB64), w = j1 - j0;
  const int ntiles = (m - j1 + kSiT - 1) / kSiT;
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* Ss = Sg + (int64_t)b * fstride + S.fptr[s];
  const double* pp = pp_front;
  const double* lc = linv_block(S, linv, b, s, bi);
  for (int e = threadIdx.x; e < kB64 * kB64; e += blockDim.x) {
    const int c = e >> 6, r = e & 63;
    if (r < w && c < w && r >= c) cp_async8(&Ld[r + c * ld], Fs + (j0 + r) + (int64_t)(j0 + c) * m);
    else Ld[r + c * ld] = 0.0;
    cp_async8(&Li[r + c * ld], lc + e);
  }
  cp_async_commit();
  {
    // partials are stored row-major: pp[j*64 + i] = P[j][i]; fixed summation order over tiles
    double acc[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc[q] = 0.0;
    for (int z = 0; z < ntiles; ++z) {
      const double* pz = pp + (int64_t)z * kB64 * kB64;
#pragma unroll
      for (int q = 0; q < 16; ++q) acc[q] += __ldcg(pz + threadIdx.x + 256 * q);
    }
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int e = threadIdx.x + 256 * q, j = e >> 6, i = e & 63;
      Pm[j + i * ld] = acc[q];
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  for (int e = threadIdx.x; e < kB64 * kB64; e += blockDim.x) {
    const int c = e >> 6, r = e & 63;
    Pm[r + c * ld] = (r < w && c < w) ? Li[r + c * ld] / Ld[r + r * ld] - Pm[r + c * ld] : 0.0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < 4) {
    const int wr = (warp & 1) * 32, wc = (warp >> 1) * 32;
    const int g = lane >> 2, tg = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[a][q][0] = acc[a][q][1] = 0.0;
#pragma unroll 4
    for (int kk = 0; kk < kB64; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = Li[(kk + tg) + (wr + a * 8 + g) * ld];  // (L^-1)^T
#pragma unroll
      for (int q = 0; q < 4; ++q) bf[q] = Pm[(kk + tg) + (wc + q * 8 + g) * ld];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 4; ++q) mma884(acc[a][q][0], acc[a][q][1], af[a], bf[q]);
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wr + a * 8 + g, c = wc + q * 8 + tg * 2 + h;
          if (r < w && c < w && r >= c) Ss[(j0 + r) + (int64_t)(j0 + c) * m] = acc[a][q][h];
        }
  }
}

// Last-arrival count: every thread's global writes are fenced, then one thread counts the
// CTA in; true in the CTA whose arrival completes the count (it then resets the counter for
// the next launch and reads what the others wrote). Nothing waits on another CTA.
__device__ __forceinline__ bool si_arrive_last(int* counter, int expected, int* sh_flag) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const int t = atomicAdd(counter, 1);
    *sh_flag = (t == expected - 1);
    if (t == expected - 1) *counter = 0;
  }
  __syncthreads();
  const bool last = *sh_flag != 0;
  if (last) __threadfence();
  return last;
}

// Off-diagonal part of one 64-column step of the selected inverse of the large fronts (block
// jb counted from the right). CTA z = I * smax + sp handles row tile I of A (64 rows) and
// K piece sp:
//   G_I = Sigma[I,A] L[A,J] over its K piece (chunks of 32 rows, three cp.async stages);
//   with a split K the pieces go to gp_front and the last piece to arrive sums them in piece
//   order; X = -G_I L_JJ^-1 (cached inverse block) is Sigma[I,J]; the tile's partial
//   P_I = L[I,J]^T X goes to pp_front (k_si_diag64 then forms Sigma_JJ).
// Every sum has a fixed order, so the result does not depend on which CTA arrives last; with
// one piece (smax == 1) the arithmetic is the single-CTA K loop.
// cnt_front: ptiles zeroed counters (one per tile), left zeroed again.
// Shared memory: three chunk buffers (Sa[32][68] + Lb[32][68] each) for the G loop;
// afterwards buffer 0 holds G (then X), buffer 1 L_JJ^-1 and buffer 2 L[I,J].
__device__ __forceinline__ void si_step64_body(const DevSym& S, int s, int b, int z, int jb,
                                               const double* __restrict__ F, double* __restrict__ Sg,
                                               int64_t fstride, double* __restrict__ pp_front,
                                               const double* __restrict__ linv, double* smem64,
                                               double* __restrict__ gp_front, int* cnt_front, int ptiles,
                                               int smax, bool allow_split) {
  __shared__ int sh_last;
  constexpr int kBuf = 64 * kLd64;  // doubles per chunk buffer (Sa[32][68] + Lb[32][68])
  typedef double Row68[kLd64];  // leading dimension 68 == 4 (mod 16): conflict-free fragments
  Row68* Gs = reinterpret_cast<Row68*>(smem64);             // [64][68]: G, then X
  Row68* Lt = reinterpret_cast<Row68*>(smem64 + 2 * kBuf);  // [64][68]: L[I0+l, j0+j]
  const int k = lg_k(S, s), m = lg_m(S, s);
  const int nblk = (k + kB64 - 1) / kB64;
  if (jb >= nblk) return;
  const int bi = nblk - 1 - jb;
  const int j0 = bi * kB64, j1 = min(k, j0 + kB64), w = j1 - j0;
  const int ntiles = (m - j1 + kSiT - 1) / kSiT;
  if (ntiles == 0) return;
  const int nch = (m - j1 + 31) / 32;
  const int ns = si_nsplit(nch, allow_split);
  const int I = z / smax, sp = z - I * smax;
  if (I >= ntiles || sp >= ns) return;
  const int I0 = j1 + I * kSiT;
  const int cb = sp * kSiChunksPerSplit, ce = ns == 1 ? nch : min(nch, cb + kSiChunksPerSplit);
  const double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  double* Ss = Sg + (int64_t)b * fstride + S.fptr[s];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // 8 warps, warp tile 32 x 16; warps whose columns lie beyond the block's w skip the products
  const int wi = (warp & 1) * 32, wj = (warp >> 1) * 16;
  const int g = lane >> 2, tg = lane & 3;
  const bool wact = wj < w && I0 + wi < m;

  // chunk loader: Sigma[I0.., l0..l0+32) (lower-triangle storage) and L[l0.., j0..j0+w)
  auto load_chunk = [&](int l0, int buf) {
    Row68* Sa = reinterpret_cast<Row68*>(smem64 + buf * kBuf);
    Row68* Lb = reinterpret_cast<Row68*>(smem64 + buf * kBuf + 32 * kLd64);
    if (I0 >= l0 + 31) {  // on/below the diagonal: stored at (i, l), coalesced over i
      for (int e = threadIdx.x; e < 32 * kSiT; e += blockDim.x) {
        const int l = e / kSiT, ii = e - l * kSiT, row = I0 + ii, col = l0 + l;
        if (row < m && col < m) cp_async8(&Sa[l][ii], Ss + row + (int64_t)col * m);
        else Sa[l][ii] = 0.0;
      }
    } else if (I0 + kSiT - 1 < l0) {  // above: read the transposed entry (l, i), coalesced over l
      for (int e = threadIdx.x; e < 32 * kSiT; e += blockDim.x) {
        const int ii = e / 32, l = e - ii * 32, row = I0 + ii, col = l0 + l;
        if (row < m && col < m) cp_async8(&Sa[l][ii], Ss + col + (int64_t)row * m);
        else Sa[l][ii] = 0.0;
      }
    } else {
      for (int e = threadIdx.x; e < 32 * kSiT; e += blockDim.x) {
        const int l = e / kSiT, ii = e - l * kSiT, row = I0 + ii, col = l0 + l;
        if (row < m && col < m)
          cp_async8(&Sa[l][ii], row >= col ? Ss + row + (int64_t)col * m : Ss + col + (int64_t)row * m);
        else Sa[l][ii] = 0.0;
      }
    }
    for (int e = threadIdx.x; e < 32 * kB64; e += blockDim.x) {
      const int t = e / 32, l = e - t * 32;
      if (t < w && l0 + l < m) cp_async8(&Lb[l][t], Fs + (l0 + l) + (int64_t)(j0 + t) * m);
      else Lb[l][t] = 0.0;
    }
    cp_async_commit();
  };

  double acc[4][2][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 2; ++q) acc[a][q][0] = acc[a][q][1] = 0.0;
  const int nc = ce - cb;
  load_chunk(j1 + 32 * cb, 0);
  if (nc > 1) load_chunk(j1 + 32 * (cb + 1), 1);
  for (int c = 0; c < nc; ++c) {
    if (c + 2 < nc) {
      load_chunk(j1 + 32 * (cb + c + 2), (c + 2) % 3);
      cp_async_wait<2>();
    } else if (c + 1 < nc) {
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const Row68* Sa = reinterpret_cast<const Row68*>(smem64 + (c % 3) * kBuf);
    const Row68* Lb = reinterpret_cast<const Row68*>(smem64 + (c % 3) * kBuf + 32 * kLd64);
    if (wact) {
#pragma unroll
      for (int kk = 0; kk < 32; kk += 4) {
        double af[4], bf[2];
#pragma unroll
        for (int a = 0; a < 4; ++a) af[a] = Sa[kk + tg][wi + a * 8 + g];
#pragma unroll
        for (int q = 0; q < 2; ++q) bf[q] = Lb[kk + tg][wj + q * 8 + g];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 2; ++q) mma884(acc[a][q][0], acc[a][q][1], af[a], bf[q]);
      }
    }
    __syncthreads();
  }
  if (ns > 1) {  // this piece to gp_front; the last piece of the tile sums them in order
    double* gp = gp_front + (int64_t)(I * smax + sp) * (kB64 * kB64);
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int h = 0; h < 2; ++h) gp[(wi + a * 8 + g) * kB64 + wj + q * 8 + tg * 2 + h] = acc[a][q][h];
    if (!si_arrive_last(cnt_front + I, ns, &sh_last)) return;
  }
  // L_JJ^-1 (cached) and L[I,J] are fetched together, G goes to buffer 0
  double* Li = smem64 + kBuf;
  const int rows = min(kSiT, m - I0);
  Row68* Lij = Lt;  // Lij[l][j] = L[I0+l, j0+j]
  {
    const double* lc = linv_block(S, linv, b, s, bi);
    for (int e = threadIdx.x; e < kB64 * kB64; e += blockDim.x) cp_async8(&Li[(e & 63) + (e >> 6) * kLd64], lc + e);
    for (int e = threadIdx.x; e < kSiT * kB64; e += blockDim.x) {
      const int j = e / kSiT, l = e - j * kSiT;
      if (l < rows && j < w) cp_async8(&Lij[l][j], Fs + (I0 + l) + (int64_t)(j0 + j) * m);
      else Lij[l][j] = 0.0;
    }
    cp_async_commit();
  }
  if (ns > 1) {
    const double* gq = gp_front + (int64_t)(I * smax) * (kB64 * kB64);
    for (int e = threadIdx.x; e < kB64 * kB64; e += blockDim.x) {
      double v = __ldcg(gq + e);
      for (int q = 1; q < ns; ++q) v += __ldcg(gq + (int64_t)q * (kB64 * kB64) + e);
      Gs[e >> 6][e & 63] = v;
    }
  } else {
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int h = 0; h < 2; ++h) Gs[wi + a * 8 + g][wj + q * 8 + tg * 2 + h] = acc[a][q][h];
  }
  // X = -G L_JJ^-1 as a tensor-core GEMM with the cached inverse of the unit
  // lower diagonal block
  cp_async_wait<0>();
  __syncthreads();
  {
    double xa[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q) xa[a][q][0] = xa[a][q][1] = 0.0;
    const int wk = (w + 3) & ~3;
    if (wact) {
#pragma unroll 4
      for (int kk = 0; kk < wk; kk += 4) {
        double af[4], bf[2];
#pragma unroll
        for (int a = 0; a < 4; ++a) af[a] = Gs[wi + a * 8 + g][kk + tg];
#pragma unroll
        for (int q = 0; q < 2; ++q) bf[q] = Li[(kk + tg) + (wj + q * 8 + g) * kLd64];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 2; ++q) mma884(xa[a][q][0], xa[a][q][1], af[a], bf[q]);
      }
    }
    __syncthreads();  // all reads of G done before X overwrites it
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int ii = wi + a * 8 + g, t = wj + q * 8 + tg * 2 + h;
          const double xv = -xa[a][q][h];
          Gs[ii][t] = xv;
          if (I0 + ii < m && t < w) Ss[(I0 + ii) + (int64_t)(j0 + t) * m] = xv;
        }
  }
  __syncthreads();
  // partial P[j][i] = sum_{rows l of this tile} L[I0+l, j0+j] X[l, i]  (tensor-core tiles)
  double pa[4][2][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 2; ++q) pa[a][q][0] = pa[a][q][1] = 0.0;
  const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;  // output rows j, cols i
  if (wr < w && wc < w) {
    const int kr = (rows + 3) & ~3;
#pragma unroll 4
    for (int kk = 0; kk < kr; kk += 4) {
      double af[4], bf[2];
#pragma unroll
      for (int a = 0; a < 4; ++a) af[a] = Lij[kk + tg][wr + a * 8 + g];
#pragma unroll
      for (int q = 0; q < 2; ++q) bf[q] = Gs[kk + tg][wc + q * 8 + g];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int q = 0; q < 2; ++q) mma884(pa[a][q][0], pa[a][q][1], af[a], bf[q]);
    }
  }
  double* pp = pp_front + (int64_t)I * (kB64 * kB64);
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) pp[(wr + a * 8 + g) * kB64 + wc + q * 8 + tg * 2 + h] = pa[a][q][h];
}

// ppart: [list index][b][tile][64*64] partial P blocks; gpart: [list index][b][tile][piece]
// [64*64] pieces of G (used when smax > 1); cnt: [list index][b][ptiles] counters.
__global__ void __launch_bounds__(256) k_si_step64(DevSym S, const int* __restrict__ list, int jb,
                                                  const double* __restrict__ F, double* __restrict__ Sg,
                                                  int64_t fstride, double* __restrict__ ppart, int ptiles,
                                                  const double* __restrict__ linv, double* __restrict__ gpart,
                                                  int* __restrict__ cnt, int smax, int allow_split) {
  extern __shared__ double smem64[];
  const int64_t slot = (int64_t)blockIdx.x * gridDim.y + blockIdx.y;
  // gpart is sized for split launches only (smax > 1)
  si_step64_body(S, list[blockIdx.x], blockIdx.y, blockIdx.z, jb, F, Sg, fstride,
                 ppart + slot * ptiles * (kB64 * kB64), linv, smem64,
                 smax > 1 ? gpart + slot * ptiles * smax * (kB64 * kB64) : gpart, cnt + slot * ptiles, ptiles, smax,
                 allow_split != 0);
}

__global__ void __launch_bounds__(256) k_si_diag64(DevSym S, const int* __restrict__ list, int jb,
                                                  const double* __restrict__ F, double* __restrict__ Sg,
                                                  int64_t fstride, const double* __restrict__ ppart, int ptiles,
                                                  const double* __restrict__ linv) {
  extern __shared__ double smem64[];
  const double* pp = ppart + ((int64_t)blockIdx.x * gridDim.y + blockIdx.y) * ptiles * (kB64 * kB64);
  si_diag64_body(S, list[blockIdx.x], blockIdx.y, jb, F, Sg, fstride, pp, linv, smem64);
}

}  // namespace
}  // namespace inla
