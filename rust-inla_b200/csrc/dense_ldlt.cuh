// Blocked dense LDL^T of a symmetric block held in shared memory.
//
// The pivots are taken 16 at a time. One warp factors the 16 x 16 diagonal
// block in registers (warp_ldlt16: one __syncwarp per pivot, no CTA barrier
// on the pivot chain) and forms its inverse Lam = L_kk^-1 alongside. The rows
// below and the trailing matrix are then updated by all warps with FP64
// tensor-core tiles (mma.sync m8n8k4):
//   U_bk = A_bk Lam^T            (= L_bk D_k),  L_bk = U_bk D_k^-1
//   A_bb -= L_bk U_bk^T          (lower triangle)
// which is the right-looking blocked LDL^T (Golub & Van Loan, Matrix
// Computations, 4th ed., Sec. 4.2) with the diagonal-block solve done through
// the explicit inverse of the unit triangle. Optionally the inverse of the
// whole unit lower factor of the leading kp x kp block is accumulated as well
// (block forward elimination: Li_k <- Lam Li_k, Li_b <- Li_b - L_bk Li_k).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace inla {
namespace {

__device__ __forceinline__ void dmma884(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// 8-byte asynchronous global -> shared copies (many in flight per thread).
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Shared scratch of the blocked routine (doubles).
constexpr int kLamLd = 20;  // leading dimension of the 16 x 16 Lam block (== 4 mod 16: conflict-free tiles)
constexpr int kDenseScratch = 64 + 16 * kLamLd + 32;

// Leading dimension for an m-row block in shared memory: >= m and == 4 (mod 16),
// so the 16 lanes of a half-warp reading an 8 x 4 fragment hit 16 distinct banks.
__host__ __device__ constexpr int dense_ld(int m) { return ((m + 11) / 16) * 16 + 4; }
// Leading dimension of the 16-column U buffer of cta_ldlt (rows rounded up to 8).
__host__ __device__ constexpr int dense_uld(int m) { return dense_ld(m + 8); }

// One warp: LDL^T and inverse of the w x w (w <= 16) leading block of A
// (shared memory, column-major, leading dimension lda; lower triangle read).
// On exit A holds L strictly below the diagonal and D on it (inside w x w
// only); Lam (ld kLamLd) holds L^-1 as a 16 x 16 unit lower triangle
// (identity beyond w); dv[t] = d_t and di[t] = 1 / d_t (1 beyond w).
// Lane layout: row r = lane / 2 and the columns j = (lane & 1) + 2q, q < 8.
// xbuf: 64 doubles (double-buffered pivot column and pivot row of Lam).
__device__ __forceinline__ void warp_ldlt16(double* A, int lda, int w, double* Lam, double* dv, double* di,
                                            double* xbuf) {
  const int lane = threadIdx.x & 31, r = lane >> 1, h = lane & 1;
  double v[8], li[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int j = h + 2 * q;
    v[q] = (r < w && j < w) ? (r >= j ? A[r + j * lda] : A[j + r * lda]) : (r == j ? 1.0 : 0.0);
    li[q] = (r == j) ? 1.0 : 0.0;
  }
#pragma unroll 16
  for (int p = 0; p < 16; ++p) {
    double* col = xbuf + (p & 1) * 32;  // col[0..15]: column p; col[16..31]: row p of Lam
    if (h == (p & 1)) col[r] = v[p >> 1];
    if (r == p) {
#pragma unroll
      for (int q = 0; q < 8; ++q) col[16 + h + 2 * q] = li[q];
    }
    __syncwarp();
    const double dinv = 1.0 / col[p];
    if (lane == p) {
      dv[p] = col[p];
      di[p] = dinv;
    }
    const double ci = (r > p) ? col[r] * dinv : 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int j = h + 2 * q;
      if (j > p) v[q] -= ci * col[j];
      li[q] -= ci * col[16 + j];
    }
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int j = h + 2 * q;
    if (r < w && j < w && r >= j) A[r + j * lda] = (r == j) ? v[q] : v[q] * di[j];
    Lam[r + j * kLamLd] = li[q];
  }
  __syncwarp();
}

// One warp: Lam = L^-1 of the unit lower w x w (w <= 16) block of L (shared
// memory, column-major, leading dimension ldl; the diagonal is not read),
// identity-padded to 16 x 16 (ld kLamLd). Forward elimination
// Lam[i,:] -= L[i,p] Lam[p,:] for i > p, one __syncwarp per step; xbuf: 32 doubles.
__device__ __forceinline__ void warp_trinv16(const double* L, int ldl, int w, double* Lam, double* xbuf) {
  const int lane = threadIdx.x & 31, r = lane >> 1, h = lane & 1;
  double li[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) li[q] = (r == h + 2 * q) ? 1.0 : 0.0;
#pragma unroll 16
  for (int p = 0; p < 16; ++p) {
    double* row = xbuf + (p & 1) * 16;
    const double lrp = (r > p && r < w && p < w) ? L[r + p * ldl] : 0.0;
    if (r == p) {
#pragma unroll
      for (int q = 0; q < 8; ++q) row[h + 2 * q] = li[q];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 8; ++q) li[q] -= lrp * row[h + 2 * q];
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) Lam[r + (h + 2 * q) * kLamLd] = li[q];
  __syncwarp();
}

// Lower-triangle tile index: task = I (I + 1) / 2 + J, J <= I.
__device__ __forceinline__ void tri_decode(int task, int& I, int& J) {
  int t = (int)((sqrtf(8.0f * (float)task + 1.0f) - 1.0f) * 0.5f);
  while ((t + 1) * (t + 2) / 2 <= task) ++t;
  while (t * (t + 1) / 2 > task) --t;
  I = t;
  J = task - t * (t + 1) / 2;
}

// Partial LDL^T of the m x m symmetric matrix A (shared memory, column-major,
// leading dimension lda, lower triangle), eliminating the first kp columns.
// On exit A[:, :kp] holds L (unit, strictly lower) with D on the diagonal and
// the lower triangle of A[kp:, kp:] holds the Schur complement. With kInv, Li
// (shared, leading dimension ldi, kp x kp) receives the inverse of the unit
// lower factor of the leading kp x kp block (Li must be zero on entry). Called
// by all threads of the CTA; U: 16 x ldu doubles with ldu = dense_uld(m);
// ws: kDenseScratch doubles. Ends with a barrier.
template <bool kInv>
__device__ __forceinline__ void cta_ldlt(double* A, int lda, int m, int kp, double* Li, int ldi, double* U, int ldu, double* ws) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int g = lane >> 2, tg = lane & 3;
  double* xbuf = ws;
  double* lam = ws + 64;
  double* dv = lam + 16 * kLamLd;
  double* di = dv + 16;
  for (int o = 0; o < kp; o += 16) {
    const int w = min(16, kp - o);
    if (warp == 0) {
      warp_ldlt16(A + o + (int64_t)o * lda, lda, w, lam, dv, di, xbuf);
      if (kInv) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int e = lane + 32 * q, rr = e & 15, cc = e >> 4;
          if (rr < w && cc < w) Li[(o + rr) + (int64_t)(o + cc) * ldi] = lam[rr + cc * kLamLd];
        }
      }
    }
    __syncthreads();
    const int base = o + w, nb = m - base, T = (nb + 7) >> 3;
    // U_bk = A_bk Lam^T and L_bk = U_bk D^-1 (8-row tasks, 16 columns each)
    for (int task = warp; task < T; task += nw) {
      const int i = base + 8 * task + g;
      double c[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
      for (int kk = 0; kk < 16; kk += 4) {
        const int u = kk + tg;
        const double a = (u < w && i < m) ? A[i + (int64_t)(o + u) * lda] : 0.0;
#pragma unroll
        for (int ct = 0; ct < 2; ++ct) dmma884(c[ct][0], c[ct][1], a, lam[(ct * 8 + g) + u * kLamLd]);
      }
      __syncwarp();
      const int ri = base + 8 * task + g;
#pragma unroll
      for (int ct = 0; ct < 2; ++ct)
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
          const int t = ct * 8 + 2 * tg + hh;
          const bool ok = ri < m && t < w;
          U[t * ldu + (ri - base)] = ok ? c[ct][hh] : 0.0;
          if (ok) A[ri + (int64_t)(o + t) * lda] = c[ct][hh] * di[t];
        }
    }
    if (kInv) {
      // Li_k[:, :o] <- Lam Li_k[:, :o]  (16 rows x 8 columns per task)
      for (int task = warp; task < (o >> 3); task += nw) {
        const int c0 = 8 * task;
        double c[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
        for (int kk = 0; kk < 16; kk += 4) {
          const int u = kk + tg;
          const double b = (u < w) ? Li[(o + u) + (int64_t)(c0 + g) * ldi] : 0.0;
#pragma unroll
          for (int rt = 0; rt < 2; ++rt) dmma884(c[rt][0], c[rt][1], lam[(rt * 8 + g) + u * kLamLd], b);
        }
        __syncwarp();
#pragma unroll
        for (int rt = 0; rt < 2; ++rt)
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            const int rr = rt * 8 + g;
            if (rr < w) Li[(o + rr) + (int64_t)(c0 + 2 * tg + hh) * ldi] = c[rt][hh];
          }
      }
    }
    __syncthreads();
    if (nb <= 0) break;
    // trailing update A_bb -= L_bk U_bk^T (lower 8 x 8 tiles)
    const int ntask = T * (T + 1) / 2;
    for (int task = warp; task < ntask; task += nw) {
      int I, J;
      tri_decode(task, I, J);
      const int i = base + 8 * I + g, jb = 8 * J + g;
      double c0 = 0.0, c1 = 0.0;
#pragma unroll
      for (int kk = 0; kk < 16; kk += 4) {
        const int u = kk + tg;
        const double a = (u < w && i < m) ? A[i + (int64_t)(o + u) * lda] : 0.0;
        const double b = U[u * ldu + jb];
        dmma884(c0, c1, a, b);
      }
      const int jc = base + 8 * J + 2 * tg;
      if (i < m) {
        if (jc < m && i >= jc) A[i + (int64_t)jc * lda] -= c0;
        if (jc + 1 < m && i >= jc + 1) A[i + (int64_t)(jc + 1) * lda] -= c1;
      }
    }
    if (kInv) {
      // Li_b[:, :base] -= L_bk Li_k[:, :base]  (rows of later blocks inside kp)
      const int nbi = kp - base, Ti = (nbi + 7) >> 3, Tc = (base + 7) >> 3;
      for (int task = warp; task < Ti * Tc; task += nw) {
        const int I = task / Tc, Jc = task - I * Tc;
        const int i = base + 8 * I + g;
        double c0 = 0.0, c1 = 0.0;
#pragma unroll
        for (int kk = 0; kk < 16; kk += 4) {
          const int u = kk + tg;
          const double a = (u < w && i < kp) ? A[i + (int64_t)(o + u) * lda] : 0.0;
          const double b = (u < w) ? Li[(o + u) + (int64_t)(8 * Jc + g) * ldi] : 0.0;
          dmma884(c0, c1, a, b);
        }
        const int jc = 8 * Jc + 2 * tg;
        if (i < kp) {
          if (jc < base) Li[i + (int64_t)jc * ldi] -= c0;
          if (jc + 1 < base) Li[i + (int64_t)(jc + 1) * ldi] -= c1;
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace
}  // namespace inla
