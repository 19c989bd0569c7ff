// Persistent batched factorization: one launch runs every front of every problem.
//
// The level kernels (snode_kernels.cuh, snode_large.cuh) need one launch per level and per
// 64-column step of the large fronts. Here the same work is a queue of tasks in a
// topological order of the supernodal elimination tree, claimed by a fixed grid of
// resident CTAs with one atomic counter:
//   tiny fronts (m <= 32): up to 8 fronts per task, one warp each;
//   small fronts (m <= 96): one task per front;
//   large fronts: extend-add chunks, then per 64-column block J one diagonal-block task,
//   the row-block tasks and the trailing-update tiles.
// Tasks are ordered level by level and, inside a level, phase by phase (every problem of the
// batch in turn). A task waits only for tasks earlier in the queue: the fronts of its
// children (all of their tasks done) and the earlier phases of its own front. Every task
// earlier in the queue was claimed by a CTA that is already running, so the smallest
// unfinished task can always proceed and the schedule cannot deadlock whatever the grid.
//
// Completion is counted per (problem, front): the last thread of a task's CTA publishes
// its writes (barrier, then a gpu-scope fence and an atomic increment); a waiting CTA reads
// the counter with a gpu-scope acquire load and releases its threads with a barrier.
// Every wait is bounded: past the time limit the CTA records an error code and leaves, and
// every other waiting CTA leaves when it sees the code, so a broken dependency ends the
// launch instead of hanging it. The host reads the code after the launch.
//
// Results equal the level kernels' bit for bit: every task runs the same arithmetic in the
// same order (the trailing update splits each 64 x 64 tile over eight warps instead of four,
// with each entry's products accumulated in the same K order).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "snode_kernels.cuh"
#include "snode_large.cuh"

namespace inla {
namespace {

enum PersistTaskType : int { PT_TINY = 0, PT_SMALL = 1, PT_GATHER = 2, PT_DIAG = 3, PT_ROWS = 4, PT_UPDATE = 5 };

// One task of one problem (the batch repeats the per-problem list).
struct PersistTask {
  int type;
  int s;      // front; PT_TINY: offset of the first front in the tiny list
  int sub;    // PT_TINY: number of fronts; PT_GATHER: chunk; PT_ROWS: row block; PT_UPDATE: tile
  int need;   // tasks of the same front that must be done first (completion count)
  int j0;     // first column of the 64-column block (steps)
  int gcols;  // PT_GATHER: columns per chunk
};

struct PersistArgs {
  DevSym S;
  double* F;
  int64_t fstride;
  int B;
  int ngroups;              // groups of tasks (a level's phase)
  const int* gstart;        // [ngroups + 1] prefix of the per-problem task counts
  const PersistTask* task;  // [gstart[ngroups]] per-problem tasks, group after group
  const int* tiny_list;     // fronts of the tiny tasks
  const int* total;         // [ns] tasks of each front (its completion count)
  int* prog;                // [B][ns] completed tasks per (problem, front)
  unsigned* head;           // next task to claim
  int* err;                 // 0, or the reason the launch stopped early
  double* dcache;           // [nlarge][B] factored diagonal blocks
  const int* lid;           // [ns] index of a large front (-1 otherwise)
  double* linv;
  const int64_t* gptr;      // extend-add chunk table of this schedule
  const int2* grng;
  long long limit_ns;       // longest wait for one dependency
};

constexpr int kPersistThreads = 256;
constexpr int kPersistTinyWarps = kPersistThreads / 32;
constexpr int kPersistTinySlice = kTinyM * kTinyLd + kTinyM + kTinyM / 2;  // doubles per warp
constexpr int kPersistTinySmem = kPersistTinyWarps * kPersistTinySlice * 8;
constexpr int kPersistUpdSmem = (2 * kB64 * kLd64 + kB64) * 8;
constexpr int kErrTimeout = 1;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ long long globaltimer_ns() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Thread 0 only: wait until *p >= target. Returns false (leave) on the time limit, after
// 2^26 polls, or when another CTA reported an error.
__device__ bool wait_at_least(const int* p, int target, int* err, long long limit_ns) {
  if (ld_acquire_gpu(p) >= target) return true;
  const long long t0 = globaltimer_ns();
  unsigned sleep = 32;
  for (int it = 0; it < (1 << 26); ++it) {
    if (ld_acquire_gpu(p) >= target) return true;
    if (*(volatile int*)err != 0) return false;
    if (globaltimer_ns() - t0 > limit_ns) break;
    __nanosleep(sleep);
    if (sleep < 1024) sleep <<= 1;
  }
  atomicCAS(err, 0, kErrTimeout);
  return false;
}

__device__ bool wait_children(const PersistArgs& a, int s, int b) {
  const DevSym& S = a.S;
  for (int q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
    const int c = S.child_list[q];
    if (!wait_at_least(a.prog + (int64_t)b * S.ns + c, a.total[c], a.err, a.limit_ns)) return false;
  }
  return true;
}

// Trailing update tile `tile` of block J of front s, problem b, over eight warps (32 x 16
// warp tiles): every entry accumulates its products over K in the same order as any other warp
// tiling of the same step, so the result does not depend on the tiling.
//
// kNext (look-ahead): tile 0 holds the next diagonal block [c, c + w') (w' = min(64, k - c))
// once its update is done, so that CTA factors it right away, exactly as k_panel64 with no
// rows would after this launch: the updated values go to shared memory as well as to the
// front, cta_ldlt<true> factors them, and the CTA writes the factored block into the front,
// D and L to dc_next (the cache slot of the next step; dc is this step's) and L^-1 to the
// inverse-block cache. The other tiles of this launch read only block column J and their own
// targets, so nothing else reads the block while it is factored. smu: kPanelSmem bytes.
template <bool kNext = false>
__device__ __forceinline__ void update64w8_body(const DevSym& S, int s, int b, int tile, int j0,
                                                double* __restrict__ F, int64_t fstride,
                                                const double* __restrict__ dc, double* smu,
                                                double* __restrict__ dc_next = nullptr,
                                                double* __restrict__ linv = nullptr) {
  if (front_skipped(S, s, b)) return;
  constexpr int ld = kLd64;
  double* As = smu;              // As[t*ld + i] = L[I0+i, j0+t]
  double* Bs = smu + kB64 * ld;  // Bs[t*ld + j] = L[J0+j, j0+t]
  double* dsh = Bs + kB64 * ld;  // [kB64]
  const int k = lg_k(S, s), m = lg_m(S, s);
  if (j0 >= k) return;
  const int w = min(kB64, k - j0);
  const int c = j0 + w;
  const int T = m - c;
  double* Fs = F + (int64_t)b * fstride + S.fptr[s];
  if (tile == 0) {  // factored diagonal block -> front
    double* D0 = Fs + j0 + (int64_t)j0 * m;
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
      const int cc = e / w, r = e - cc * w;
      if (r >= cc) D0[r + (int64_t)cc * m] = dc[r + cc * kB64];
    }
  }
  if (T <= 0) return;
  const int nt = (T + kUT64 - 1) / kUT64;
  if (tile >= nt * (nt + 1) / 2) return;
  int J = 0, rem = tile;
  while (rem >= nt - J) {
    rem -= nt - J;
    ++J;
  }
  const int I = J + rem;
  const int I0 = c + I * kUT64, J0 = c + J * kUT64;
  const double* Lb = Fs + (int64_t)j0 * m;
  for (int e = threadIdx.x; e < kB64 * kUT64; e += blockDim.x) {
    const int t = e >> 6, ii = e & 63;
    const double* col = Lb + (int64_t)t * m;
    if (t < w && I0 + ii < m) cp_async8(&As[t * ld + ii], col + I0 + ii);
    else As[t * ld + ii] = 0.0;
    if (t < w && J0 + ii < m) cp_async8(&Bs[t * ld + ii], col + J0 + ii);
    else Bs[t * ld + ii] = 0.0;
  }
  cp_async_commit();
  for (int t = threadIdx.x; t < kB64; t += blockDim.x) dsh[t] = t < w ? dc[t + t * kB64] : 0.0;
  cp_async_wait<0>();
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wi = (warp & 1) * 32, wj = (warp >> 1) * 16;
  const int g = lane >> 2, tg = lane & 3;
  double acc[4][2][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 2; ++q) acc[a][q][0] = acc[a][q][1] = 0.0;
  // warps whose 32 x 16 sub-tile lies above the diagonal or past the last row skip the products
  const int wk = (I0 + wi >= m || J0 + wj >= m || (I == J && wj > wi + 31)) ? 0 : (w + 3) & ~3;
#pragma unroll 2
  for (int kk = 0; kk < wk; kk += 4) {
    double af[4], bf[2];
    const double dk = dsh[kk + tg];
#pragma unroll
    for (int a = 0; a < 4; ++a) af[a] = As[(kk + tg) * ld + wi + a * 8 + g];
#pragma unroll
    for (int q = 0; q < 2; ++q) bf[q] = Bs[(kk + tg) * ld + wj + q * 8 + g] * dk;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q) mma884(acc[a][q][0], acc[a][q][1], af[a], bf[q]);
  }
  double cv[4][2][2];  // read all targets before writing any (the loads stay in flight together)
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = I0 + wi + a * 8 + g;
        const int j = J0 + wj + q * 8 + tg * 2 + h;
        cv[a][q][h] = (i < m && j < m && i >= j) ? Fs[i + (int64_t)j * m] : 0.0;
      }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int i = I0 + wi + a * 8 + g;
        const int j = J0 + wj + q * 8 + tg * 2 + h;
        if (i < m && j < m && i >= j) Fs[i + (int64_t)j * m] = cv[a][q][h] - acc[a][q][h];
      }
  if (kNext && tile == 0 && c < k) {
    const int wn = min(kB64, k - c);
    double* Ds = smu;             // [64 cols][ld]: the next diagonal block, factored in place
    double* Li = Ds + kB64 * ld;  // its L^-1
    double* U = Li + kB64 * ld;
    double* ws = U + 16 * kULd64;
    __syncthreads();  // the operand tiles are consumed
    for (int e = threadIdx.x; e < kB64 * kB64; e += blockDim.x) {
      Ds[(e & 63) + (e >> 6) * ld] = 0.0;
      Li[(e & 63) + (e >> 6) * ld] = 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wi + a * 8 + g, cc = wj + q * 8 + tg * 2 + h;  // I0 == J0 == c for tile 0
          if (r < wn && cc < wn && r >= cc) Ds[r + cc * ld] = cv[a][q][h] - acc[a][q][h];
        }
    __syncthreads();
    cta_ldlt<true>(Ds, ld, wn, wn, Li, ld, U, kULd64, ws);
    double* D0 = Fs + c + (int64_t)c * m;
    double* lc = const_cast<double*>(linv_block(S, linv, b, s, c / kB64));
    for (int e = threadIdx.x; e < kB64 * kB64; e += blockDim.x) {
      const int cc = e >> 6, r = e & 63;
      const double v = (r < wn && cc < wn) ? Ds[r + cc * ld] : 0.0;
      dc_next[e] = v;
      lc[e] = Li[r + cc * ld];
      if (r < wn && cc < wn && r >= cc) D0[r + (int64_t)cc * m] = v;
    }
  }
}

__global__ void __launch_bounds__(kPersistThreads, 2) k_factor_persist(PersistArgs a) {
  extern __shared__ double psm[];
  __shared__ int sh_task, sh_go;
  const DevSym& S = a.S;
  const int per = a.gstart[a.ngroups];
  const long long total = (long long)a.B * per;
  for (;;) {
    if (threadIdx.x == 0) sh_task = (int)atomicAdd(a.head, 1u);
    __syncthreads();
    const long long t = sh_task;
    if (t >= total) break;
    // group g: the last one with B * gstart[g] <= t
    const int q = (int)(t / a.B);
    int lo = 0, hi = a.ngroups;  // gstart[lo] <= q < gstart[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (a.gstart[mid] <= q) lo = mid;
      else hi = mid;
    }
    const int g = lo, cnt = a.gstart[g + 1] - a.gstart[g];
    const long long j = t - (long long)a.B * a.gstart[g];
    const int b = (int)(j / cnt), i = (int)(j - (long long)b * cnt);
    const PersistTask T = a.task[a.gstart[g] + i];
    int* pg = a.prog + (int64_t)b * S.ns;
    if (threadIdx.x == 0) {
      bool ok = true;
      if (T.type == PT_TINY) {
        for (int u = 0; u < T.sub && ok; ++u) ok = wait_children(a, a.tiny_list[T.s + u], b);
      } else if (T.type == PT_SMALL || T.type == PT_GATHER) {
        ok = wait_children(a, T.s, b);
      } else {
        ok = wait_at_least(pg + T.s, T.need, a.err, a.limit_ns);
      }
      sh_go = ok;
    }
    __syncthreads();
    if (!sh_go) break;
    // (the bodies skip the fronts of inactive (problem, model) pairs themselves: DevSym::active)
    switch (T.type) {
      case PT_TINY: {
        const int warp = threadIdx.x >> 5;
        if (warp < T.sub) {
          double* A = psm + warp * kPersistTinySlice;
          factor_tiny_warp(S, a.tiny_list[T.s + warp], b, a.F, a.fstride, A, A + kTinyM * kTinyLd,
                           reinterpret_cast<int*>(A + kTinyM * kTinyLd + kTinyM));
        }
        break;
      }
      case PT_SMALL:
        factor_small_body<kPersistThreads>(S, T.s, b, a.F, a.fstride, psm);
        break;
      case PT_GATHER:
        gather8_body(S, T.s, b, T.sub, a.F, a.fstride, T.gcols, a.gptr, a.grng, psm);
        break;
      case PT_DIAG:
        panel64_body(S, T.s, b, 0, T.j0, 0, a.F, a.fstride,
                     a.dcache + ((int64_t)a.lid[T.s] * a.B + b) * (kB64 * kB64), a.linv, psm);
        break;
      case PT_ROWS:
        rows64_body(S, T.s, b, T.sub, T.j0, a.F, a.fstride,
                    a.dcache + ((int64_t)a.lid[T.s] * a.B + b) * (kB64 * kB64), a.linv, psm);
        break;
      default:
        update64w8_body(S, T.s, b, T.sub, T.j0, a.F, a.fstride,
                        a.dcache + ((int64_t)a.lid[T.s] * a.B + b) * (kB64 * kB64), psm);
        break;
    }
    __syncthreads();  // every thread's writes of this task are issued
    if (threadIdx.x == 0) {
      __threadfence();
      if (T.type == PT_TINY) {
        for (int u = 0; u < T.sub; ++u) atomicAdd(pg + a.tiny_list[T.s + u], 1);
      } else {
        atomicAdd(pg + T.s, 1);
      }
    }
  }
}

}  // namespace
}  // namespace inla

namespace inla {
namespace {

// ---------------------------------------------------------------------------
// Persistent triangular solve: the forward sweep bottom-up and the backward sweep top-down as
// one task queue (tiny fronts eight per task, one warp each; other fronts one CTA each). A
// forward task waits for its children's forward tasks; a backward task waits for its
// parent's backward task (a root: for its own forward task). Same bounded waits and
// completion counting as the factorization; the bodies are the level kernels' bodies.
// ---------------------------------------------------------------------------
enum SolveTaskType : int { ST_FWD_TINY = 0, ST_FWD = 1, ST_BWD = 2, ST_BWD_TINY = 3 };

struct SolveArgs {
  DevSym S;
  const double* F;
  int64_t fstride;
  int B;
  int ngroups;
  const int* gstart;
  const PersistTask* task;
  const int* tiny_list;
  const double* linv;  // inverse-block cache of the factorization (large fronts)
  double* xp;
  double* ub;
  int64_t ustride;
  int* progf;  // [B][ns] forward sweep done
  int* progb;  // [B][ns] backward sweep done
  unsigned* head;
  int* err;
  long long limit_ns;
};

__device__ bool solve_wait(const SolveArgs& a, int type, int sn, int b) {
  const DevSym& S = a.S;
  const int64_t o = (int64_t)b * S.ns;
  if (type == ST_FWD_TINY || type == ST_FWD) {
    for (int q = S.child_ptr[sn]; q < S.child_ptr[sn + 1]; ++q)
      if (!wait_at_least(a.progf + o + S.child_list[q], 1, a.err, a.limit_ns)) return false;
    return true;
  }
  const int p = S.parent[sn];
  if (p < 0 || p >= S.ns) return wait_at_least(a.progf + o + sn, 1, a.err, a.limit_ns);
  return wait_at_least(a.progb + o + p, 1, a.err, a.limit_ns);
}

__global__ void __launch_bounds__(kPersistThreads, 2) k_solve_persist(SolveArgs a) {
  extern __shared__ double ssm[];
  __shared__ int sh_task, sh_go;
  const DevSym& S = a.S;
  const int per = a.gstart[a.ngroups];
  const long long total = (long long)a.B * per;
  for (;;) {
    if (threadIdx.x == 0) sh_task = (int)atomicAdd(a.head, 1u);
    __syncthreads();
    const long long t = sh_task;
    if (t >= total) break;
    const int q = (int)(t / a.B);
    int lo = 0, hi = a.ngroups;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (a.gstart[mid] <= q) lo = mid;
      else hi = mid;
    }
    const int g = lo, cnt = a.gstart[g + 1] - a.gstart[g];
    const long long j = t - (long long)a.B * a.gstart[g];
    const int b = (int)(j / cnt), i = (int)(j - (long long)b * cnt);
    const PersistTask T = a.task[a.gstart[g] + i];
    const bool tiny = T.type == ST_FWD_TINY || T.type == ST_BWD_TINY;
    if (threadIdx.x == 0) {
      bool ok = true;
      if (tiny) {
        for (int u = 0; u < T.sub && ok; ++u) ok = solve_wait(a, T.type, a.tiny_list[T.s + u], b);
      } else {
        ok = solve_wait(a, T.type, T.s, b);
      }
      sh_go = ok;
    }
    __syncthreads();
    if (!sh_go) break;
    const int warp = threadIdx.x >> 5;
    switch (T.type) {
      case ST_FWD_TINY:
        if (warp < T.sub)
          fwd_tiny_warp(S, a.tiny_list[T.s + warp], b, a.F, a.fstride, a.xp, a.ub, a.ustride, ssm + 32 * warp);
        break;
      case ST_FWD:
        if (S.lbo[T.s] >= 0) fwd64_body<kPersistThreads, false>(S, T.s, b, a.F, a.fstride, a.linv, a.xp, a.ub, a.ustride, ssm);
        else fwd32_body<kPersistThreads>(S, T.s, b, a.F, a.fstride, a.xp, a.ub, a.ustride, ssm);
        break;
      case ST_BWD:
        if (S.lbo[T.s] >= 0) bwd64_body<kPersistThreads, false>(S, T.s, b, a.F, a.fstride, a.linv, a.xp, ssm);
        else bwd32_body<kPersistThreads>(S, T.s, b, a.F, a.fstride, a.xp, ssm);
        break;
      default:
        if (warp < T.sub) bwd_tiny_warp(S, a.tiny_list[T.s + warp], b, a.F, a.fstride, a.xp);
        break;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      int* pc = (T.type == ST_FWD_TINY || T.type == ST_FWD ? a.progf : a.progb) + (int64_t)b * S.ns;
      if (tiny) {
        for (int u = 0; u < T.sub; ++u) atomicAdd(pc + a.tiny_list[T.s + u], 1);
      } else {
        atomicAdd(pc + T.s, 1);
      }
    }
  }
}

}  // namespace
}  // namespace inla
