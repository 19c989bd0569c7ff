// Host orchestration of the batched supernodal kernels.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <list>
#include <mutex>

#include "gpu_factor.hpp"
#include "host_par.hpp"
#include "snode_kernels.cuh"
#include "snode_large.cuh"
#include "snode_persist.cuh"

namespace inla {

namespace {
inline int cdiv(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Panel forms of a level's large fronts (entries of the per-level schedule).
constexpr char kFormSplit = 0, kFormFused = 1, kFormLookahead = 2, kNumForms = 3;
// Process-wide panel form for engines built from now on: -1 the autotuner's choice per level
// (default), otherwise that form at every level.
std::atomic<int> g_panel_form{-1};

// Trailing-update tile on eight warps (32 x 16 warp tiles; the body the persistent schedule
// runs too), two CTAs per SM: 16 warps per SM where the four-warp form with 32 x 32 warp tiles
// fitted 12 (168 registers, 70 KB of staging). Measured on the SPDE 200^2 factorization: 7 %
// faster at B = 1, 3 % at B = 7, 2 % at B = 21.
__global__ void __launch_bounds__(256, 2) k_update64w8(DevSym S, const int* __restrict__ list, int j0,
                                                         double* __restrict__ F, int64_t fstride,
                                                         const double* __restrict__ dcache) {
  extern __shared__ double smu[];
  const double* dc = dcache + ((int64_t)blockIdx.x * gridDim.y + blockIdx.y) * (kB64 * kB64);
  update64w8_body(S, list[blockIdx.x], blockIdx.y, blockIdx.z, j0, F, fstride, dc, smu);
}

// The same update with look-ahead: tile 0 of every (front, problem) also factors the next
// diagonal block (D and L into the other cache slot, L^-1 into the inverse-block cache), so the
// pivot chain of block J + 1 runs while the other tiles of step J are updated and the step
// after needs no diagonal-block launch. Results are bit-identical to the split form.
__global__ void __launch_bounds__(256, 2) k_update64la(DevSym S, const int* __restrict__ list, int j0,
                                                         double* __restrict__ F, int64_t fstride,
                                                         const double* __restrict__ dcache,
                                                         double* __restrict__ dcache_next, double* __restrict__ linv) {
  extern __shared__ double smu[];
  const int64_t slot = ((int64_t)blockIdx.x * gridDim.y + blockIdx.y) * (kB64 * kB64);
  update64w8_body<true>(S, list[blockIdx.x], blockIdx.y, blockIdx.z, j0, F, fstride, dcache + slot, smu,
                        dcache_next + slot, linv);
}

// Parent columns per extend-add CTA: the m-row slice must fit in shared memory.
inline int gather_cols(int m) { return std::max(1, std::min(kGatherCols, (200 * 1024) / (8 * std::max(m, 1)))); }

// The dynamic shared-memory limit is an attribute of the kernel on the current
// device, shared by every engine in the process. Engines of different sizes
// need different limits, so the attribute only ever rises: a smaller engine
// built later must not lower it below what a larger one still launches with.
std::mutex g_smem_mu;
std::map<std::pair<const void*, int>, int> g_smem_set;  // (kernel, device) -> limit set

template <class K>
void set_smem(K kernel, int bytes) {
  int dev = 0;
  INLA_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_smem_mu);
  int& cur = g_smem_set[{(const void*)kernel, dev}];
  if (bytes <= cur) return;
  INLA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  cur = bytes;
}
}  // namespace

// Host tables of a symbolic analysis that the engine uploads (32-bit supernode arrays, front
// offsets, the panel map and the front positions of the input entries). They depend on the
// analysis only, so they are built once per analysis id and shared by every engine created on
// it (a model rebuilt on the same mesh skips the ~10-20 ms of building them); at most
// kMapsCacheBytes are kept, most recently used first.
namespace {
constexpr size_t kMapsCacheBytes = size_t(1) << 30;
std::mutex g_maps_mu;
std::list<std::pair<uint64_t, std::shared_ptr<const HostMaps>>> g_maps;
size_t g_maps_bytes = 0;

size_t host_maps_bytes(const HostMaps& M) {
  return sizeof(int) * (M.first.size() + M.rowptr.size() + M.rows.size() + M.relx.size() + M.child_ptr.size() +
                        M.child_list.size() + M.parent.size() + M.uoff.size() + M.perm.size() + M.pmap.size()) +
         sizeof(int64_t) * (M.fptr.size() + M.lptr.size() + M.dpos.size() + M.spos.size() + M.spos_full.size());
}

std::shared_ptr<const HostMaps> build_host_maps(const Symbolic& S) {
  auto out = std::make_shared<HostMaps>();
  HostMaps& M = *out;
  const int64_t ns = S.nsuper, n = S.n;
  const int64_t nnz_ = (int64_t)S.rowidx.size();
  std::vector<int>&first = M.first, &rowptr = M.rowptr, &rows = M.rows, &relx = M.relx, &child_ptr = M.child_ptr,
                   &child_list = M.child_list, &parent = M.parent, &uoff = M.uoff, &perm = M.perm;
  std::vector<int64_t>&fptr = M.fptr, &lptr = M.lptr, &dpos = M.dpos;
  first.resize(ns + 1);
  rowptr.resize(ns + 1);
  rows.resize(S.sn_rows.size());
  relx.assign(S.sn_rows.size(), -1);
  child_ptr.resize(ns + 1);
  child_list.resize(S.child_list.size());
  parent.resize(ns);
  uoff.assign(ns + 1, 0);
  perm.resize(n);
  fptr.assign(ns + 1, 0);
  lptr.resize(ns + 1);
  dpos.resize(n);
  for (int64_t s = 0; s <= ns; ++s) {
    first[s] = (int)S.sn_first[s];
    rowptr[s] = (int)S.sn_rowptr[s];
    child_ptr[s] = (int)S.child_ptr[s];
    lptr[s] = S.sn_lptr[s];
  }
  for (size_t i = 0; i < S.sn_rows.size(); ++i) rows[i] = (int)S.sn_rows[i];
  for (size_t i = 0; i < S.child_list.size(); ++i) child_list[i] = (int)S.child_list[i];
  for (int64_t s = 0; s < ns; ++s) {
    int64_t k = S.sn_first[s + 1] - S.sn_first[s], m = S.sn_rowptr[s + 1] - S.sn_rowptr[s];
    parent[s] = (int)S.sn_parent[s];
    fptr[s + 1] = fptr[s] + m * m;
    uoff[s + 1] = uoff[s] + (int)(m - k);
    for (int64_t t = 0; t < m - k; ++t) relx[S.sn_rowptr[s] + k + t] = S.rel[S.rel_ptr[s] + t];
    for (int64_t j = S.sn_first[s]; j < S.sn_first[s + 1]; ++j) {
      int64_t c = j - S.sn_first[s];
      dpos[j] = fptr[s] + c * (m + 1);
    }
  }
  for (int64_t j = 0; j < n; ++j) perm[j] = (int)S.perm[j];

  // panel map (compact panel index -> input entry) and front positions of input entries
  std::vector<int>& pmap = M.pmap;
  std::vector<int64_t>&spos = M.spos, &spos_full = M.spos_full;
  pmap.assign(S.nnz_l_stored, -1);
  spos.assign(nnz_, -1);
  spos_full.assign(nnz_, -1);
  parallel_for(n, [&](int64_t c0, int64_t c1) {  // disjoint writes: entry p, panel slot qmap[p]
    for (int64_t c = c0; c < c1; ++c)
      for (int64_t p = S.colptr[c]; p < S.colptr[c + 1]; ++p) {
        int64_t i = S.iperm[S.rowidx[p]], j = S.iperm[c];
        int64_t lo = std::min(i, j), hi = std::max(i, j);
        int64_t s = S.col_to_sn[lo];
        const int64_t* R = S.sn_rows.data() + S.sn_rowptr[s];
        int64_t m = S.sn_rowptr[s + 1] - S.sn_rowptr[s];
        const int64_t* it = std::lower_bound(R, R + m, hi);
        if (it == R + m || *it != hi) throw std::runtime_error("entry outside the filled pattern");
        spos_full[p] = fptr[s] + (lo - S.sn_first[s]) * m + (it - R);
        int64_t q = S.qmap[p];
        if (q < 0) continue;
        pmap[q] = (int)p;
        spos[p] = spos_full[p];
      }
  });
  return out;
}
}  // namespace

void release_host_maps() {
  std::lock_guard<std::mutex> lk(g_maps_mu);
  g_maps.clear();
  g_maps_bytes = 0;
}

std::shared_ptr<const HostMaps> host_maps(const Symbolic& S) {
  // without the symbolic cache every engine has an analysis of its own: nothing to share
  static const bool on = std::getenv("INLA_NO_SYMBOLIC_CACHE") == nullptr;
  if (!on) return build_host_maps(S);
  if (S.id != 0) {
    std::lock_guard<std::mutex> lk(g_maps_mu);
    for (auto it = g_maps.begin(); it != g_maps.end(); ++it)
      if (it->first == S.id) {
        g_maps.splice(g_maps.begin(), g_maps, it);
        return g_maps.front().second;
      }
  }
  std::shared_ptr<const HostMaps> m = build_host_maps(S);
  if (S.id != 0) {
    const size_t bytes = host_maps_bytes(*m);
    std::lock_guard<std::mutex> lk(g_maps_mu);
    if (bytes <= kMapsCacheBytes / 2) {
      g_maps.emplace_front(S.id, m);
      g_maps_bytes += bytes;
      while (g_maps_bytes > kMapsCacheBytes && g_maps.size() > 1) {
        g_maps_bytes -= host_maps_bytes(*g_maps.back().second);
        g_maps.pop_back();
      }
    }
  }
  return m;
}

GpuFactor::GpuFactor(const Symbolic& sym, int max_batch, cudaStream_t stream)
    : sym_(sym), max_batch_(max_batch), stream_(stream) {
  const auto tstart = std::chrono::steady_clock::now();
  if (max_batch < 1) throw std::runtime_error("max_batch must be >= 1");
  const Symbolic& S = sym_;
  const int64_t ns = S.nsuper, n = S.n;
  nnz_ = (int64_t)S.rowidx.size();
  if (n >= (1LL << 31) || (int64_t)S.sn_rows.size() >= (1LL << 31) || nnz_ >= (1LL << 31))
    throw std::runtime_error("problem too large for 32-bit indices");
  if (S.max_m > 25600) throw std::runtime_error("front with more than 25600 rows (extend-add slice exceeds shared memory)");

  const std::shared_ptr<const HostMaps> maps = host_maps(S);
  const HostMaps& M = *maps;
  const std::vector<int>&first = M.first, &rowptr = M.rowptr, &rows = M.rows, &relx = M.relx,
                  &child_ptr = M.child_ptr, &child_list = M.child_list, &parent = M.parent, &uoff = M.uoff,
                  &perm = M.perm, &pmap = M.pmap;
  const std::vector<int64_t>&fptr = M.fptr, &lptr = M.lptr, &dpos = M.dpos, &spos = M.spos,
                      &spos_full = M.spos_full;
  ftotal_ = fptr[ns];
  usum_ = uoff[ns];

  const auto tm1 = std::chrono::steady_clock::now();
  d_first_.upload(first, stream_);
  d_rowptr_.upload(rowptr, stream_);
  d_rows_.upload(rows, stream_);
  d_relx_.upload(relx, stream_);
  d_child_ptr_.upload(child_ptr, stream_);
  d_child_list_.upload(child_list, stream_);
  d_parent_.upload(parent, stream_);
  d_uoff_.upload(uoff, stream_);
  d_perm_.upload(perm, stream_);
  d_fptr_.upload(fptr, stream_);
  d_lptr_.upload(lptr, stream_);
  d_dpos_.upload(dpos, stream_);
  d_pmap_.upload(pmap, stream_);
  spos_.upload(spos, stream_);
  spos_full_.upload(spos_full, stream_);

  ds_.n = (int)n;
  ds_.ns = (int)ns;
  ds_.first = d_first_.p;
  ds_.rowptr = d_rowptr_.p;
  ds_.rows = d_rows_.p;
  ds_.relx = d_relx_.p;
  ds_.fptr = d_fptr_.p;
  ds_.lptr = d_lptr_.p;
  ds_.child_ptr = d_child_ptr_.p;
  ds_.child_list = d_child_list_.p;
  ds_.parent = d_parent_.p;
  ds_.uoff = d_uoff_.p;
  ds_.dpos = d_dpos_.p;
  ds_.perm = d_perm_.p;

  const auto tm2 = std::chrono::steady_clock::now();
  // inverse-block cache: one 64 x 64 block per 64 pivot columns of every large front
  {
    std::vector<int> lbo(ns, -1);
    int64_t nblk = 0;
    for (int64_t s = 0; s < ns; ++s) {
      const int64_t k = S.sn_first[s + 1] - S.sn_first[s], m = S.sn_rowptr[s + 1] - S.sn_rowptr[s];
      if (m > kSmallB) {
        lbo[s] = (int)nblk;
        nblk += cdiv(k, kB64);
      }
    }
    d_lbo_.upload(lbo, stream_);
    ds_.lbo = d_lbo_.p;
    ds_.lstride = nblk * kB64 * kB64;
    linv_.alloc((size_t)max_batch_ * std::max<int64_t>(ds_.lstride, 1));
  }
  // value-fill chunks over the compact panel numbering (kFillChunk entries for
  // the input-values fill, kFillModelChunk for the component-model fill)
  {
    ntot_ = S.sn_lptr[ns];
    auto chunk_table = [&](int chunk, int& count, DBuf<int>& dst) {
      count = std::max(1, cdiv(ntot_, chunk));
      std::vector<int> csn(count + 1);
      int64_t s = 0;
      for (int c = 0; c < count; ++c) {
        const int64_t e = (int64_t)c * chunk;
        while (s + 1 < ns && S.sn_lptr[s + 1] <= e) ++s;
        csn[c] = (int)s;
      }
      csn[count] = (int)(ns - 1);
      dst.upload(csn, stream_);
    };
    chunk_table(kFillChunk, nfill_, d_csn_);
    chunk_table(kFillModelChunk, nfillm_, d_csnm_);
  }
  nldchunk_ = std::max(1, cdiv(n, kLogdetChunk));
  ldpart_.alloc((size_t)max_batch_ * nldchunk_);
  ldflag_.alloc((size_t)max_batch_ * nldchunk_);
  ldticket_.alloc((size_t)max_batch_);
  INLA_CUDA(cudaMemsetAsync(ldticket_.p, 0, sizeof(unsigned) * max_batch_, stream_));

  const auto tm3 = std::chrono::steady_clock::now();
  plan_levels();
  // extend-add range table: for every large front, column chunk z (of the
  // level's gcols columns) and child, the child's source columns whose parent
  // column lies in the chunk
  {
    std::vector<int64_t> gptr(ns, 0);
    std::vector<int2> grng;
    for (const LevelPlan& P : levels_) {
      if (P.large.empty()) continue;
      const int gcols = gather_cols(P.mmax_large);
      for (int s : P.large) {
        const int m = rowptr[s + 1] - rowptr[s];
        gptr[s] = (int64_t)grng.size();
        for (int z = 0; z < cdiv(m, gcols); ++z) {
          const int c0 = z * gcols, c1 = std::min(c0 + gcols, m);
          for (int64_t q = S.child_ptr[s]; q < S.child_ptr[s + 1]; ++q) {
            const int c = (int)S.child_list[q];
            const int kc = first[c + 1] - first[c], rc = (rowptr[c + 1] - rowptr[c]) - kc;
            const int* rel = relx.data() + rowptr[c] + kc;
            const int lo = (int)(std::lower_bound(rel, rel + rc, c0) - rel);
            const int hi = (int)(std::lower_bound(rel, rel + rc, c1) - rel);
            grng.push_back(make_int2(lo, hi));
          }
        }
      }
    }
    if (grng.empty()) grng.push_back(make_int2(0, 0));
    d_gptr_.upload(gptr, stream_);
    d_grng_.upload(grng, stream_);
  }

  panel_form_ = g_panel_form.load();
  plan_persist();
  const auto ta = std::chrono::steady_clock::now();
  F_.alloc((size_t)max_batch_ * ftotal_);
  xp_.alloc((size_t)max_batch_ * n);
  ub_.alloc((size_t)max_batch_ * std::max<int64_t>(usum_, 1));
  logdet_.alloc(max_batch_);
  status_.alloc(max_batch_);

  {
    int64_t nlmax = 1, ppmax = 1, gpmax = 1, cmax = 1;
    int sms = 0, dev = 0;
    INLA_CUDA(cudaGetDevice(&dev));
    INLA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (const LevelPlan& P : levels_) {
      nlmax = std::max<int64_t>(nlmax, (int64_t)P.large.size());
      ppmax = std::max<int64_t>(ppmax, (int64_t)P.si_large.size() * cdiv(P.mmax_si_large, kSiT));
      const int64_t nls = (int64_t)P.si_large.size(), pt = cdiv(P.mmax_si_large, kSiT);
      // split launches have nls * B * pt <= SM count: B <= bmax
      const int64_t bmax = std::min<int64_t>(max_batch_, sms / std::max<int64_t>(1, nls * pt));
      const int sm = si_nsplit(cdiv(P.mmax_si_large, 32), bmax >= 1);
      if (sm > 1) gpmax = std::max<int64_t>(gpmax, nls * pt * sm * bmax);
      cmax = std::max<int64_t>(cmax, nls * pt);
    }
    // two slots: the look-ahead form factors block J + 1 while step J still reads block J
    dslot_ = nlmax * max_batch_ * kB64 * kB64;
    dcache_.alloc((size_t)(2 * dslot_));
    ppart_.alloc((size_t)ppmax * max_batch_ * kB64 * kB64);
    gpart_.alloc((size_t)gpmax * kB64 * kB64);
    sicnt_.alloc((size_t)cmax * max_batch_);
    INLA_CUDA(cudaMemsetAsync(sicnt_.p, 0, sizeof(int) * (size_t)cmax * max_batch_, stream_));
  }
  set_smem(k_factor_small<128>, small_factor_smem(kSmallA));
  set_smem(k_factor_small<256>, small_factor_smem(kSmallB));
  set_smem(k_selinv_small<256>, small_selinv_smem(kSiSmall, kSiSmall));
  set_smem(k_panel64, kPanelSmem);
  {
    int dev = 0;
    INLA_CUDA(cudaGetDevice(&dev));
    INLA_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
  }
  {  // key of the tuning table: FNV-1a over the supernode partition and row counts
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](int64_t v) {
      for (int b = 0; b < 8; ++b) h = (h ^ (uint64_t)((v >> (8 * b)) & 0xff)) * 1099511628211ull;
    };
    mix(n);
    mix(ns);
    mix(num_sms_);
    for (int64_t s = 0; s <= ns; ++s) mix(S.sn_first[s]), mix(S.sn_rowptr[s]);
    struct_hash_ = h;
  }
  set_smem(k_update64w8, kPersistUpdSmem);
  set_smem(k_update64la, kPanelSmem);
  set_smem(k_rows64, kRowsSmem);
  set_smem(k_fwd32<128>, (int)((S.max_m + 2 + 32 * 33) * 8));
  set_smem(k_bwd32<128>, (int)((S.max_m + 2 + 32 * 33) * 8));
  set_smem(k_fwd64<256, true>, (int)((S.max_m + 2) * 8));
  set_smem(k_fwd64<256, false>, (int)((S.max_m + 2) * 8));
  set_smem(k_bwd64<256, true>, (int)((S.max_m + 2) * 8));
  set_smem(k_bwd64<256, false>, (int)((S.max_m + 2) * 8));
  set_smem(k_gather8, 200 * 1024 + 8 * kGatherCols * 8);
  set_smem(k_si_step64, kSiGemmSmem);
  set_smem(k_si_diag64, kSiDiagSmem);
  if (persist_) {
    set_smem(k_factor_persist, persist_smem_);
    int per_sm = 0;
    INLA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_factor_persist, kPersistThreads,
                                                            persist_smem_));
    persist_grid_ = std::max(1, per_sm) * num_sms_;
    if (per_sm < 1) persist_ = false;
  }
  if (solve_persist_) {
    set_smem(k_solve_persist, solve_smem_);
    int per_sm = 0;
    INLA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_persist, kPersistThreads, solve_smem_));
    solve_grid_ = std::max(1, per_sm) * num_sms_;
    if (per_sm < 1) solve_persist_ = false;
  }
  INLA_CUDA(cudaStreamSynchronize(stream_));
  if (std::getenv("INLA_DEBUG"))
    std::fprintf(stderr, "device factor: maps %.1f ms, symbolic uploads %.1f ms, caches %.1f ms, levels %.1f ms, buffers %.1f ms (%d slots)\n",
                 std::chrono::duration<double, std::milli>(tm1 - tstart).count(),
                 std::chrono::duration<double, std::milli>(tm2 - tm1).count(),
                 std::chrono::duration<double, std::milli>(tm3 - tm2).count(),
                 std::chrono::duration<double, std::milli>(ta - tm3).count(),
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta).count(),
                 max_batch_);
}

GpuFactor::~GpuFactor() {
  for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second.exec);
}

// Level plans of a symbolic analysis (host lists; offsets into the flattened device list).
std::vector<LevelPlan> make_level_plans(const Symbolic& S, std::vector<int>& flat) {
  std::vector<LevelPlan> levels(S.nlevels);
  flat.clear();
  // fronts of at most kTinyM rows: one warp each (INLA_NO_TINY_FRONTS keeps them on k_factor_small)
  static const bool tiny_on = std::getenv("INLA_NO_TINY_FRONTS") == nullptr;
  constexpr int kSmallA = GpuFactor::kSmallA, kSmallB = GpuFactor::kSmallB, kSiSmall = GpuFactor::kSiSmall;
  for (int32_t l = 0; l < S.nlevels; ++l) {
    LevelPlan& P = levels[l];
    for (int64_t t = S.level_ptr[l]; t < S.level_ptr[l + 1]; ++t) {
      int s = (int)S.level_list[t];
      int k = (int)(S.sn_first[s + 1] - S.sn_first[s]);
      int m = (int)(S.sn_rowptr[s + 1] - S.sn_rowptr[s]);
      P.all.push_back(s);
      P.mmax_all = std::max(P.mmax_all, m);
      if (!(tiny_on && m <= kTinyM)) {
        P.nontiny.push_back(s);
        P.mmax_nontiny = std::max(P.mmax_nontiny, m);
      }
      if (tiny_on && m <= kTinyM) {
        P.tiny.push_back(s);
      } else if (m <= kSmallA) {
        P.small_a.push_back(s);
        P.mmax_a = std::max(P.mmax_a, m);
      } else if (m <= kSmallB) {
        P.small_b.push_back(s);
        P.mmax_b = std::max(P.mmax_b, m);
      } else {
        P.large.push_back(s);
        P.kmax_large = std::max(P.kmax_large, k);
        P.mmax_large = std::max(P.mmax_large, m);
      }
      if (tiny_on && m <= kTinyM) {
        P.si_tiny.push_back(s);
      } else if (m <= kSiSmall) {
        P.si_small.push_back(s);
        P.mmax_si_small = std::max(P.mmax_si_small, m);
        P.kmax_si_small = std::max(P.kmax_si_small, k);
      } else {
        P.si_large.push_back(s);
        P.kmax_si_large = std::max(P.kmax_si_large, k);
        P.mmax_si_large = std::max(P.mmax_si_large, m);
        P.rmax_si_large = std::max(P.rmax_si_large, m - k);
      }
    }
    auto put = [&](const std::vector<int>& v) {
      int off = (int)flat.size();
      flat.insert(flat.end(), v.begin(), v.end());
      return off;
    };
    P.off_tiny = put(P.tiny);
    P.off_small_a = put(P.small_a);
    P.off_small_b = put(P.small_b);
    P.off_large = put(P.large);
    P.off_all = put(P.all);
    P.off_nontiny = put(P.nontiny);
    P.off_si_tiny = put(P.si_tiny);
    P.off_si_small = put(P.si_small);
    P.off_si_large = put(P.si_large);
  }
  return levels;
}

void GpuFactor::plan_levels() {
  std::vector<int> flat;
  levels_ = make_level_plans(sym_, flat);
  d_lists_.upload(flat, stream_);
}

// ---------------------------------------------------------------------------
// Persistent schedule: the task queue of k_factor_persist (see snode_persist.cuh).
// Per level: tiny fronts in groups of eight, small fronts, then the large fronts phase by
// phase (extend-add chunks; per 64-column block the diagonal block, the row blocks and the
// trailing-update tiles). Each phase of a level is one group; within a group the tasks of
// problem 0 come first, then problem 1, and so on.
// ---------------------------------------------------------------------------
namespace {
// Process-wide schedule mode for engines built from now on: 0 level launches only, 1 measured
// per batch size (default), 2 persistent wherever it fits. INLA_NO_PERSIST in the environment
// starts it at 0; inla_set_persistent_schedule changes it.
std::atomic<int> g_persist_default{-1};
// measured choice per (supernodal structure, batch size): true = persistent
std::mutex g_sched_mu;
std::map<std::pair<uint64_t, int>, bool> g_sched;
}  // namespace

void set_persistent_default(int mode) { g_persist_default.store(mode < 0 ? 0 : (mode > 2 ? 2 : mode)); }

void set_panel_form(int form) { g_panel_form.store(form < 0 || form >= kNumForms ? -1 : form); }

// The task queue of the persistent schedule for one problem (host arrays).
bool make_persist_plan(const Symbolic& S, const std::vector<LevelPlan>& levels, PersistPlan& out) {
  const int ns = (int)S.nsuper;
  constexpr int kGatherBudget = 110 * 1024;  // bytes of one extend-add column slice
  int smem = std::max({kPersistTinySmem, small_factor_smem(GpuFactor::kSmallB), kPanelSmem, kRowsSmem,
                       kPersistUpdSmem});
  PersistPlan& pl = out;
  pl = PersistPlan();
  pl.gstart = {0};
  pl.total.assign(ns, 0);
  pl.lid.assign(ns, -1);
  pl.gptr.assign(ns, 0);
  auto push = [&](int type, int sn, int sub, int need, int j0, int gcols) {
    pl.task.insert(pl.task.end(), {type, sn, sub, need, j0, gcols});
  };
  auto close_group = [&] {
    const int cnt = (int)(pl.task.size() / 6);
    if (cnt > pl.gstart.back()) pl.gstart.push_back(cnt);
  };
  struct Phase {
    int type, count, j0;
  };
  for (const LevelPlan& P : levels) {
    for (size_t i = 0; i < P.tiny.size(); i += kPersistTinyWarps) {
      const int cnt = (int)std::min<size_t>(kPersistTinyWarps, P.tiny.size() - i);
      push(PT_TINY, (int)pl.tiny.size(), cnt, 0, 0, 0);
      for (int u = 0; u < cnt; ++u) {
        pl.tiny.push_back(P.tiny[i + u]);
        pl.total[P.tiny[i + u]] = 1;
      }
    }
    close_group();
    for (const std::vector<int>* v : {&P.small_a, &P.small_b})
      for (int sn : *v) {
        push(PT_SMALL, sn, 0, 0, 0, 0);
        pl.total[sn] = 1;
      }
    close_group();
    if (P.large.empty()) continue;
    // phases of every large front: 0 extend-add, then (diagonal, rows, update) per block
    std::vector<std::vector<Phase>> ph(P.large.size());
    std::vector<int> gc(P.large.size());
    size_t maxp = 0;
    for (size_t f = 0; f < P.large.size(); ++f) {
      const int sn = P.large[f];
      const int k = (int)(S.sn_first[sn + 1] - S.sn_first[sn]), m = (int)(S.sn_rowptr[sn + 1] - S.sn_rowptr[sn]);
      const int gcols = std::max(1, std::min(kGatherCols, kGatherBudget / (8 * m)));
      gc[f] = gcols;
      smem = std::max(smem, gcols * m * 8);
      pl.lid[sn] = pl.nlarge++;
      const int nz = cdiv(m, gcols);
      pl.gptr[sn] = (int64_t)pl.grng.size();
      for (int z = 0; z < nz; ++z) {
        const int c0 = z * gcols, c1 = std::min(c0 + gcols, m);
        for (int64_t q = S.child_ptr[sn]; q < S.child_ptr[sn + 1]; ++q) {
          const int c = (int)S.child_list[q];
          const int kc = (int)(S.sn_first[c + 1] - S.sn_first[c]);
          const int rc = (int)(S.sn_rowptr[c + 1] - S.sn_rowptr[c]) - kc;
          const int32_t* rel = S.rel.data() + S.rel_ptr[c];
          const int lo = (int)(std::lower_bound(rel, rel + rc, c0) - rel);
          const int hi = (int)(std::lower_bound(rel, rel + rc, c1) - rel);
          pl.grng.push_back(make_int2(lo, hi));
        }
      }
      ph[f].push_back({PT_GATHER, nz, 0});
      for (int j0 = 0; j0 < k; j0 += kB64) {
        const int w = std::min(kB64, k - j0), below = std::max(m - j0 - w, 0);
        const int nt = cdiv(below, kUT64);
        ph[f].push_back({PT_DIAG, 1, j0});
        ph[f].push_back({PT_ROWS, cdiv(below, kPanelRows), j0});
        ph[f].push_back({PT_UPDATE, std::max(1, nt * (nt + 1) / 2), j0});
      }
      maxp = std::max(maxp, ph[f].size());
      int tot = 0;
      for (const Phase& x : ph[f]) tot += x.count;
      pl.total[sn] = tot;
    }
    std::vector<int> done(P.large.size(), 0);
    for (size_t p = 0; p < maxp; ++p) {
      for (size_t f = 0; f < P.large.size(); ++f) {
        if (p >= ph[f].size()) continue;
        const Phase& x = ph[f][p];
        for (int u = 0; u < x.count; ++u) push(x.type, P.large[f], u, done[f], x.j0, gc[f]);
        done[f] += x.count;
      }
      close_group();
    }
  }
  pl.smem = smem;
  if (pl.tiny.empty()) pl.tiny.push_back(0);
  if (pl.grng.empty()) pl.grng.push_back(make_int2(0, 0));
  return smem <= 227 * 1024 && pl.gstart.size() > 1;
}

// Host check of the schedule's invariants: processed one task at a time in queue order (one
// problem), every task's dependencies are complete when it is reached (so the smallest
// unfinished task of the GPU queue can always run), every front ends with its completion count,
// and every table index is in range. Returns an empty string or the first violation.
std::string check_persist_plan(const Symbolic& S, const PersistPlan& pl) {
  const int ns = (int)S.nsuper;
  const int ntask = (int)(pl.task.size() / 6);
  if (pl.gstart.back() != ntask) return "group table does not cover the tasks";
  for (size_t g = 0; g + 1 < pl.gstart.size(); ++g)
    if (pl.gstart[g + 1] <= pl.gstart[g]) return "empty or decreasing group " + std::to_string(g);
  std::vector<int> prog(ns, 0);
  auto children_done = [&](int sn) {
    for (int64_t q = S.child_ptr[sn]; q < S.child_ptr[sn + 1]; ++q) {
      const int c = (int)S.child_list[q];
      if (prog[c] != pl.total[c]) return false;
    }
    return true;
  };
  for (int t = 0; t < ntask; ++t) {
    const int* T = pl.task.data() + 6 * t;
    const int type = T[0], sn = T[1], sub = T[2], need = T[3];
    const std::string at = "task " + std::to_string(t) + ": ";
    if (type == PT_TINY) {
      if (sub < 1 || sub > kPersistTinyWarps || sn < 0 || sn + sub > (int)pl.tiny.size()) return at + "tiny range";
      for (int u = 0; u < sub; ++u) {
        const int f = pl.tiny[sn + u];
        if (f < 0 || f >= ns || !children_done(f)) return at + "tiny front before its children";
        const int m = (int)(S.sn_rowptr[f + 1] - S.sn_rowptr[f]);
        if (m > kTinyM) return at + "front too large for a warp";
      }
      for (int u = 0; u < sub; ++u) ++prog[pl.tiny[sn + u]];
      continue;
    }
    if (sn < 0 || sn >= ns) return at + "front out of range";
    const int k = (int)(S.sn_first[sn + 1] - S.sn_first[sn]), m = (int)(S.sn_rowptr[sn + 1] - S.sn_rowptr[sn]);
    if (type == PT_SMALL) {
      if (m > GpuFactor::kSmallB) return at + "front too large for the small body";
      if (!children_done(sn)) return at + "small front before its children";
    } else if (type == PT_GATHER) {
      if (pl.lid[sn] < 0 || !children_done(sn)) return at + "extend-add before the children";
      const int gcols = T[5], nch = (int)(S.child_ptr[sn + 1] - S.child_ptr[sn]);
      if (gcols < 1 || (int64_t)gcols * m * 8 > pl.smem) return at + "extend-add slice exceeds shared memory";
      if (sub >= cdiv(m, gcols) || pl.gptr[sn] + (int64_t)(sub + 1) * nch > (int64_t)pl.grng.size())
        return at + "extend-add chunk out of range";
      if (need != 0 || prog[sn] != sub) return at + "extend-add count";
    } else if (type == PT_DIAG || type == PT_ROWS || type == PT_UPDATE) {
      if (pl.lid[sn] < 0) return at + "step of a front that is not large";
      if (T[4] < 0 || T[4] >= k || T[4] % kB64) return at + "block column out of range";
      if (prog[sn] < need) return at + "phase before its predecessors";
    } else {
      return at + "unknown task type";
    }
    ++prog[sn];
  }
  for (int sn = 0; sn < ns; ++sn)
    if (pl.total[sn] < 1 || prog[sn] != pl.total[sn]) return "front " + std::to_string(sn) + " incomplete";
  return std::string();
}

void make_solve_plan(const Symbolic& S, const std::vector<LevelPlan>& levels, PersistPlan& pl) {
  pl = PersistPlan();
  pl.gstart = {0};
  auto push = [&](int type, int sn, int sub) { pl.task.insert(pl.task.end(), {type, sn, sub, 0, 0, 0}); };
  auto close_group = [&] {
    const int cnt = (int)(pl.task.size() / 6);
    if (cnt > pl.gstart.back()) pl.gstart.push_back(cnt);
  };
  auto tiny_tasks = [&](const std::vector<int>& v, int type) {
    for (size_t i = 0; i < v.size(); i += kPersistTinyWarps) {
      const int cnt = (int)std::min<size_t>(kPersistTinyWarps, v.size() - i);
      push(type, (int)pl.tiny.size(), cnt);
      for (int u = 0; u < cnt; ++u) pl.tiny.push_back(v[i + u]);
    }
    close_group();
  };
  int mmax = 0;
  for (const LevelPlan& P : levels) {
    tiny_tasks(P.tiny, ST_FWD_TINY);
    for (int sn : P.nontiny) push(ST_FWD, sn, 0);
    close_group();
    mmax = std::max(mmax, P.mmax_nontiny);
  }
  for (size_t l = levels.size(); l-- > 0;) {
    for (int sn : levels[l].nontiny) push(ST_BWD, sn, 0);
    close_group();
    tiny_tasks(levels[l].tiny, ST_BWD_TINY);
  }
  pl.smem = std::max(kPersistTinyWarps * 32, mmax + 2 + 32 * 33) * 8;
  if (pl.tiny.empty()) pl.tiny.push_back(0);
}

// As check_persist_plan, for the solve queue: forward tasks after their children's forward
// tasks, backward tasks after their parent's backward task (roots: after their own forward).
std::string check_solve_plan(const Symbolic& S, const PersistPlan& pl) {
  const int ns = (int)S.nsuper;
  const int ntask = (int)(pl.task.size() / 6);
  if (pl.gstart.back() != ntask) return "group table does not cover the tasks";
  std::vector<int> pf(ns, 0), pb(ns, 0);
  auto ready = [&](int type, int sn) {
    if (type == ST_FWD_TINY || type == ST_FWD) {
      for (int64_t q = S.child_ptr[sn]; q < S.child_ptr[sn + 1]; ++q)
        if (pf[S.child_list[q]] != 1) return false;
      return pf[sn] == 0;
    }
    const int64_t p = S.sn_parent[sn];
    return pb[sn] == 0 && (p < 0 ? pf[sn] == 1 : pb[p] == 1);
  };
  for (int t = 0; t < ntask; ++t) {
    const int* T = pl.task.data() + 6 * t;
    const bool tiny = T[0] == ST_FWD_TINY || T[0] == ST_BWD_TINY;
    const bool fwd = T[0] == ST_FWD_TINY || T[0] == ST_FWD;
    const int cnt = tiny ? T[2] : 1;
    for (int u = 0; u < cnt; ++u) {
      const int sn = tiny ? pl.tiny[T[1] + u] : T[1];
      if (sn < 0 || sn >= ns || !ready(T[0], sn)) return "task " + std::to_string(t) + " before its dependencies";
      if (tiny && S.sn_rowptr[sn + 1] - S.sn_rowptr[sn] > kTinyM) return "tiny task with a wide front";
      (fwd ? pf : pb)[sn] = 1;
    }
  }
  for (int sn = 0; sn < ns; ++sn)
    if (pf[sn] != 1 || pb[sn] != 1) return "front " + std::to_string(sn) + " not swept";
  return std::string();
}

void GpuFactor::plan_solve_persist() {
  PersistPlan pl;
  make_solve_plan(sym_, levels_, pl);
  if (pl.smem > 227 * 1024 || pl.gstart.size() < 2) return;
  const int ns = (int)sym_.nsuper;
  solve_groups_ = (int)pl.gstart.size() - 1;
  d_sgstart_.upload(pl.gstart, stream_);
  d_stask_.upload(pl.task, stream_);
  d_stiny_.upload(pl.tiny, stream_);
  d_sstate_.alloc(2 + 2 * (size_t)max_batch_ * ns);
  INLA_CUDA(cudaMemsetAsync(d_sstate_.p, 0, sizeof(int) * (2 + 2 * (size_t)max_batch_ * ns), stream_));
  solve_smem_ = pl.smem;
  solve_persist_ = true;
}

void GpuFactor::plan_persist() {
  int def = g_persist_default.load();
  if (def < 0) {
    def = std::getenv("INLA_NO_PERSIST") ? 0 : 1;
    int expect = -1;
    g_persist_default.compare_exchange_strong(expect, def);
    def = g_persist_default.load();
  }
  if (def == 0) return;
  persist_mode_ = def;
  if (const char* w = std::getenv("INLA_PERSIST_WAIT_MS")) persist_limit_ns_ = (long long)(std::atof(w) * 1e6);
  PersistPlan pl;
  if (!make_persist_plan(sym_, levels_, pl)) return;  // a front too wide for the schedule's shared memory
  const int ns = (int)sym_.nsuper;
  const size_t dc_doubles = (size_t)std::max(pl.nlarge, 1) * max_batch_ * kB64 * kB64;
  if (dc_doubles * 8 > ((size_t)4 << 30)) return;
  persist_groups_ = (int)pl.gstart.size() - 1;
  d_pgstart_.upload(pl.gstart, stream_);
  d_ptask_.upload(pl.task, stream_);
  d_ptiny_.upload(pl.tiny, stream_);
  d_ptotal_.upload(pl.total, stream_);
  d_plid_.upload(pl.lid, stream_);
  d_pgptr_.upload(pl.gptr, stream_);
  d_pgrng_.upload(pl.grng, stream_);
  d_pstate_.alloc(2 + (size_t)max_batch_ * ns);
  INLA_CUDA(cudaMemsetAsync(d_pstate_.p, 0, sizeof(int) * (2 + (size_t)max_batch_ * ns), stream_));
  dcache_p_.alloc(dc_doubles);
  persist_smem_ = pl.smem;
  persist_ = true;
  plan_solve_persist();
}

void GpuFactor::set_front_groups(const std::vector<int>& fseg) {
  if ((int64_t)fseg.size() != sym_.nsuper) throw std::runtime_error("one group per front expected");
  d_fseg_.upload(fseg, stream_);
}

void GpuFactor::run_factor_persist(int B, const int* total_override, long long limit_ns,
                                   const unsigned char* active, int nseg) {
  const int ns = (int)sym_.nsuper;
  // head and the completion counts start at zero; the error record (word 0) stays until read
  INLA_CUDA(cudaMemsetAsync(d_pstate_.p + 1, 0, sizeof(int) * (1 + (size_t)B * ns), stream_));
  PersistArgs a;
  a.S = ds_;
  a.F = F_.p;
  a.fstride = ftotal_;
  a.B = B;
  a.ngroups = persist_groups_;
  a.gstart = d_pgstart_.p;
  a.task = reinterpret_cast<const PersistTask*>(d_ptask_.p);
  a.tiny_list = d_ptiny_.p;
  a.total = total_override ? total_override : d_ptotal_.p;
  a.prog = d_pstate_.p + 2;
  a.head = reinterpret_cast<unsigned*>(d_pstate_.p + 1);
  a.err = d_pstate_.p;
  a.dcache = dcache_p_.p;
  a.lid = d_plid_.p;
  a.linv = linv_.p;
  a.gptr = d_pgptr_.p;
  a.grng = d_pgrng_.p;
  a.limit_ns = limit_ns > 0 ? limit_ns : persist_limit_ns_;
  if (active) {
    a.S.active = active;
    a.S.fseg = d_fseg_.p;
    a.S.nseg = nseg;
  }
  k_factor_persist<<<persist_grid_, kPersistThreads, persist_smem_, stream_>>>(a);
  k_logdet_chunks<<<dim3(nldchunk_, B), 256, 0, stream_>>>(ds_, F_.p, ftotal_, ldpart_.p, ldflag_.p, ldticket_.p,
                                                           logdet_.p, status_.p, d_pstate_.p);
  launches_ += 2;
}

// Persistent or level launches for batch size B: fixed by the mode, or measured on the
// first factorization at B (the level sequence in its tuned form and the persistent launch,
// each after a warm-up, with CUDA events on the engine's stream) and kept for the structure
// and B. The triangular solve follows the same choice.
bool GpuFactor::use_persist(int B, const std::function<void()>& fill) {
  if (!persist_) return false;
  if (persist_mode_ == 2) return true;
  auto it = persist_at_.find(B);
  if (it != persist_at_.end()) return it->second;
  {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    auto g = g_sched.find({struct_hash_, B});
    if (g != g_sched.end()) return persist_at_[B] = g->second;
  }
  const std::vector<char>* pol = schedule(B, fill);
  cudaEvent_t e[4];
  for (auto& x : e) INLA_CUDA(cudaEventCreate(&x));
  fill();
  run_factor_levels(B, pol);  // warm-up
  fill();
  INLA_CUDA(cudaEventRecord(e[0], stream_));
  run_factor_levels(B, pol);
  INLA_CUDA(cudaEventRecord(e[1], stream_));
  fill();
  run_factor_persist(B);  // warm-up
  fill();
  INLA_CUDA(cudaEventRecord(e[2], stream_));
  run_factor_persist(B);
  INLA_CUDA(cudaEventRecord(e[3], stream_));
  INLA_CUDA(cudaStreamSynchronize(stream_));
  float tl = 0.f, tp = 0.f;
  INLA_CUDA(cudaEventElapsedTime(&tl, e[0], e[1]));
  INLA_CUDA(cudaEventElapsedTime(&tp, e[2], e[3]));
  for (auto& x : e) cudaEventDestroy(x);
  check_schedule();
  const bool pick = tp < tl;
  if (std::getenv("INLA_DEBUG"))
    std::fprintf(stderr, "schedule B=%d: level launches %.3f ms, persistent %.3f ms -> %s\n", B, tl, tp,
                 pick ? "persistent" : "levels");
  {
    std::lock_guard<std::mutex> lk(g_sched_mu);
    g_sched[{struct_hash_, B}] = pick;
  }
  return persist_at_[B] = pick;
}

void GpuFactor::check_schedule() {
  if (!persist_) return;
  int err = 0, serr = 0;
  INLA_CUDA(cudaMemcpyAsync(&err, d_pstate_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  if (solve_persist_) INLA_CUDA(cudaMemcpyAsync(&serr, d_sstate_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaStreamSynchronize(stream_));
  if (err == 0 && serr == 0) return;
  INLA_CUDA(cudaMemsetAsync(d_pstate_.p, 0, sizeof(int), stream_));
  if (solve_persist_) INLA_CUDA(cudaMemsetAsync(d_sstate_.p, 0, sizeof(int), stream_));
  INLA_CUDA(cudaStreamSynchronize(stream_));
  if (err == 0) err = serr;
  throw CudaError("persistent factorization stopped: a dependency wait ran out (code " + std::to_string(err) + ")",
                  (int)cudaErrorLaunchTimeout);
}

int GpuFactor::persist_wait_limit_selftest(double limit_ms) {
  if (!persist_) return -1;
  const int ns = (int)sym_.nsuper;
  // completion counts no front can reach: every front with children waits until the limit
  std::vector<int> never(ns, 1 << 30);
  DBuf<int> d_never;
  d_never.upload(never, stream_);
  INLA_CUDA(cudaMemsetAsync(F_.p, 0, sizeof(double) * ftotal_, stream_));  // a defined input for the fronts that run
  run_factor_persist(1, d_never.p, (long long)(limit_ms * 1e6));
  INLA_CUDA(cudaGetLastError());
  int err = 0;
  INLA_CUDA(cudaMemcpyAsync(&err, d_pstate_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
  INLA_CUDA(cudaStreamSynchronize(stream_));
  INLA_CUDA(cudaMemsetAsync(d_pstate_.p, 0, sizeof(int), stream_));
  INLA_CUDA(cudaStreamSynchronize(stream_));
  return err;
}

void GpuFactor::run_factor_levels(int B, const std::vector<char>* fuse, cudaEvent_t* ev) {
  const int64_t fs = ftotal_;
  for (size_t li = 0; li < levels_.size(); ++li) {
    const LevelPlan& P = levels_[li];
    if (!P.tiny.empty()) {
      const int nt = (int)P.tiny.size();
      k_factor_tiny<<<dim3(cdiv(nt, kTinyWarps), B), 32 * kTinyWarps, 0, stream_>>>(ds_, d_lists_.p + P.off_tiny, nt,
                                                                                 F_.p, fs);
      ++launches_;
    }
    if (!P.small_a.empty()) {
      dim3 g((unsigned)P.small_a.size(), B);
      k_factor_small<128><<<g, 128, small_factor_smem(P.mmax_a), stream_>>>(ds_, d_lists_.p + P.off_small_a, F_.p,
                                                                             fs);
      ++launches_;
    }
    if (!P.small_b.empty()) {
      dim3 g((unsigned)P.small_b.size(), B);
      k_factor_small<256><<<g, 256, small_factor_smem(P.mmax_b), stream_>>>(ds_, d_lists_.p + P.off_small_b, F_.p,
                                                                             fs);
      ++launches_;
    }
    if (ev) INLA_CUDA(cudaEventRecord(ev[2 * li], stream_));
    if (!P.large.empty()) {
      const int nl = (int)P.large.size();
      const int* lst = d_lists_.p + P.off_large;
      const int gcols = gather_cols(P.mmax_large);
      k_gather8<<<dim3(nl, B, cdiv(P.mmax_large, gcols)), 256, gcols * P.mmax_large * 8, stream_>>>(
          ds_, lst, F_.p, fs, gcols, d_gptr_.p, d_grng_.p);
      ++launches_;
      const int form = fuse ? (*fuse)[li] : -1;
      for (int j0 = 0; j0 < P.kmax_large; j0 += kB64) {
        int rows = P.mmax_large - j0;
        const int nrb = std::max(1, cdiv(rows, kPanelRows));
        int nt = cdiv(rows, kUT64);
        const dim3 ug(nl, B, std::max(1, nt * (nt + 1) / 2));
        if (form == kFormLookahead) {
          // block 0 by one CTA per (front, problem); every later diagonal block by tile 0 of
          // the previous step's update
          double* cur = dcache_.p + ((j0 / kB64) & 1) * dslot_;
          double* nxt = dcache_.p + (((j0 / kB64) + 1) & 1) * dslot_;
          if (j0 == 0) {
            k_panel64<<<dim3(nl, B, 1), 256, kPanelSmem, stream_>>>(ds_, lst, j0, 0, F_.p, fs, cur, linv_.p);
            ++launches_;
          }
          k_rows64<<<dim3(nl, B, nrb), 256, kRowsSmem, stream_>>>(ds_, lst, j0, F_.p, fs, cur, linv_.p);
          k_update64la<<<ug, 256, kPanelSmem, stream_>>>(ds_, lst, j0, F_.p, fs, cur, nxt, linv_.p);
          launches_ += 2;
          continue;
        }
        // While every (front, problem, 64-row block) gets its own CTA within about
        // one wave (two CTAs per SM), each row CTA factors the diagonal block
        // itself (one launch). Beyond that, one CTA per (front, problem) factors
        // it and k_rows64 forms the rows from the cached factor (no redundant
        // factorizations).
        const int per = std::max(1, (2 * num_sms_) / std::max(1, nl * B));
        const bool fused = form >= 0 ? form == kFormFused : per >= nrb;
        if (fused) {
          k_panel64<<<dim3(nl, B, nrb), 256, kPanelSmem, stream_>>>(ds_, lst, j0, kPanelRows, F_.p, fs, dcache_.p,
                                                                     linv_.p);
        } else {
          k_panel64<<<dim3(nl, B, 1), 256, kPanelSmem, stream_>>>(ds_, lst, j0, 0, F_.p, fs, dcache_.p, linv_.p);
          k_rows64<<<dim3(nl, B, nrb), 256, kRowsSmem, stream_>>>(ds_, lst, j0, F_.p, fs, dcache_.p, linv_.p);
          ++launches_;
        }
        k_update64w8<<<ug, 256, kPersistUpdSmem, stream_>>>(ds_, lst, j0, F_.p, fs, dcache_.p);
        launches_ += 2;
      }
    }
    if (ev) INLA_CUDA(cudaEventRecord(ev[2 * li + 1], stream_));
  }
  k_logdet_chunks<<<dim3(nldchunk_, B), 256, 0, stream_>>>(ds_, F_.p, fs, ldpart_.p, ldflag_.p, ldticket_.p,
                                                           logdet_.p, status_.p);
  ++launches_;
}

// ---------------------------------------------------------------------------
// Panel-schedule autotuner. For every level with large fronts the panel step has
// three forms with bit-identical results: "split" (one CTA per front factors the
// 64 x 64 diagonal block, k_rows64 forms the rows from the cached factor, then the
// trailing update: three launches per step), "fused" (each of the nrb row CTAs
// factors the diagonal block itself, then the update: two launches) and
// "look-ahead" (rows, then the update whose tile-0 CTAs factor the next diagonal
// block: two launches per step plus one for the first block). Which is faster
// depends on the level's fronts, the batch size and the GPU, so on the first
// factorization at a batch size B the level sequence runs once in each form
// (after a fill, untimed warm-up first) with CUDA events around every level's
// large-front work, and each level keeps the fastest form. Decisions are kept in a
// process-wide table keyed by the supernodal structure and B, so later handles on
// the same pattern reuse them. INLA_NO_AUTOTUNE in the environment keeps the
// occupancy rule (fused while every row CTA fits in about one wave, else split).
// ---------------------------------------------------------------------------
namespace {
std::mutex g_tune_mu;
std::map<std::pair<uint64_t, int>, std::vector<char>> g_tune;  // (structure hash, B) -> schedule
}  // namespace

const std::vector<char>* GpuFactor::schedule(int B, const std::function<void()>& fill) {
  static const bool off = std::getenv("INLA_NO_AUTOTUNE") != nullptr;
  if (off) return nullptr;
  bool any_large = false;
  for (const LevelPlan& P : levels_) any_large = any_large || !P.large.empty();
  if (!any_large) return nullptr;
  auto it = fuse_.find(B);
  if (it != fuse_.end()) return &it->second;
  if (panel_form_ >= 0) return &(fuse_[B] = std::vector<char>(levels_.size(), (char)panel_form_));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto g = g_tune.find({struct_hash_, B});
    if (g != g_tune.end()) return &(fuse_[B] = g->second);
  }
  const size_t L = levels_.size();
  std::vector<cudaEvent_t> ev(2 * L);
  for (auto& e : ev) INLA_CUDA(cudaEventCreate(&e));
  std::vector<double> t[kNumForms];
  for (int form = 0; form < kNumForms; ++form) {
    const std::vector<char> pol(L, (char)form);
    fill();
    run_factor_levels(B, &pol, nullptr);  // warm-up (module load, caches)
    fill();
    run_factor_levels(B, &pol, ev.data());
    INLA_CUDA(cudaStreamSynchronize(stream_));
    t[form].assign(L, 0.0);
    for (size_t l = 0; l < L; ++l) {
      float ms = 0.f;
      INLA_CUDA(cudaEventElapsedTime(&ms, ev[2 * l], ev[2 * l + 1]));
      t[form][l] = ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  std::vector<char> best(L, kFormSplit);
  double tot[kNumForms] = {0.0, 0.0, 0.0}, tbest = 0.0;
  for (size_t l = 0; l < L; ++l) {
    for (int f = 0; f < kNumForms; ++f) {
      tot[f] += t[f][l];
      if (t[f][l] < t[(int)best[l]][l]) best[l] = (char)f;
    }
    tbest += t[(int)best[l]][l];
  }
  if (std::getenv("INLA_DEBUG"))
    std::fprintf(stderr, "autotune B=%d: split %.3f ms, fused %.3f ms, look-ahead %.3f ms, per-level best %.3f ms\n",
                 B, tot[kFormSplit], tot[kFormFused], tot[kFormLookahead], tbest);
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[{struct_hash_, B}] = best;
  }
  return &(fuse_[B] = best);
}

template <class Body>
void GpuFactor::launch_cached(const std::vector<int64_t>& key, Body&& body) {
  if (!use_graphs_ || uncaptured_.count(key)) {
    body();
    INLA_CUDA(cudaGetLastError());
    return;
  }
  auto it = graphs_.find(key);
  if (it == graphs_.end()) {
    const int64_t before = launches_;
    INLA_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    bool host_error = false;
    try {
      body();
    } catch (...) {
      host_error = true;
    }
    // A launch rejected during capture (configuration, resources, a call that
    // capture does not allow) returns its error here and invalidates the capture.
    const cudaError_t launch_err = cudaGetLastError();
    cudaGraph_t g = nullptr;
    const cudaError_t end_err = cudaStreamEndCapture(stream_, &g);
    const int64_t captured = launches_ - before;
    launches_ = before;
    if (host_error || launch_err != cudaSuccess || end_err != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();  // the capture's errors are not sticky: clear them
      // Keep the handle usable: this key runs without a graph from now on. A
      // host-side exception of the body surfaces again, with its message, from
      // the direct run.
      const cudaError_t why = launch_err != cudaSuccess ? launch_err : end_err;
      std::fprintf(stderr, "inla_b200: CUDA graph capture of launch sequence %lld failed (%s); running it uncaptured\n",
                   (long long)key[0], host_error ? "host exception" : cudaGetErrorString(why));
      uncaptured_.insert(key);
      ++capture_failures_;
      body();
      const cudaError_t run_err = cudaGetLastError();
      if (run_err != cudaSuccess)
        throw CudaError(std::string("launch sequence failed (capture: ") + cudaGetErrorString(why) +
                            "; direct run: " + cudaGetErrorString(run_err) + ")",
                        (int)run_err);
      return;
    }
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) throw CudaError(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e), (int)e);
    it = graphs_.emplace(key, GraphEntry{ex, captured}).first;
  }
  INLA_CUDA(cudaGraphLaunch(it->second.exec, stream_));
  launches_ += it->second.nkernels;
}

void GpuFactor::factor_values(const double* d_vals, int B) {
  if (B < 1 || B > max_batch_) throw std::runtime_error("batch size out of range");
  auto fill = [&] {
    k_fill_panels<<<dim3(nfill_, B), 256, 0, stream_>>>(ds_, d_csn_.p, ntot_, d_pmap_.p, d_vals, nnz_, F_.p,
                                                        ftotal_);
    ++launches_;
  };
  const bool per = use_persist(B, fill);  // settled before any capture
  const std::vector<char>* pol = per ? nullptr : schedule(B, fill);
  launch_cached({1, B, (int64_t)(uintptr_t)d_vals, per}, [&] {
    fill();
    if (per) run_factor_persist(B);
    else run_factor_levels(B, pol);
  });
}

void GpuFactor::factor_model(int ncomp, const double* d_comp, const double* d_coef, double diag_add,
                             const unsigned char* d_pdiag, const int* d_cptr, const int* d_cobs,
                             const double* d_cprod, const double* d_w, int64_t wstride, int B, int nprior,
                             double diag_add_post, const int* d_pseg, int nseg, const unsigned char* d_active) {
  if (B < 1 || B > max_batch_) throw std::runtime_error("batch size out of range");
  if (nprior < 0 || nprior > B) throw std::runtime_error("prior count out of range");
  if (ncomp < 1 || ncomp > 8) throw std::runtime_error("1..8 precision components supported");
  int64_t dbits, dpbits;
  std::memcpy(&dbits, &diag_add, sizeof(dbits));
  std::memcpy(&dpbits, &diag_add_post, sizeof(dpbits));

  const unsigned char* fill_mask = nullptr;  // the measurements below fill and factorize every pair
  auto fill = [&] {
    k_fill_panels_model<<<dim3(nfillm_), 256, 0, stream_>>>(ds_, d_csnm_.p, ntot_, d_pmap_.p, ncomp, d_comp, nnz_,
                                                            d_coef, diag_add, d_pdiag, d_cptr, d_cobs, d_cprod, d_w,
                                                            wstride, B, nprior, diag_add_post, d_pseg, nseg, F_.p,
                                                            ftotal_, d_fseg_.p, fill_mask);
    ++launches_;
  };
  const bool per = use_persist(B, fill);  // settled before any capture
  if (!d_fseg_.p) d_active = nullptr;
  fill_mask = d_active;
  const std::vector<char>* pol = per ? nullptr : schedule(B, fill);
  launch_cached({2, B, ncomp, (int64_t)(uintptr_t)d_comp, (int64_t)(uintptr_t)d_coef, dbits,
                 (int64_t)(uintptr_t)d_pdiag, (int64_t)(uintptr_t)d_cptr, (int64_t)(uintptr_t)d_cobs,
                 (int64_t)(uintptr_t)d_cprod, (int64_t)(uintptr_t)d_w, wstride, nprior, dpbits,
                 (int64_t)(uintptr_t)d_pseg, nseg, (int64_t)(uintptr_t)d_active, per},
                [&] {
                  fill();
                  if (per) {
                    run_factor_persist(B, nullptr, 0, d_active, nseg);
                  } else {
                    const DevSym plain = ds_;
                    if (d_active) {  // the level kernels read the mask through the device view
                      ds_.active = d_active;
                      ds_.fseg = d_fseg_.p;
                      ds_.nseg = nseg;
                    }
                    run_factor_levels(B, pol);
                    ds_ = plain;
                  }
                });
}

void GpuFactor::solve(double* d_x, int64_t xstride, int B, int slot0) {
  if (B < 1 || slot0 < 0 || slot0 + B > max_batch_) throw std::runtime_error("batch size out of range");
  const int n = (int)sym_.n;
  const int64_t fs = ftotal_;
  const double* Fp = F_.p + (int64_t)slot0 * fs;
  dim3 gp(cdiv(n, 256) > 1024 ? 1024 : cdiv(n, 256), B);
  auto pa = persist_at_.find(B);
  const bool per = solve_persist_ && (persist_mode_ == 2 || (pa != persist_at_.end() && pa->second));
  if (per) {
    launch_cached({3, B, (int64_t)(uintptr_t)d_x, xstride, slot0, 1}, [&] {
      const int ns = (int)sym_.nsuper;
      k_permute_in<<<gp, 256, 0, stream_>>>(n, d_perm_.p, d_x, xstride, xp_.p);
      INLA_CUDA(cudaMemsetAsync(d_sstate_.p + 1, 0, sizeof(int) * (1 + 2 * (size_t)B * ns), stream_));
      SolveArgs a;
      a.S = ds_;
      a.F = Fp;
      a.fstride = fs;
      a.B = B;
      a.ngroups = solve_groups_;
      a.gstart = d_sgstart_.p;
      a.task = reinterpret_cast<const PersistTask*>(d_stask_.p);
      a.tiny_list = d_stiny_.p;
      a.linv = linv_.p + (int64_t)slot0 * ds_.lstride;
      a.xp = xp_.p;
      a.ub = ub_.p;
      a.ustride = std::max<int64_t>(usum_, 1);
      a.progf = d_sstate_.p + 2;
      a.progb = d_sstate_.p + 2 + (size_t)B * ns;
      a.head = reinterpret_cast<unsigned*>(d_sstate_.p + 1);
      a.err = d_sstate_.p;
      a.limit_ns = persist_limit_ns_;
      k_solve_persist<<<solve_grid_, kPersistThreads, solve_smem_, stream_>>>(a);
      k_permute_out<<<gp, 256, 0, stream_>>>(n, d_perm_.p, xp_.p, d_x, xstride);
      launches_ += 3;
    });
    return;
  }
  launch_cached({3, B, (int64_t)(uintptr_t)d_x, xstride, slot0}, [&] {
    k_permute_in<<<gp, 256, 0, stream_>>>(n, d_perm_.p, d_x, xstride, xp_.p);
    ++launches_;
    const int64_t us = std::max<int64_t>(usum_, 1);
    const double* Lp = linv_.p + (int64_t)slot0 * ds_.lstride;
    // fronts of up to kSmallB rows (contiguous lists small_a, small_b) in 32-column blocks by one
    // CTA each; larger fronts in 64-column blocks with their cached inverse blocks
    for (const LevelPlan& P : levels_) {
      if (!P.tiny.empty()) {
        const int nt = (int)P.tiny.size();
        k_fwd_tiny<<<dim3(cdiv(nt, kTinySweepWarps), B), 32 * kTinySweepWarps, 0, stream_>>>(
            ds_, d_lists_.p + P.off_tiny, nt, Fp, fs, xp_.p, ub_.p, us);
        ++launches_;
      }
      const int nsm = (int)(P.small_a.size() + P.small_b.size());
      if (nsm > 0) {
        k_fwd32<128><<<dim3((unsigned)nsm, B), 128, (std::max(P.mmax_a, P.mmax_b) + 2 + 32 * 33) * 8, stream_>>>(
            ds_, d_lists_.p + P.off_small_a, Fp, fs, xp_.p, ub_.p, us);
        ++launches_;
      }
      if (!P.large.empty()) {
        const dim3 g((unsigned)P.large.size(), B);
        const int sm = (P.mmax_large + 2) * 8;
        if ((int64_t)P.large.size() * B <= num_sms_)
          k_fwd64<256, true><<<g, 256, sm, stream_>>>(ds_, d_lists_.p + P.off_large, Fp, fs, Lp, xp_.p, ub_.p, us);
        else
          k_fwd64<256, false><<<g, 256, sm, stream_>>>(ds_, d_lists_.p + P.off_large, Fp, fs, Lp, xp_.p, ub_.p, us);
        ++launches_;
      }
    }
    for (int l = (int)levels_.size() - 1; l >= 0; --l) {
      const LevelPlan& P = levels_[l];
      if (!P.tiny.empty()) {
        const int nt = (int)P.tiny.size();
        k_bwd_tiny<<<dim3(cdiv(nt, kTinySweepWarps), B), 32 * kTinySweepWarps, 0, stream_>>>(
            ds_, d_lists_.p + P.off_tiny, nt, Fp, fs, xp_.p);
        ++launches_;
      }
      const int nsm = (int)(P.small_a.size() + P.small_b.size());
      if (nsm > 0) {
        k_bwd32<128><<<dim3((unsigned)nsm, B), 128, (std::max(P.mmax_a, P.mmax_b) + 2 + 32 * 33) * 8, stream_>>>(
            ds_, d_lists_.p + P.off_small_a, Fp, fs, xp_.p);
        ++launches_;
      }
      if (!P.large.empty()) {
        const dim3 g((unsigned)P.large.size(), B);
        const int sm = (P.mmax_large + 2) * 8;
        if ((int64_t)P.large.size() * B <= num_sms_)
          k_bwd64<256, true><<<g, 256, sm, stream_>>>(ds_, d_lists_.p + P.off_large, Fp, fs, Lp, xp_.p);
        else
          k_bwd64<256, false><<<g, 256, sm, stream_>>>(ds_, d_lists_.p + P.off_large, Fp, fs, Lp, xp_.p);
        ++launches_;
      }
    }
    k_permute_out<<<gp, 256, 0, stream_>>>(n, d_perm_.p, xp_.p, d_x, xstride);
    ++launches_;
  });
}

void GpuFactor::selinv(int B, int slot0) {
  if (B < 1 || slot0 < 0 || slot0 + B > max_batch_) throw std::runtime_error("batch size out of range");
  Sg_.alloc((size_t)max_batch_ * ftotal_);  // outside any capture
  launch_cached({4, B, slot0}, [&] { selinv_levels(B, slot0); });
}

void GpuFactor::selinv_levels(int B, int slot0) {
  const int64_t fs = ftotal_;
  const double* Fp = F_.p + (int64_t)slot0 * fs;
  double* Sp = Sg_.p + (int64_t)slot0 * fs;
  const double* Lp = linv_.p + (int64_t)slot0 * ds_.lstride;
  for (int l = (int)levels_.size() - 1; l >= 0; --l) {
    const LevelPlan& P = levels_[l];
    if (!P.si_tiny.empty()) {
      const int nt = (int)P.si_tiny.size();
      k_selinv_tiny<<<dim3(cdiv(nt, kTinySiWarps), B), 32 * kTinySiWarps, 0, stream_>>>(
          ds_, d_lists_.p + P.off_si_tiny, nt, Fp, Sp, fs);
      ++launches_;
    }
    if (!P.si_small.empty()) {
      int mm = P.mmax_si_small;
      k_selinv_small<256><<<dim3((unsigned)P.si_small.size(), B), 256, small_selinv_smem(mm, P.kmax_si_small),
                            stream_>>>(
          ds_, d_lists_.p + P.off_si_small, Fp, Sp, fs);
      ++launches_;
    }
    if (!P.si_large.empty()) {
      const int nl = (int)P.si_large.size();
      const int* lst = d_lists_.p + P.off_si_large;
      if (P.rmax_si_large > 0) {
        k_si_gather8<<<dim3(nl, B, cdiv(P.rmax_si_large, kGatherCols)), 256, 0, stream_>>>(ds_, lst, Sp, fs);
        ++launches_;
      }
      const int nblk = cdiv(P.kmax_si_large, kB64);
      const int ptiles = cdiv(P.mmax_si_large, kSiT);
      // the K range of G is split over several CTAs only where one CTA per (front, problem,
      // row tile) would not give every SM one (the top of the tree at small batch sizes)
      const bool split = (int64_t)nl * B * ptiles <= num_sms_;
      const int smax = si_nsplit(cdiv(P.mmax_si_large, 32), split);
      for (int jb = 0; jb < nblk; ++jb) {
        k_si_step64<<<dim3(nl, B, ptiles * smax), 256, kSiGemmSmem, stream_>>>(
            ds_, lst, jb, Fp, Sp, fs, ppart_.p, ptiles, Lp, gpart_.p, sicnt_.p, smax, split ? 1 : 0);
        k_si_diag64<<<dim3(nl, B), 256, kSiDiagSmem, stream_>>>(ds_, lst, jb, Fp, Sp, fs, ppart_.p, ptiles,
                                                                Lp);
        launches_ += 2;
      }
    }
  }
}

void GpuFactor::extract_diag(double* d_out, int64_t ostride, int B, int slot0) {
  const int n = (int)sym_.n;
  k_extract_diag<<<dim3(std::min(cdiv(n, 256), 1024), B), 256, 0, stream_>>>(ds_, Sg_.p + (int64_t)slot0 * ftotal_,
                                                                              ftotal_, d_out, ostride);
  ++launches_;
  INLA_CUDA(cudaGetLastError());
}

void GpuFactor::sigma_on_pattern(double* d_out, int B, int slot0) {
  k_pattern_values<<<dim3(std::min(cdiv(nnz_, 256), 2048), B), 256, 0, stream_>>>(
      nnz_, spos_.p, Sg_.p + (int64_t)slot0 * ftotal_, ftotal_, d_out);
  ++launches_;
  INLA_CUDA(cudaGetLastError());
}

}  // namespace inla
