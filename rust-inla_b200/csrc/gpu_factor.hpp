// Device-resident numeric engine for one symbolic analysis: batched
// multifrontal LDL^T, log-determinants, solves and selected inversion.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "devsym.hpp"
#include "symbolic.hpp"

namespace inla {

struct CudaError : std::runtime_error {
  int code;
  CudaError(const std::string& s, int c) : std::runtime_error(s), code(c) {}
};

#define INLA_CUDA(call)                                                                    \
  do {                                                                                     \
    cudaError_t _e = (call);                                                               \
    if (_e != cudaSuccess)                                                                 \
      throw ::inla::CudaError(std::string(#call) + ": " + cudaGetErrorString(_e), (int)_e); \
  } while (0)

// Device allocation through the library's cache of released blocks (devmem.cu).
void* device_alloc(size_t bytes);
void device_free(void* p);
void device_release_cached();

// Schedule of the engines built from now on: 0 level launches, 1 measured per batch size, 2
// persistent wherever it fits.
void set_persistent_default(int mode);
// Panel form of the level launches for engines built from now on: -1 autotuned per level
// (default), 0 split, 1 fused, 2 look-ahead (bit-identical results).
void set_panel_form(int form);

// Small RAII device buffer.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) device_free(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count <= n && p) return;
    release();
    if (count == 0) count = 1;
    p = static_cast<T*>(device_alloc(count * sizeof(T)));
    n = count;
  }
  void upload(const T* h, size_t count, cudaStream_t st = 0) {
    alloc(count);
    if (count) INLA_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  void upload(const std::vector<T>& v, cudaStream_t st = 0) { upload(v.data(), v.size(), st); }
};

struct LevelPlan {
  std::vector<int> tiny, small_a, small_b, large, all, nontiny;  // host copies (supernode ids)
  int off_tiny = 0, off_small_a = 0, off_small_b = 0, off_large = 0, off_all = 0, off_nontiny = 0;  // offsets into one device list
  int mmax_nontiny = 0;
  int mmax_a = 0, mmax_b = 0, mmax_all = 0, kmax_large = 0, mmax_large = 0;
  // selected inversion grouping
  std::vector<int> si_tiny, si_small, si_large;
  int off_si_tiny = 0, off_si_small = 0, off_si_large = 0, mmax_si_small = 0, kmax_si_small = 0, kmax_si_large = 0, mmax_si_large = 0, rmax_si_large = 0;
};

// Task queue of the persistent schedule for one problem (snode_persist.cuh): 6 ints per task
// {type, front, sub, need, j0, gcols}, group starts, tiny-front list, completion counts per
// front, large-front index, extend-add chunk table, shared memory in bytes.
struct PersistPlan {
  std::vector<int> gstart, task, tiny, total, lid;
  std::vector<int64_t> gptr;
  std::vector<int2> grng;
  int nlarge = 0, smem = 0;
};
// Host tables of an analysis that an engine uploads: 32-bit copies of the supernode arrays,
// front offsets fptr (sum m^2) and panel offsets lptr, D positions dpos, the panel map pmap
// (compact panel index -> input entry) and the front positions of the input entries (spos:
// entries stored in a panel; spos_full: every entry). Shared by the engines built on one
// analysis (cached by Symbolic::id).
struct HostMaps {
  std::vector<int> first, rowptr, rows, relx, child_ptr, child_list, parent, uoff, perm, pmap;
  std::vector<int64_t> fptr, lptr, dpos, spos, spos_full;
};
std::shared_ptr<const HostMaps> host_maps(const Symbolic& S);
void release_host_maps();
std::vector<LevelPlan> make_level_plans(const Symbolic& S, std::vector<int>& flat);
bool make_persist_plan(const Symbolic& S, const std::vector<LevelPlan>& levels, PersistPlan& out);
std::string check_persist_plan(const Symbolic& S, const PersistPlan& pl);
// Task queue of the persistent triangular solve (forward sweep bottom-up, then backward).
void make_solve_plan(const Symbolic& S, const std::vector<LevelPlan>& levels, PersistPlan& out);
std::string check_solve_plan(const Symbolic& S, const PersistPlan& pl);

class GpuFactor {
 public:
  // Size classes (rows of the front): <= kSmallA uses 128 threads, <= kSmallB 256
  // threads (one CTA per front), larger fronts use the blocked multi-CTA
  // kernels in both the factorization and the selected inverse.
  static constexpr int kSmallA = 64;
  static constexpr int kSmallB = 96;
  static constexpr int kSiSmall = kSmallB;

  GpuFactor(const Symbolic& sym, int max_batch, cudaStream_t stream);
  ~GpuFactor();

  const Symbolic& sym() const { return sym_; }
  int max_batch() const { return max_batch_; }
  cudaStream_t stream() const { return stream_; }
  int64_t front_total() const { return ftotal_; }
  int64_t nnz() const { return nnz_; }

  // Factorize B problems whose full-CSC values (input pattern order) are at
  // d_vals [B][nnz] on the device. Results stay resident.
  void factor_values(const double* d_vals, int B);
  // Factorize from the component model (see k_fill_panels_model): problems
  // [0, nprior) get diag_add and no observation term, problems [nprior, B)
  // diag_add_post and the weights w + (b - nprior) * wstride (if d_w).
  void factor_model(int ncomp, const double* d_comp, const double* d_coef, double diag_add,
                    const unsigned char* d_pdiag, const int* d_cptr, const int* d_cobs, const double* d_cprod,
                    const double* d_w, int64_t wstride, int B, int nprior = 0, double diag_add_post = 0.0,
                    const int* d_pseg = nullptr, int nseg = 1, const unsigned char* d_active = nullptr);
  // Model of every front when the pattern holds independent models block-diagonally: lets
  // factor_model skip the fronts of inactive (problem, model) pairs (d_active [B][nseg]),
  // which then keep their previous factor.
  void set_front_groups(const std::vector<int>& fseg);
  bool can_skip_groups() const { return d_fseg_.p != nullptr; }
  // Device view of the symbolic analysis (pivot offsets, permutation, ...).
  const DevSym& dev_sym() const { return ds_; }
  // Front offset of every input entry's lower twin (both triangles), for
  // reading Sigma / L on the full pattern.
  const int64_t* d_spos_full() const { return spos_full_.p; }
  // log|Q_b| and status words (after factor_*) -> device arrays of length B.
  const double* d_logdet() const { return logdet_.p; }
  const int* d_status() const { return status_.p; }
  // The operations below act on the B problems in slots [slot0, slot0 + B) of
  // the last factorization (e.g. the posterior part of a prior + posterior batch).
  // Solve Q_b x = rhs_b in place; d_x is [B][xstride] in original order.
  void solve(double* d_x, int64_t xstride, int B, int slot0 = 0);
  // Selected inverse on the filled pattern; then extract diag / pattern values.
  void selinv(int B, int slot0 = 0);
  void extract_diag(double* d_out, int64_t ostride, int B, int slot0 = 0);
  void sigma_on_pattern(double* d_out, int B, int slot0 = 0);  // [B][nnz], lower entries, upper = 0
  const int64_t* d_spos() const { return spos_.p; }
  double* d_front() { return F_.p; }
  double* d_sigma(int slot0 = 0) { return Sg_.p + (int64_t)slot0 * ftotal_; }

  // Launch counters (kernels issued by this engine since construction).
  int64_t launches() const { return launches_; }

  // Replay the fixed launch sequences (fill+factor, solve, selected inverse)
  // from CUDA graphs captured on first use (default on).
  void set_use_graphs(bool on) { use_graphs_ = on; }
  // Launch sequences whose capture failed and that now run without a graph.
  int64_t capture_failures() const { return capture_failures_; }

  // Persistent schedule (snode_persist.cuh): the whole factorization as one launch. On by
  // default when the fronts fit its shared-memory budget (INLA_NO_PERSIST=1 keeps the level
  // launches). After a synchronization point, check_schedule() throws if a dependency wait
  // of an earlier persistent launch ran out (and clears the record).
  bool persistent() const { return persist_; }
  // Whether factorizations (and solves) at batch size B use the persistent launch: the mode's
  // fixed answer, or measured once per structure and B (see gpu_factor.cu).
  bool use_persist(int B, const std::function<void()>& fill);
  void check_schedule();
  // Diagnostic: one persistent launch whose dependencies can never complete, with a wait
  // limit of limit_ms; returns the error code the launch recorded (1: a wait ran out) after
  // clearing it. The engine stays usable.
  int persist_wait_limit_selftest(double limit_ms);

 private:
  void plan_levels();
  // fuse: per level, 1 = each row CTA factors the diagonal block itself, 0 = one CTA
  // factors it and k_rows64 forms the rows; nullptr = the occupancy rule. ev: events
  // recorded before and after every level's large-front work (2 per level).
  void run_factor_levels(int B, const std::vector<char>* fuse = nullptr, cudaEvent_t* ev = nullptr);
  // Per-level panel schedule for batch size B, measured on first use (see gpu_factor.cu).
  const std::vector<char>* schedule(int B, const std::function<void()>& fill);
  void selinv_levels(int B, int slot0);
  void plan_persist();
  void run_factor_persist(int B, const int* total_override = nullptr, long long limit_ns = 0,
                          const unsigned char* active = nullptr, int nseg = 1);
  template <class Body>
  void launch_cached(const std::vector<int64_t>& key, Body&& body);

  struct GraphEntry {
    cudaGraphExec_t exec;
    int64_t nkernels;
  };
  std::map<std::vector<int64_t>, GraphEntry> graphs_;
  std::set<std::vector<int64_t>> uncaptured_;  // sequences whose capture failed: run directly
  int64_t capture_failures_ = 0;
  bool use_graphs_ = true;
  std::map<int, std::vector<char>> fuse_;  // tuned panel schedule per batch size
  uint64_t struct_hash_ = 0;               // key of the process-wide tuning cache

  Symbolic sym_;
  int max_batch_;
  cudaStream_t stream_;
  int64_t ftotal_ = 0, nnz_ = 0, usum_ = 0;
  DevSym ds_;
  std::vector<LevelPlan> levels_;
  DBuf<int> d_first_, d_rowptr_, d_rows_, d_relx_, d_child_ptr_, d_child_list_, d_parent_, d_uoff_, d_perm_;
  DBuf<int64_t> d_fptr_, d_lptr_, d_dpos_, spos_, spos_full_, d_gptr_;
  DBuf<int2> d_grng_;  // extend-add source-column ranges per (front, chunk, child)
  DBuf<int> d_pmap_, d_lists_, d_csn_, d_csnm_, d_lbo_;
  DBuf<double> F_, Sg_, xp_, ub_, logdet_, dcache_, ppart_, linv_, ldpart_;
  DBuf<int> status_, ldflag_;
  DBuf<double> gpart_;  // split-K pieces of the selected inverse's G (narrow levels)
  DBuf<int> sicnt_;     // arrival counters of the selected inverse's step kernel (kept zeroed)
  DBuf<unsigned> ldticket_;
  int nfill_ = 0, nfillm_ = 0, nldchunk_ = 0;  // fill chunks (values, model); log-det chunks per problem
  int num_sms_ = 148;
  int64_t ntot_ = 0;              // compact panel entries per problem
  int64_t launches_ = 0;
  // persistent schedule
  bool persist_ = false;
  int persist_mode_ = 1;
  std::map<int, bool> persist_at_;  // measured choice per batch size
  int persist_smem_ = 0, persist_grid_ = 0, persist_groups_ = 0;
  long long persist_limit_ns_ = 2000000000LL;
  DBuf<int> d_pgstart_, d_ptask_, d_ptiny_, d_ptotal_, d_plid_, d_pstate_;  // pstate: err, head, prog[B][ns]
  DBuf<int64_t> d_pgptr_;
  DBuf<int2> d_pgrng_;
  DBuf<double> dcache_p_;
  int64_t dslot_ = 0;  // doubles per slot of dcache_ (two slots)
  int panel_form_ = -1;  // forced panel form (set_panel_form at construction), -1 autotuned
  DBuf<int> d_fseg_;
  // persistent solve
  bool solve_persist_ = false;
  int solve_smem_ = 0, solve_grid_ = 0, solve_groups_ = 0;
  DBuf<int> d_sgstart_, d_stask_, d_stiny_, d_sstate_;  // sstate: err, head, progf[B][ns], progb[B][ns]
  void plan_solve_persist();
};

}  // namespace inla
