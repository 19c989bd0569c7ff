// extern "C" boundary: InlaSolver seam + batched engine.
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>

#include "capi_common.hpp"
#include "gpu_factor.hpp"
#include "inla_b200.h"

namespace inla {

thread_local std::string g_last_error;
std::atomic<int64_t> g_launches{0};

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int map_exception() {
  try {
    throw;
  } catch (const CudaError& e) {
    if (e.code == cudaErrorMemoryAllocation) return fail(INLA_ERR_OOM, e.what());
    return fail(INLA_ERR_CUDA, e.what());
  } catch (const std::bad_alloc& e) {
    return fail(INLA_ERR_OOM, "host allocation failed");
  } catch (const InlaError& e) {
    return fail(e.code, e.what());
  } catch (const std::exception& e) {
    return fail(INLA_ERR_INVALID, e.what());
  } catch (...) {
    return fail(INLA_ERR_INTERNAL, "unknown exception");
  }
}

int status_to_code(int st) {
  if (st == kStatusOk) return INLA_OK;
  if (st & kStatusSchedule) return INLA_ERR_CUDA;  // the persistent schedule stopped early
  return INLA_ERR_SINGULAR;  // sparse_ldlt.rs:117-120,140-142: tiny or non-finite pivot => Singular
}

void check_pattern(int64_t n, const int64_t* colptr, const int64_t* rowidx) {
  if (n <= 0 || !colptr || (!rowidx && colptr[n] > 0)) throw InlaError(INLA_ERR_INVALID, "invalid CSC pattern");
}

// Stream bridge: order our stream after `ext`, and `ext` after our work.
// ext == NULL is the legacy default stream (it does not synchronize with the
// handle's non-blocking stream by itself, so it is bridged like any other).
struct StreamBridge {
  cudaStream_t own, ext;
  cudaEvent_t ev;
  StreamBridge(cudaStream_t own_, cudaStream_t ext_) : own(own_), ext(ext_), ev(nullptr) {
    if (ext != own) {
      INLA_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      INLA_CUDA(cudaEventRecord(ev, ext));
      INLA_CUDA(cudaStreamWaitEvent(own, ev, 0));
    }
  }
  void done() {
    if (ev) {
      INLA_CUDA(cudaEventRecord(ev, own));
      INLA_CUDA(cudaStreamWaitEvent(ext, ev, 0));
    }
  }
  ~StreamBridge() {
    if (ev) cudaEventDestroy(ev);
  }
};

}  // namespace inla

using namespace inla;

struct inla_solver {
  int ordering = INLA_ORDER_AMD;
  std::vector<int64_t> custom_perm;
  cudaStream_t stream = nullptr;
  std::unique_ptr<Symbolic> sym;  // host symbolic analysis of the cached pattern
  std::unique_ptr<GpuFactor> eng;
  bool factored = false;
  double logdet = 0.0;
  DBuf<double> d_vals, d_x, d_logdet_unused;
  PinnedBuf<double> h_stage;
};

struct inla_batch {
  cudaStream_t stream = nullptr;
  std::unique_ptr<GpuFactor> eng;
  int factored_b = 0;
  DBuf<double> d_vals, d_x, d_out, d_logdet;
  DBuf<int> d_status;
};

extern "C" {

const char* inla_last_error(void) { return g_last_error.c_str(); }

int64_t inla_kernel_launches(void) { return g_launches.load(); }

int inla_release_cached_memory(void) {
  try {
    device_release_cached();
    release_symbolic_cache();
    release_host_maps();
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_choose_symmetric_order(int64_t n, const int64_t* colptr, const int64_t* rowidx, int64_t* fwd) {
  try {
    check_pattern(n, colptr, rowidx);
    std::vector<int64_t> f;
    int kind = choose_symmetric_order(n, colptr, rowidx, f);
    if (fwd && !f.empty()) std::memcpy(fwd, f.data(), sizeof(int64_t) * n);
    return kind;
  } catch (...) {
    return -map_exception();
  }
}

int inla_solver_new(int ordering, inla_solver** out) {
  try {
    if (!out) return fail(INLA_ERR_INVALID, "null output handle");
    if (ordering < 0 || ordering > INLA_ORDER_ND) return fail(INLA_ERR_INVALID, "unsupported ordering");
    auto* s = new inla_solver();
    s->ordering = ordering;
    *out = s;
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

void inla_solver_free(inla_solver* s) {
  if (!s) return;
  s->eng.reset();
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

static bool same_pattern(const Symbolic* S, int64_t n, const int64_t* colptr, const int64_t* rowidx) {
  if (!S || S->n != n) return false;
  const int64_t nnz = colptr[n];
  return (int64_t)S->rowidx.size() == nnz &&
         std::memcmp(S->colptr.data(), colptr, sizeof(int64_t) * (n + 1)) == 0 &&
         std::memcmp(S->rowidx.data(), rowidx, sizeof(int64_t) * nnz) == 0;
}

// Host-only part of factorize: (re)run the symbolic analysis when the pattern
// differs from the cached one.
static void solver_analyze(inla_solver* s, int64_t n, const int64_t* colptr, const int64_t* rowidx) {
  check_pattern(n, colptr, rowidx);
  if (same_pattern(s->sym.get(), n, colptr, rowidx)) return;
  s->factored = false;
  s->eng.reset();
  s->sym.reset();
  std::unique_ptr<Symbolic> sym(new Symbolic());
  SymbolicOptions opt;
  opt.ordering = s->ordering;
  if (s->ordering == INLA_ORDER_CUSTOM && (int64_t)s->custom_perm.size() != n)
    throw InlaError(INLA_ERR_DIM_MISMATCH, "custom permutation length does not match n");
  analyze(n, colptr, rowidx, opt, s->ordering == INLA_ORDER_CUSTOM ? s->custom_perm.data() : nullptr, *sym);
  s->sym = std::move(sym);
}

int inla_solver_set_perm(inla_solver* s, int64_t n, const int64_t* perm) {
  try {
    if (!s || !perm || n <= 0) return fail(INLA_ERR_INVALID, "invalid permutation");
    s->custom_perm.assign(perm, perm + n);
    s->ordering = INLA_ORDER_CUSTOM;
    s->sym.reset();
    s->eng.reset();
    s->factored = false;
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_solver_analyze(inla_solver* s, int64_t n, const int64_t* colptr, const int64_t* rowidx) {
  try {
    if (!s) return fail(INLA_ERR_INVALID, "null solver");
    solver_analyze(s, n, colptr, rowidx);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_solver_factorize(inla_solver* s, int64_t n, const int64_t* colptr, const int64_t* rowidx,
                          const double* values) {
  try {
    if (!s) return fail(INLA_ERR_INVALID, "null solver");
    if (!values) return fail(INLA_ERR_INVALID, "null values");
    solver_analyze(s, n, colptr, rowidx);
    if (!s->stream) INLA_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    if (!s->eng) s->eng.reset(new GpuFactor(*s->sym, 1, s->stream));
    s->factored = false;
    GpuFactor& E = *s->eng;
    const int64_t nnz = colptr[n];
    s->d_vals.alloc(nnz);
    INLA_CUDA(cudaMemcpyAsync(s->d_vals.p, values, sizeof(double) * nnz, cudaMemcpyHostToDevice, s->stream));
    int64_t before = E.launches();
    E.factor_values(s->d_vals.p, 1);
    g_launches += E.launches() - before;
    double ld = 0;
    int st = 0;
    INLA_CUDA(cudaMemcpyAsync(&ld, E.d_logdet(), sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    INLA_CUDA(cudaMemcpyAsync(&st, E.d_status(), sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    INLA_CUDA(cudaStreamSynchronize(s->stream));
    E.check_schedule();
    int code = status_to_code(st);
    if (code != INLA_OK) return fail(code, "Matrix is singular or structurally rank-deficient");
    s->logdet = ld;
    s->factored = true;
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_solver_solve(inla_solver* s, const double* rhs, double* x) {
  try {
    if (!s) return fail(INLA_ERR_INVALID, "null solver");
    if (!s->factored) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *s->eng;
    const int64_t n = E.sym().n;
    s->d_x.alloc(n);
    INLA_CUDA(cudaMemcpyAsync(s->d_x.p, rhs, sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
    int64_t before = E.launches();
    E.solve(s->d_x.p, n, 1);
    g_launches += E.launches() - before;
    INLA_CUDA(cudaMemcpyAsync(x, s->d_x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    INLA_CUDA(cudaStreamSynchronize(s->stream));
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_solver_diag_inv(inla_solver* s, double* diag) {
  try {
    if (!s) return fail(INLA_ERR_INVALID, "null solver");
    if (!s->factored) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *s->eng;
    const int64_t n = E.sym().n;
    s->d_x.alloc(n);
    int64_t before = E.launches();
    E.selinv(1);
    E.extract_diag(s->d_x.p, n, 1);
    g_launches += E.launches() - before;
    INLA_CUDA(cudaMemcpyAsync(diag, s->d_x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s->stream));
    INLA_CUDA(cudaStreamSynchronize(s->stream));
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_solver_log_abs_det(const inla_solver* s, double* out) {
  if (!s) return fail(INLA_ERR_INVALID, "null solver");
  if (!s->factored) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
  *out = s->logdet;
  return INLA_OK;
}

int inla_solver_selinv_pattern(inla_solver* s, double* sigma) {
  try {
    if (!s) return fail(INLA_ERR_INVALID, "null solver");
    if (!s->factored) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *s->eng;
    const int64_t nnz = E.nnz();
    s->d_x.alloc(nnz);
    int64_t before = E.launches();
    E.selinv(1);
    E.sigma_on_pattern(s->d_x.p, 1);
    g_launches += E.launches() - before;
    INLA_CUDA(cudaMemcpyAsync(sigma, s->d_x.p, sizeof(double) * nnz, cudaMemcpyDeviceToHost, s->stream));
    INLA_CUDA(cudaStreamSynchronize(s->stream));
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

static int fill_info(const Symbolic& S, int64_t ftotal, int64_t* info) {
  info[0] = S.n;
  info[1] = S.nnz_l;
  info[2] = S.nnz_l_stored;
  info[3] = S.nsuper;
  info[4] = S.nlevels;
  info[5] = S.max_m;
  info[6] = S.order_used;
  info[7] = ftotal;
  return INLA_OK;
}

int inla_solver_info(const inla_solver* s, int64_t* info) {
  if (!s || !s->sym) return fail(INLA_ERR_NOT_FACTORED, "no symbolic analysis yet");
  int64_t ft = 0;
  for (int64_t t = 0; t < s->sym->nsuper; ++t) {
    int64_t m = s->sym->sn_rowptr[t + 1] - s->sym->sn_rowptr[t];
    ft += m * m;
  }
  return fill_info(*s->sym, ft, info);
}

int inla_solver_perm(const inla_solver* s, int64_t* perm) {
  if (!s || !s->sym) return fail(INLA_ERR_NOT_FACTORED, "no symbolic analysis yet");
  std::memcpy(perm, s->sym->perm.data(), sizeof(int64_t) * s->sym->n);
  return INLA_OK;
}

int inla_solver_etree(const inla_solver* s, int64_t* parent) {
  if (!s || !s->sym) return fail(INLA_ERR_NOT_FACTORED, "no symbolic analysis yet");
  std::memcpy(parent, s->sym->etree.data(), sizeof(int64_t) * s->sym->n);
  return INLA_OK;
}

int inla_solver_supernodes(const inla_solver* s, int64_t* first, int64_t* count) {
  if (!s || !s->sym) return fail(INLA_ERR_NOT_FACTORED, "no symbolic analysis yet");
  const Symbolic& S = *s->sym;
  if (count) *count = S.nsuper;
  if (first) std::memcpy(first, S.sn_first.data(), sizeof(int64_t) * (S.nsuper + 1));
  return INLA_OK;
}

int inla_solver_check_schedule(const inla_solver* s, int64_t* info3) {
  try {
    if (!s || !s->sym) return fail(INLA_ERR_NOT_FACTORED, "no symbolic analysis yet");
    std::vector<int> flat;
    const std::vector<LevelPlan> levels = make_level_plans(*s->sym, flat);
    PersistPlan pl;
    const bool fits = make_persist_plan(*s->sym, levels, pl);
    std::string err = check_persist_plan(*s->sym, pl);
    if (err.empty()) {
      PersistPlan sp;
      make_solve_plan(*s->sym, levels, sp);
      err = check_solve_plan(*s->sym, sp);
      if (!err.empty()) err = "solve: " + err;
    }
    if (info3) {
      info3[0] = (int64_t)(pl.task.size() / 6);
      info3[1] = pl.smem;
      info3[2] = fits ? 1 : 0;
    }
    if (!err.empty()) return fail(INLA_ERR_INTERNAL, "persistent schedule: " + err);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_solver_colcounts(const inla_solver* s, int64_t* counts) {
  if (!s || !s->sym) return fail(INLA_ERR_NOT_FACTORED, "no symbolic analysis yet");
  std::memcpy(counts, s->sym->colcount.data(), sizeof(int64_t) * s->sym->n);
  return INLA_OK;
}

// ---------------------------------------------------------------------------
// batched engine
// ---------------------------------------------------------------------------

int inla_batch_create(int64_t n, const int64_t* colptr, const int64_t* rowidx, int ordering, int max_batch,
                      inla_batch** out) {
  inla_batch* h = nullptr;
  try {
    if (!out) return fail(INLA_ERR_INVALID, "null output handle");
    check_pattern(n, colptr, rowidx);
    if (max_batch < 1) return fail(INLA_ERR_INVALID, "max_batch must be >= 1");
    h = new inla_batch();
    INLA_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    Symbolic sym;
    SymbolicOptions opt;
    opt.ordering = ordering;
    analyze(n, colptr, rowidx, opt, nullptr, sym);
    h->eng.reset(new GpuFactor(sym, max_batch, h->stream));
    *out = h;
    return INLA_OK;
  } catch (...) {
    int code = map_exception();
    inla_batch_free(h);
    return code;
  }
}

void inla_batch_free(inla_batch* h) {
  if (!h) return;
  h->eng.reset();
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

int inla_set_persistent_schedule(int mode) {
  if (mode < 0 || mode > 2) return fail(INLA_ERR_INVALID, "schedule mode must be 0, 1 or 2");
  set_persistent_default(mode);
  return INLA_OK;
}

int inla_set_panel_form(int form) {
  if (form < -1 || form > 2) return fail(INLA_ERR_INVALID, "panel form must be -1, 0, 1 or 2");
  set_panel_form(form);
  return INLA_OK;
}

int inla_batch_schedule(inla_batch* h, int* persistent) {
  if (!h || !h->eng || !persistent) return fail(INLA_ERR_INVALID, "null batch handle or output");
  *persistent = h->eng->persistent() ? 1 : 0;
  return INLA_OK;
}

int inla_batch_wait_limit_selftest(inla_batch* h, double limit_ms, int* code) {
  try {
    if (!h || !h->eng || !code || !(limit_ms > 0.0)) return fail(INLA_ERR_INVALID, "invalid argument");
    if (!h->eng->persistent()) return fail(INLA_ERR_INVALID, "the handle does not use the persistent schedule");
    *code = h->eng->persist_wait_limit_selftest(limit_ms);
    h->factored_b = 0;  // the fronts hold nothing usable now
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

static void check_batch(inla_batch* h, int B) {
  if (!h || !h->eng) throw InlaError(INLA_ERR_INVALID, "null batch handle");
  if (B < 1 || B > h->eng->max_batch()) throw InlaError(INLA_ERR_DIM_MISMATCH, "batch size out of range");
}

int inla_batch_factorize_dev(inla_batch* h, int B, const double* d_values, double* d_logdet, int* d_status,
                             void* stream) {
  try {
    check_batch(h, B);
    GpuFactor& E = *h->eng;
    StreamBridge br(h->stream, (cudaStream_t)stream);
    int64_t before = E.launches();
    E.factor_values(d_values, B);
    if (d_logdet)
      INLA_CUDA(cudaMemcpyAsync(d_logdet, E.d_logdet(), sizeof(double) * B, cudaMemcpyDeviceToDevice, h->stream));
    if (d_status)
      INLA_CUDA(cudaMemcpyAsync(d_status, E.d_status(), sizeof(int) * B, cudaMemcpyDeviceToDevice, h->stream));
    g_launches += E.launches() - before;
    h->factored_b = B;
    br.done();
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_batch_factorize(inla_batch* h, int B, const double* values, double* logdet, int* status) {
  try {
    check_batch(h, B);
    GpuFactor& E = *h->eng;
    const int64_t nnz = E.nnz();
    h->d_vals.alloc((size_t)B * nnz);
    INLA_CUDA(cudaMemcpyAsync(h->d_vals.p, values, sizeof(double) * B * nnz, cudaMemcpyHostToDevice, h->stream));
    int64_t before = E.launches();
    E.factor_values(h->d_vals.p, B);
    g_launches += E.launches() - before;
    std::vector<int> st(B);
    std::vector<double> ld(B);
    INLA_CUDA(cudaMemcpyAsync(ld.data(), E.d_logdet(), sizeof(double) * B, cudaMemcpyDeviceToHost, h->stream));
    INLA_CUDA(cudaMemcpyAsync(st.data(), E.d_status(), sizeof(int) * B, cudaMemcpyDeviceToHost, h->stream));
    INLA_CUDA(cudaStreamSynchronize(h->stream));
    E.check_schedule();
    int code = INLA_OK;
    for (int b = 0; b < B; ++b) {
      if (logdet) logdet[b] = ld[b];
      if (status) status[b] = status_to_code(st[b]);
      if (st[b] != kStatusOk) code = INLA_ERR_SINGULAR;
    }
    h->factored_b = B;
    if (code != INLA_OK) return fail(code, "at least one batch member is singular");
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_batch_solve_dev(inla_batch* h, int B, double* d_x, void* stream) {
  try {
    check_batch(h, B);
    if (B > h->factored_b) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *h->eng;
    StreamBridge br(h->stream, (cudaStream_t)stream);
    int64_t before = E.launches();
    E.solve(d_x, E.sym().n, B);
    g_launches += E.launches() - before;
    br.done();
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_batch_solve(inla_batch* h, int B, const double* rhs, double* x) {
  try {
    check_batch(h, B);
    if (B > h->factored_b) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *h->eng;
    const int64_t n = E.sym().n;
    h->d_x.alloc((size_t)B * n);
    INLA_CUDA(cudaMemcpyAsync(h->d_x.p, rhs, sizeof(double) * B * n, cudaMemcpyHostToDevice, h->stream));
    int64_t before = E.launches();
    E.solve(h->d_x.p, n, B);
    g_launches += E.launches() - before;
    INLA_CUDA(cudaMemcpyAsync(x, h->d_x.p, sizeof(double) * B * n, cudaMemcpyDeviceToHost, h->stream));
    INLA_CUDA(cudaStreamSynchronize(h->stream));
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_batch_diag_inv_dev(inla_batch* h, int B, double* d_diag, void* stream) {
  try {
    check_batch(h, B);
    if (B > h->factored_b) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *h->eng;
    StreamBridge br(h->stream, (cudaStream_t)stream);
    int64_t before = E.launches();
    E.selinv(B);
    E.extract_diag(d_diag, E.sym().n, B);
    g_launches += E.launches() - before;
    br.done();
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_batch_diag_inv(inla_batch* h, int B, double* diag) {
  try {
    check_batch(h, B);
    if (B > h->factored_b) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *h->eng;
    const int64_t n = E.sym().n;
    h->d_out.alloc((size_t)B * n);
    int64_t before = E.launches();
    E.selinv(B);
    E.extract_diag(h->d_out.p, n, B);
    g_launches += E.launches() - before;
    INLA_CUDA(cudaMemcpyAsync(diag, h->d_out.p, sizeof(double) * B * n, cudaMemcpyDeviceToHost, h->stream));
    INLA_CUDA(cudaStreamSynchronize(h->stream));
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_batch_selinv_pattern_dev(inla_batch* h, int B, double* d_sigma, void* stream) {
  try {
    check_batch(h, B);
    if (B > h->factored_b) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *h->eng;
    StreamBridge br(h->stream, (cudaStream_t)stream);
    int64_t before = E.launches();
    E.selinv(B);
    E.sigma_on_pattern(d_sigma, B);
    g_launches += E.launches() - before;
    br.done();
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_batch_selinv_pattern(inla_batch* h, int B, double* sigma) {
  try {
    check_batch(h, B);
    if (B > h->factored_b) return fail(INLA_ERR_NOT_FACTORED, "Factorization not computed yet");
    GpuFactor& E = *h->eng;
    const int64_t nnz = E.nnz();
    h->d_out.alloc((size_t)B * nnz);
    int64_t before = E.launches();
    E.selinv(B);
    E.sigma_on_pattern(h->d_out.p, B);
    g_launches += E.launches() - before;
    INLA_CUDA(cudaMemcpyAsync(sigma, h->d_out.p, sizeof(double) * B * nnz, cudaMemcpyDeviceToHost, h->stream));
    INLA_CUDA(cudaStreamSynchronize(h->stream));
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

}  // extern "C"
