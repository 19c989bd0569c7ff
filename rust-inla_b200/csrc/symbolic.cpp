// Symbolic analysis: ordering choice, elimination tree, column counts,
// relaxed supernodes, row structures, level schedule and index maps.
#include "symbolic.hpp"

#include "host_par.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <list>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <tuple>

namespace inla {

// ---------------------------------------------------------------------------
// ordering.rs restatements (bit-exact choice logic)
// ---------------------------------------------------------------------------

// ordering.rs:8-18 — max(row - col) over stored entries with row >= col.
int64_t lower_bandwidth(int64_t n, const int64_t* colptr, const int64_t* rowidx) {
  int64_t bw = 0;
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      int64_t r = rowidx[p];
      if (r >= c) bw = std::max(bw, r - c);
    }
  return bw;
}

// ordering.rs:21-30 — bandwidth after new = fwd[old], over all stored entries.
int64_t bandwidth_with_fwd(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                           const int64_t* fwd) {
  int64_t bw = 0;
  for (int64_t c = 0; c < n; ++c) {
    int64_t jc = fwd[c];
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      int64_t d = fwd[rowidx[p]] - jc;
      bw = std::max(bw, d < 0 ? -d : d);
    }
  }
  return bw;
}

// ordering.rs:36-49 — mixture-major c*n_time+t -> time-major t*n_comp+c.
static void mixture_to_time_major(int64_t n_time, int64_t n_comp, std::vector<int64_t>& fwd) {
  fwd.assign(n_time * n_comp, 0);
  for (int64_t c = 0; c < n_comp; ++c)
    for (int64_t t = 0; t < n_time; ++t) fwd[c * n_time + t] = t * n_comp + c;
}

// ordering.rs:56-89
bool try_time_major_kronecker(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                              std::vector<int64_t>& fwd_out) {
  if (n < 16) return false;
  int64_t bw = lower_bandwidth(n, colptr, rowidx);
  if (bw < n / 8) return false;
  bool have = false;
  int64_t best_bw = 0;
  std::vector<int64_t> best, fwd;
  for (int64_t n_comp = 2; n_comp <= 8; ++n_comp) {
    if (n % n_comp != 0) continue;
    int64_t n_time = n / n_comp;
    if (n_time < 8) continue;
    mixture_to_time_major(n_time, n_comp, fwd);
    int64_t bw_new = bandwidth_with_fwd(n, colptr, rowidx, fwd.data());
    if (bw_new < bw) {
      if (!(have && best_bw <= bw_new)) {
        have = true;
        best_bw = bw_new;
        best = fwd;
      }
    }
  }
  if (!have) return false;
  int64_t nnz = colptr[n];
  int64_t per = std::max<int64_t>(nnz / std::max<int64_t>(n, 1), 2);
  if (best_bw * 4 < bw || best_bw <= 4 * per) {
    fwd_out = best;
    return true;
  }
  return false;
}

// ordering.rs:92-140 — RCM; neighbours sorted by (degree, index), start node
// is the unvisited node of minimum (degree, index).
void reverse_cuthill_mckee(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                           std::vector<int64_t>& fwd) {
  std::vector<std::vector<int64_t>> adj(n);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      int64_t r = rowidx[p];
      if (r != c) {
        adj[c].push_back(r);
        adj[r].push_back(c);
      }
    }
  for (auto& a : adj) {
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
  }
  std::vector<int64_t> deg(n);
  for (int64_t i = 0; i < n; ++i) deg[i] = (int64_t)adj[i].size();
  for (auto& a : adj)
    std::stable_sort(a.begin(), a.end(), [&](int64_t x, int64_t y) {
      return std::make_pair(deg[x], x) < std::make_pair(deg[y], y);
    });
  std::vector<char> visited(n, 0);
  std::vector<int64_t> order;
  order.reserve(n);
  // Candidate starts in (degree, index) order; skipping visited ones gives the
  // same choice as a fresh minimum scan per component.
  std::vector<int64_t> cand(n);
  std::iota(cand.begin(), cand.end(), 0);
  std::stable_sort(cand.begin(), cand.end(), [&](int64_t x, int64_t y) {
    return std::make_pair(deg[x], x) < std::make_pair(deg[y], y);
  });
  size_t ci = 0;
  std::deque<int64_t> q;
  while (true) {
    while (ci < cand.size() && visited[cand[ci]]) ++ci;
    if (ci >= cand.size()) break;
    int64_t start = cand[ci];
    visited[start] = 1;
    q.push_back(start);
    while (!q.empty()) {
      int64_t u = q.front();
      q.pop_front();
      order.push_back(u);
      for (int64_t v : adj[u])
        if (!visited[v]) {
          visited[v] = 1;
          q.push_back(v);
        }
    }
  }
  std::reverse(order.begin(), order.end());
  fwd.assign(n, 0);
  for (int64_t k = 0; k < n; ++k) fwd[order[k]] = k;
}

// ordering.rs:149-162
int choose_symmetric_order(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                           std::vector<int64_t>& fwd) {
  int64_t bw = lower_bandwidth(n, colptr, rowidx);
  if (try_time_major_kronecker(n, colptr, rowidx, fwd)) return ORDER_TIME_MAJOR;
  if (bw > 32) {
    reverse_cuthill_mckee(n, colptr, rowidx, fwd);
    int64_t bw_new = bandwidth_with_fwd(n, colptr, rowidx, fwd.data());
    if (bw_new * 2 < bw) return ORDER_RCM;
  }
  fwd.clear();
  return ORDER_AMD;
}

// ---------------------------------------------------------------------------
// analysis
// ---------------------------------------------------------------------------

namespace {

// Upper-triangle pattern of P A P^T by columns: for column j the rows i < j (unsorted).
void permuted_upper(int64_t n, const int64_t* colptr, const int64_t* rowidx,
                    const std::vector<int64_t>& iperm, std::vector<int64_t>& uptr,
                    std::vector<int64_t>& uidx) {
  uptr.assign(n + 1, 0);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      int64_t r = rowidx[p];
      if (r <= c) continue;  // lower entries (row > col) define the symmetric pattern
      int64_t i = iperm[r], j = iperm[c];
      if (i > j) std::swap(i, j);
      uptr[j + 1]++;
    }
  for (int64_t j = 0; j < n; ++j) uptr[j + 1] += uptr[j];
  uidx.assign(uptr[n], 0);
  std::vector<int64_t> fill(uptr.begin(), uptr.end() - 1);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      int64_t r = rowidx[p];
      if (r <= c) continue;
      int64_t i = iperm[r], j = iperm[c];
      if (i > j) std::swap(i, j);
      uidx[fill[j]++] = i;
    }
}

// Liu's elimination tree of P A P^T with path compression, read straight from the
// input columns (full symmetric pattern): column k of P A P^T is input column perm[k],
// its rows i < k are the permuted rows below k. The tree does not depend on the order
// in which a column's rows are visited.
void etree_permuted(int64_t n, const int64_t* colptr, const int64_t* rowidx, const std::vector<int64_t>& perm,
                    const std::vector<int64_t>& iperm, std::vector<int64_t>& parent) {
  parent.assign(n, -1);
  std::vector<int64_t> anc(n, -1);
  for (int64_t k = 0; k < n; ++k) {
    const int64_t c = perm[k];
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      int64_t i = iperm[rowidx[p]];
      while (i != -1 && i < k) {
        int64_t next = anc[i];
        anc[i] = k;
        if (next == -1) parent[i] = k;
        i = next;
      }
    }
  }
}

void postorder(int64_t n, const std::vector<int64_t>& parent, std::vector<int64_t>& post) {
  std::vector<int64_t> head(n, -1), next(n, -1);
  for (int64_t j = n - 1; j >= 0; --j) {
    int64_t p = parent[j];
    if (p == -1) continue;
    next[j] = head[p];
    head[p] = j;
  }
  post.clear();
  post.reserve(n);
  std::vector<int64_t> stack;
  for (int64_t r = 0; r < n; ++r) {
    if (parent[r] != -1) continue;
    stack.push_back(r);
    while (!stack.empty()) {
      int64_t top = stack.back();
      int64_t c = head[top];
      if (c == -1) {
        stack.pop_back();
        post.push_back(top);
      } else {
        head[top] = next[c];
        stack.push_back(c);
      }
    }
  }
}

}  // namespace

static void analyze_uncached(int64_t n, const int64_t* colptr, const int64_t* rowidx, const SymbolicOptions& opt,
                             const int64_t* custom_perm, Symbolic& S) {
  const bool dbg = std::getenv("INLA_DEBUG") != nullptr;
  auto tprev = std::chrono::steady_clock::now();
  auto phase = [&](const char* name) {
    if (!dbg) return;
    const auto t = std::chrono::steady_clock::now();
    std::fprintf(stderr, "symbolic: %s %.1f ms\n", name, std::chrono::duration<double, std::milli>(t - tprev).count());
    tprev = t;
  };
  if (n <= 0) throw std::runtime_error("symbolic: n must be > 0");
  if (colptr[0] != 0) throw std::runtime_error("symbolic: colptr[0] must be 0");
  for (int64_t c = 0; c < n; ++c) {
    if (colptr[c + 1] < colptr[c]) throw std::runtime_error("symbolic: colptr not monotone");
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p)
      if (rowidx[p] < 0 || rowidx[p] >= n) throw std::runtime_error("symbolic: row index out of bounds");
  }
  S = Symbolic();
  S.n = n;
  const int64_t nnz = colptr[n];
  S.colptr.assign(colptr, colptr + n + 1);
  S.rowidx.assign(rowidx, rowidx + nnz);

  // ---- ordering -----------------------------------------------------------
  std::vector<int64_t> fwd, perm0(n);
  int kind = opt.ordering;
  if (kind == ORDER_AUTO) {
    kind = choose_symmetric_order(n, colptr, rowidx, fwd);
  } else if (kind == ORDER_RCM) {
    reverse_cuthill_mckee(n, colptr, rowidx, fwd);
  } else if (kind == ORDER_TIME_MAJOR) {
    if (!try_time_major_kronecker(n, colptr, rowidx, fwd)) kind = ORDER_AMD;
  }
  S.order_used = kind;
  if (kind == ORDER_AMD) {
    amd_order(n, colptr, rowidx, perm0);
  } else if (kind == ORDER_ND) {
    nd_order(n, colptr, rowidx, perm0);
  } else if (kind == ORDER_NATURAL) {
    std::iota(perm0.begin(), perm0.end(), 0);
  } else if (kind == ORDER_CUSTOM) {
    if (!custom_perm) throw std::runtime_error("symbolic: custom ordering requires a permutation");
    std::vector<char> seen(n, 0);
    for (int64_t k = 0; k < n; ++k) {
      int64_t o = custom_perm[k];
      if (o < 0 || o >= n || seen[o]) throw std::runtime_error("symbolic: invalid custom permutation");
      seen[o] = 1;
      perm0[k] = o;
    }
  } else {  // RCM / time-major give fwd (old -> new)
    for (int64_t o = 0; o < n; ++o) perm0[fwd[o]] = o;
  }
  phase("ordering");
  std::vector<int64_t> iperm0(n);
  for (int64_t k = 0; k < n; ++k) iperm0[perm0[k]] = k;

  // ---- etree + postorder ----------------------------------------------------
  std::vector<int64_t> uptr, uidx, parent0, post;
  etree_permuted(n, colptr, rowidx, perm0, iperm0, parent0);
  postorder(n, parent0, post);
  S.perm.resize(n);
  S.iperm.resize(n);
  for (int64_t k = 0; k < n; ++k) S.perm[k] = perm0[post[k]];
  for (int64_t k = 0; k < n; ++k) S.iperm[S.perm[k]] = k;
  // the postorder relabels the same tree: parent of k is the relabeled parent of post[k]
  {
    std::vector<int64_t> ipost(n);
    for (int64_t k = 0; k < n; ++k) ipost[post[k]] = k;
    S.etree.assign(n, -1);
    for (int64_t k = 0; k < n; ++k) {
      const int64_t q = parent0[post[k]];
      S.etree[k] = q == -1 ? -1 : ipost[q];
    }
  }
  permuted_upper(n, colptr, rowidx, S.iperm, uptr, uidx);
  const std::vector<int64_t>& par = S.etree;

  phase("etree + postorder");
  // ---- column counts (row-subtree traversal) ------------------------------
  S.colcount.assign(n, 1);
  {
    std::vector<int64_t> mark(n, -1);
    for (int64_t k = 0; k < n; ++k) {
      mark[k] = k;
      for (int64_t p = uptr[k]; p < uptr[k + 1]; ++p) {
        int64_t j = uidx[p];
        while (j != -1 && mark[j] != k) {
          S.colcount[j]++;
          mark[j] = k;
          j = par[j];
        }
      }
    }
  }
  S.nnz_l = 0;
  S.flops_factor = S.flops_selinv = 0;
  for (int64_t j = 0; j < n; ++j) {
    double c = (double)(S.colcount[j] - 1);
    S.nnz_l += S.colcount[j];
    S.flops_factor += c * c + 2 * c;
    S.flops_selinv += 2 * c * c + 2 * c;
  }
  S.flops_solve = 4.0 * (double)S.nnz_l + (double)n;

  phase("column counts");
  // ---- fundamental supernodes ---------------------------------------------
  std::vector<int64_t> nchild(n, 0);
  for (int64_t j = 0; j < n; ++j)
    if (par[j] != -1) nchild[par[j]]++;
  std::vector<int64_t> fstart;  // fundamental supernode starts
  for (int64_t j = 0; j < n; ++j) {
    bool cont = j > 0 && par[j - 1] == j && S.colcount[j - 1] == S.colcount[j] + 1 && nchild[j] == 1 &&
                (j - fstart.back()) < opt.max_width;
    if (!cont) fstart.push_back(j);
  }
  int64_t nf = (int64_t)fstart.size();
  fstart.push_back(n);

  // ---- relaxed amalgamation -------------------------------------------------
  // Work on groups of consecutive fundamental supernodes. A group ending just
  // before fundamental supernode t (its last child in postorder) may merge into
  // t when the criteria hold. Track per group: first column, width, true nnz.
  std::vector<int64_t> fparent(nf, -1);
  std::vector<int64_t> col2f(n);
  for (int64_t f = 0; f < nf; ++f)
    for (int64_t j = fstart[f]; j < fstart[f + 1]; ++j) col2f[j] = f;
  for (int64_t f = 0; f < nf; ++f) {
    int64_t last = fstart[f + 1] - 1;
    fparent[f] = par[last] == -1 ? -1 : col2f[par[last]];
  }
  // Merge decisions, bottom-up. group_of[f] = representative (the top-most
  // fundamental supernode of the merged group, i.e. the one whose columns end
  // the group). Groups are contiguous column ranges.
  std::vector<int64_t> gfirst(nf), gwidth(nf), gnnz(nf), gm_top(nf);
  for (int64_t f = 0; f < nf; ++f) {
    int64_t k = fstart[f + 1] - fstart[f];
    int64_t m = S.colcount[fstart[f]];  // rows of the first column (incl. diagonal)
    gfirst[f] = fstart[f];
    gwidth[f] = k;
    gm_top[f] = m - (k - 1);            // rows of the last column
    int64_t nz = 0;
    for (int64_t j = fstart[f]; j < fstart[f + 1]; ++j) nz += S.colcount[j];
    gnnz[f] = nz;
  }
  std::vector<char> merged_into_next(nf, 0);
  // `cur` is the group currently ending at fundamental supernode f-1.
  for (int64_t f = 1; f < nf; ++f) {
    int64_t c = f - 1;  // group ending at c (represented by c)
    if (fparent[c] != f) continue;  // only the last child is contiguous
    int64_t kc = gwidth[c], kp = gwidth[f];
    int64_t ns = kc + kp;
    if (ns > opt.max_width) continue;
    // Merged panel: columns [gfirst[c], last of f]; rows of the merged first
    // column = kc + (rows of f's first column) since struct(c)_below ⊆ struct(f).
    int64_t mp_first = S.colcount[fstart[f]];
    int64_t m_merged = kc + mp_first;
    // true entries in the lower trapezoid of the merged panel
    double total = 0;
    for (int64_t t = 0; t < ns; ++t) total += (double)(m_merged - t);
    double nz_true = (double)(gnnz[c] + gnnz[f]);
    double z = (total - nz_true) / total;
    bool ok = ns <= opt.nrelax0 || (ns <= opt.nrelax1 && z < opt.zrelax0) ||
              (ns <= opt.nrelax2 && z < opt.zrelax1) || z < opt.zrelax2;
    if (!ok) continue;
    merged_into_next[c] = 1;
    gfirst[f] = gfirst[c];
    gwidth[f] = ns;
    gnnz[f] = gnnz[c] + gnnz[f];
  }
  // Final supernodes: a group is represented by a fundamental supernode that
  // was not merged into the next one.
  S.sn_first.clear();
  for (int64_t f = 0; f < nf; ++f)
    if (!merged_into_next[f]) S.sn_first.push_back(gfirst[f]);
  S.nsuper = (int64_t)S.sn_first.size();
  S.sn_first.push_back(n);
  const int64_t ns = S.nsuper;
  S.col_to_sn.assign(n, 0);
  for (int64_t s = 0; s < ns; ++s)
    for (int64_t j = S.sn_first[s]; j < S.sn_first[s + 1]; ++j) S.col_to_sn[j] = s;

  phase("supernodes");
  // ---- supernodal row structures + parents ----------------------------------
  // lower pattern of P A P^T by columns: rows > j (from the upper lists).
  std::vector<int64_t> lptr(n + 1, 0), lidx;
  for (int64_t j = 0; j < n; ++j)
    for (int64_t p = uptr[j]; p < uptr[j + 1]; ++p) lptr[uidx[p] + 1]++;
  for (int64_t j = 0; j < n; ++j) lptr[j + 1] += lptr[j];
  lidx.assign(lptr[n], 0);
  {
    std::vector<int64_t> fill(lptr.begin(), lptr.end() - 1);
    for (int64_t j = 0; j < n; ++j)
      for (int64_t p = uptr[j]; p < uptr[j + 1]; ++p) lidx[fill[uidx[p]]++] = j;
  }
  S.sn_parent.assign(ns, -1);
  std::vector<std::vector<int64_t>> kids(ns);
  std::vector<std::vector<int64_t>> rows(ns);
  std::vector<int64_t> mark(n, -1);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t f = S.sn_first[s], l = S.sn_first[s + 1] - 1;
    std::vector<int64_t>& R = rows[s];
    for (int64_t j = f; j <= l; ++j) {
      R.push_back(j);
      mark[j] = s;
    }
    size_t nown = R.size();
    for (int64_t j = f; j <= l; ++j)
      for (int64_t p = lptr[j]; p < lptr[j + 1]; ++p) {
        int64_t i = lidx[p];
        if (i > l && mark[i] != s) {
          mark[i] = s;
          R.push_back(i);
        }
      }
    for (int64_t c : kids[s]) {
      const std::vector<int64_t>& RC = rows[c];
      for (int64_t i : RC)
        if (i > l && mark[i] != s) {
          mark[i] = s;
          R.push_back(i);
        }
    }
    std::sort(R.begin() + nown, R.end());
    if (R.size() > nown) {
      int64_t p = S.col_to_sn[R[nown]];
      S.sn_parent[s] = p;
      kids[p].push_back(s);
    }
  }

  phase("row structures");
  // ---- storage offsets, levels, children CSR --------------------------------
  S.sn_rowptr.assign(ns + 1, 0);
  S.sn_lptr.assign(ns + 1, 0);
  S.sn_uptr.assign(ns + 1, 0);
  S.child_ptr.assign(ns + 1, 0);
  S.sn_level.assign(ns, 0);
  S.max_m = S.max_k = S.max_r = 0;
  for (int64_t s = 0; s < ns; ++s) {
    int64_t m = (int64_t)rows[s].size(), k = S.sn_first[s + 1] - S.sn_first[s], r = m - k;
    S.sn_rowptr[s + 1] = S.sn_rowptr[s] + m;
    S.sn_lptr[s + 1] = S.sn_lptr[s] + m * k;
    S.sn_uptr[s + 1] = S.sn_uptr[s] + r * r;
    S.child_ptr[s + 1] = S.child_ptr[s] + (int64_t)kids[s].size();
    S.max_m = std::max(S.max_m, m);
    S.max_k = std::max(S.max_k, k);
    S.max_r = std::max(S.max_r, r);
    int32_t lv = 0;
    for (int64_t c : kids[s]) lv = std::max(lv, S.sn_level[c] + 1);
    S.sn_level[s] = lv;
  }
  S.nnz_l_stored = S.sn_lptr[ns];
  S.u_total = S.sn_uptr[ns];
  S.sn_rows.resize(S.sn_rowptr[ns]);
  S.child_list.resize(S.child_ptr[ns]);
  for (int64_t s = 0; s < ns; ++s) {
    std::copy(rows[s].begin(), rows[s].end(), S.sn_rows.begin() + S.sn_rowptr[s]);
    std::copy(kids[s].begin(), kids[s].end(), S.child_list.begin() + S.child_ptr[s]);
  }
  S.nlevels = 0;
  for (int64_t s = 0; s < ns; ++s) S.nlevels = std::max(S.nlevels, S.sn_level[s] + 1);
  S.level_ptr.assign(S.nlevels + 1, 0);
  for (int64_t s = 0; s < ns; ++s) S.level_ptr[S.sn_level[s] + 1]++;
  for (int32_t l = 0; l < S.nlevels; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
  S.level_list.assign(ns, 0);
  {
    std::vector<int64_t> fill(S.level_ptr.begin(), S.level_ptr.end() - 1);
    for (int64_t s = 0; s < ns; ++s) S.level_list[fill[S.sn_level[s]]++] = s;
  }

  phase("offsets + levels");
  // ---- extend-add relative maps ---------------------------------------------
  S.rel_ptr.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s) {
    int64_t k = S.sn_first[s + 1] - S.sn_first[s];
    int64_t m = S.sn_rowptr[s + 1] - S.sn_rowptr[s];
    S.rel_ptr[s + 1] = S.rel_ptr[s] + (m - k);
  }
  S.rel.assign(S.rel_ptr[ns], 0);
  {
    std::vector<int32_t> pos(n, -1);
    for (int64_t p = 0; p < ns; ++p) {
      for (int64_t t = S.sn_rowptr[p]; t < S.sn_rowptr[p + 1]; ++t)
        pos[S.sn_rows[t]] = (int32_t)(t - S.sn_rowptr[p]);
      for (int64_t q = S.child_ptr[p]; q < S.child_ptr[p + 1]; ++q) {
        int64_t c = S.child_list[q];
        int64_t k = S.sn_first[c + 1] - S.sn_first[c];
        int64_t base = S.sn_rowptr[c] + k;
        int64_t r = S.sn_rowptr[c + 1] - base;
        for (int64_t t = 0; t < r; ++t) {
          int32_t ps = pos[S.sn_rows[base + t]];
          if (ps < 0) throw std::runtime_error("symbolic: child structure not contained in parent");
          S.rel[S.rel_ptr[c] + t] = ps;
        }
      }
    }
  }

  phase("relative maps");
  // ---- value map: input entry -> L storage ----------------------------------
  S.qmap.assign(nnz, -1);
  parallel_for(n, [&](int64_t c0, int64_t c1) {
    for (int64_t c = c0; c < c1; ++c)
      for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
        int64_t r = rowidx[p];
        if (r < c) continue;
        int64_t i = S.iperm[r], j = S.iperm[c];
        if (i < j) std::swap(i, j);
        int64_t s = S.col_to_sn[j];
        const int64_t* R = S.sn_rows.data() + S.sn_rowptr[s];
        int64_t m = S.sn_rowptr[s + 1] - S.sn_rowptr[s];
        const int64_t* it = std::lower_bound(R, R + m, i);
        if (it == R + m || *it != i) throw std::runtime_error("symbolic: entry outside the filled pattern");
        S.qmap[p] = S.sn_lptr[s] + (j - S.sn_first[s]) * m + (it - R);
      }
  });
  phase("value map");
}

// ---- process-wide cache of analyses --------------------------------------
// The analysis is a deterministic function of (n, colptr, rowidx, opt, custom_perm): the
// ordering threads do not change its result and nothing else is read. Handles created on the
// same pattern (a model rebuilt for new data, a solver per worker) therefore take a copy of the
// cached analysis instead of repeating it. Entries are matched by byte-exact comparison of every
// input, kept most recently used first, and bounded in bytes; INLA_NO_SYMBOLIC_CACHE disables the
// cache.
namespace {

struct SymCacheEntry {
  int64_t n = 0;
  std::vector<int64_t> colptr, rowidx, custom;
  bool has_custom = false;
  SymbolicOptions opt;
  Symbolic sym;
  size_t bytes = 0;
};

constexpr size_t kSymCacheBytes = size_t(1) << 30;

std::mutex g_sym_mu;
std::list<SymCacheEntry> g_sym_cache;  // most recently used first
size_t g_sym_bytes = 0;

template <class T>
size_t vec_bytes(const std::vector<T>& v) {
  return v.size() * sizeof(T);
}

size_t symbolic_bytes(const Symbolic& S) {
  return vec_bytes(S.perm) + vec_bytes(S.iperm) + vec_bytes(S.etree) + vec_bytes(S.colcount) + vec_bytes(S.sn_first) +
         vec_bytes(S.sn_rowptr) + vec_bytes(S.sn_rows) + vec_bytes(S.sn_parent) + vec_bytes(S.sn_lptr) +
         vec_bytes(S.sn_uptr) + vec_bytes(S.sn_level) + vec_bytes(S.col_to_sn) + vec_bytes(S.child_ptr) +
         vec_bytes(S.child_list) + vec_bytes(S.rel_ptr) + vec_bytes(S.rel) + vec_bytes(S.level_ptr) +
         vec_bytes(S.level_list) + vec_bytes(S.colptr) + vec_bytes(S.rowidx) + vec_bytes(S.qmap) + sizeof(Symbolic);
}

bool same_options(const SymbolicOptions& a, const SymbolicOptions& b) {
  return a.ordering == b.ordering && a.nrelax0 == b.nrelax0 && a.nrelax1 == b.nrelax1 && a.nrelax2 == b.nrelax2 &&
         a.zrelax0 == b.zrelax0 && a.zrelax1 == b.zrelax1 && a.zrelax2 == b.zrelax2 && a.max_width == b.max_width;
}

bool same_inputs(const SymCacheEntry& e, int64_t n, const int64_t* colptr, const int64_t* rowidx,
                 const SymbolicOptions& opt, const int64_t* custom_perm) {
  if (e.n != n || e.has_custom != (custom_perm != nullptr) || !same_options(e.opt, opt)) return false;
  const int64_t nnz = colptr[n];
  if ((int64_t)e.rowidx.size() != nnz) return false;
  if (std::memcmp(e.colptr.data(), colptr, sizeof(int64_t) * (n + 1)) != 0) return false;
  if (std::memcmp(e.rowidx.data(), rowidx, sizeof(int64_t) * nnz) != 0) return false;
  if (custom_perm && std::memcmp(e.custom.data(), custom_perm, sizeof(int64_t) * n) != 0) return false;
  return true;
}

bool sym_cache_enabled() {
  static const bool on = std::getenv("INLA_NO_SYMBOLIC_CACHE") == nullptr;
  return on;
}

}  // namespace

void analyze(int64_t n, const int64_t* colptr, const int64_t* rowidx, const SymbolicOptions& opt,
             const int64_t* custom_perm, Symbolic& S) {
  // inputs the cache compares must be readable: reject what the analysis would reject
  if (n <= 0) throw std::runtime_error("symbolic: n must be > 0");
  if (colptr[0] != 0) throw std::runtime_error("symbolic: colptr[0] must be 0");
  for (int64_t c = 0; c < n; ++c)
    if (colptr[c + 1] < colptr[c]) throw std::runtime_error("symbolic: colptr not monotone");
  if (sym_cache_enabled()) {
    std::lock_guard<std::mutex> lock(g_sym_mu);
    for (auto it = g_sym_cache.begin(); it != g_sym_cache.end(); ++it)
      if (same_inputs(*it, n, colptr, rowidx, opt, custom_perm)) {
        S = it->sym;
        g_sym_cache.splice(g_sym_cache.begin(), g_sym_cache, it);
        return;
      }
  }
  analyze_uncached(n, colptr, rowidx, opt, custom_perm, S);
  static std::atomic<uint64_t> next_id{1};
  S.id = next_id.fetch_add(1);
  if (!sym_cache_enabled()) return;
  SymCacheEntry e;
  e.n = n;
  e.colptr.assign(colptr, colptr + n + 1);
  e.rowidx.assign(rowidx, rowidx + colptr[n]);
  e.has_custom = custom_perm != nullptr;
  if (custom_perm) e.custom.assign(custom_perm, custom_perm + n);
  e.opt = opt;
  e.bytes = symbolic_bytes(S) + vec_bytes(e.colptr) + vec_bytes(e.rowidx) + vec_bytes(e.custom);
  if (e.bytes > kSymCacheBytes / 2) return;
  e.sym = S;
  std::lock_guard<std::mutex> lock(g_sym_mu);
  g_sym_bytes += e.bytes;
  g_sym_cache.push_front(std::move(e));
  while (g_sym_bytes > kSymCacheBytes && !g_sym_cache.empty()) {
    g_sym_bytes -= g_sym_cache.back().bytes;
    g_sym_cache.pop_back();
  }
}

void release_symbolic_cache() {
  std::lock_guard<std::mutex> lock(g_sym_mu);
  g_sym_cache.clear();
  g_sym_bytes = 0;
}

}  // namespace inla
