// Nested-dissection ordering for the GPU engine.
//
// The supernodal kernels run one launch sequence per elimination-tree level,
// and the pivot columns along the longest root-to-leaf path are eliminated in
// sequence; both shrink when the top of the tree is a balanced hierarchy of
// separators instead of the long chain that minimum degree tends to produce on
// meshes. This is George's level-structure nested dissection (A. George,
// "Nested dissection of a regular finite element mesh", SIAM J. Numer. Anal.
// 10(2), 1973; A. George & J. W. H. Liu, "Computer Solution of Large Sparse
// Positive Definite Systems", Prentice-Hall 1981, ch. 8):
//   * graph of A + A^T without self loops, handled one connected part at a time;
//   * a pseudo-peripheral root by repeated breadth-first search (restart from a
//     minimum-degree node of the last level while the level count grows);
//   * the separator is one level L_i of a rooted level structure, thinned to
//     the nodes of L_i that have a neighbour in L_{i+1}; among the levels that
//     leave at least kBalance of the part on either side (the middle level when
//     none does) the one with the smallest thinned size is taken, comparing the
//     structures rooted at both ends of the pseudo-diameter;
//   * the two sides are ordered first (recursively), the separator last;
//   * parts of at most kLeaf nodes are ordered by approximate minimum degree on
//     their induced subgraph;
//   * the parts created by the first few splits are ordered on separate host
//     threads (the result does not depend on the thread count).
// The reference (faer) has no nested-dissection ordering: this is a GPU-side
// choice of the symbolic analysis; factors, solves and selected inverses
// agree with those under any other ordering up to rounding.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <thread>
#include <vector>

#include "symbolic.hpp"

namespace inla {

namespace {
constexpr int64_t kLeaf = 64;
constexpr double kBalance = 0.45;
constexpr int kParallelDepth = 3;        // parts of the first three splits are ordered on their own threads
constexpr int64_t kParallelMin = 4096;  // smallest part handed to a thread

// State shared by the threads: a part is a set of nodes stamped with a unique
// task id in `owner`; concurrent parts are disjoint, so dist/dstamp entries of a
// part are only touched by its thread, while owner stamps of neighbouring parts
// are read (atomically) to test membership.
// Node ids, levels, task ids and BFS stamps are 32-bit (half the memory traffic of the sweeps);
// nd_order rejects graphs with 2^31 or more nodes.
struct NdCtx {
  std::vector<int64_t> aptr;
  std::vector<int32_t> adj;
  std::vector<std::atomic<int32_t>> owner;
  std::vector<int32_t> dist, dstamp;
  std::atomic<int32_t> next_task{0}, bfs_id{0};

  explicit NdCtx(int64_t n) : owner(n), dist(n, -1), dstamp(n, -1) {
    for (auto& o : owner) o.store(-1, std::memory_order_relaxed);
  }
  int32_t own(int64_t v) const { return owner[v].load(std::memory_order_relaxed); }
  void stamp(int64_t v, int64_t t) { owner[v].store((int32_t)t, std::memory_order_relaxed); }

  // rooted level structure: nodes in BFS order, level l = nodes[start[l] .. start[l+1])
  struct Levels {
    std::vector<int64_t> nodes, start;
    int64_t depth() const { return (int64_t)start.size() - 1; }
    const int64_t* begin(int64_t l) const { return nodes.data() + start[l]; }
    const int64_t* end(int64_t l) const { return nodes.data() + start[l + 1]; }
  };
  void bfs(int64_t task, int64_t root, Levels& L) {
    const int64_t id = bfs_id++;
    L.nodes.clear();
    L.start.clear();
    L.nodes.push_back(root);
    L.start.push_back(0);
    dstamp[root] = id;
    dist[root] = 0;
    int64_t lev_begin = 0;
    while (lev_begin < (int64_t)L.nodes.size()) {
      const int64_t lev_end = (int64_t)L.nodes.size();
      const int64_t l = (int64_t)L.start.size() - 1;
      for (int64_t h = lev_begin; h < lev_end; ++h) {
        const int64_t u = L.nodes[h];
        for (int64_t q = aptr[u]; q < aptr[u + 1]; ++q) {
          const int64_t v = adj[q];
          if (own(v) != task || dstamp[v] == id) continue;
          dstamp[v] = id;
          dist[v] = l + 1;
          L.nodes.push_back(v);
        }
      }
      L.start.push_back(lev_end);
      lev_begin = lev_end;
    }
  }
  // dist[] of the nodes of a stored level structure (what bfs() from its root leaves there)
  void restore_dist(const Levels& L) {
    for (int64_t l = 0; l < L.depth(); ++l)
      for (const int64_t* it = L.begin(l); it != L.end(l); ++it) dist[*it] = l;
  }
  int64_t part_degree(int64_t task, int64_t u) const {
    int64_t d = 0;
    for (int64_t q = aptr[u]; q < aptr[u + 1]; ++q) d += own(adj[q]) == task;
    return d;
  }
  int64_t min_degree_last(int64_t task, const Levels& L) const {
    const int64_t l = L.depth() - 1;
    int64_t cand = *L.begin(l), cd = part_degree(task, cand);
    for (const int64_t* it = L.begin(l); it != L.end(l); ++it) {
      const int64_t d = part_degree(task, *it);
      if (d < cd) cand = *it, cd = d;
    }
    return cand;
  }
  // approximate minimum degree on the induced subgraph of a leaf part
  void emit_amd(const std::vector<int64_t>& nodes, std::vector<int64_t>& out) {
    if (nodes.size() <= 2) {
      out.insert(out.end(), nodes.begin(), nodes.end());
      return;
    }
    const int64_t m = (int64_t)nodes.size();
    const int64_t task = next_task++;
    for (int64_t i = 0; i < m; ++i) stamp(nodes[i], task), dist[nodes[i]] = i;
    std::vector<int64_t> cp(m + 1, 0), ri;
    for (int64_t i = 0; i < m; ++i) {
      const int64_t u = nodes[i];
      for (int64_t q = aptr[u]; q < aptr[u + 1]; ++q)
        if (own(adj[q]) == task) ri.push_back(dist[adj[q]]);
      cp[i + 1] = (int64_t)ri.size();
    }
    std::vector<int64_t> lp;
    amd_order(m, cp.data(), ri.data(), lp);
    for (int64_t k = 0; k < m; ++k) out.push_back(nodes[lp[k]]);
  }

  // One dissection step of a part with more than kLeaf nodes: either its
  // connected components (comps, more than one), or a separator and the rest
  // (sep non-empty), or neither (order the part as a leaf).
  struct Split {
    std::vector<std::vector<int64_t>> comps;
    std::vector<int64_t> sep, rest;
  };
  void split(const std::vector<int64_t>& nodes, Split& out) {
    out.comps.clear();
    out.sep.clear();
    out.rest.clear();
    const int64_t task = next_task++;
    for (int64_t u : nodes) stamp(u, task);
    {
      const int64_t id = bfs_id++;
      for (int64_t s0 : nodes) {
        if (dstamp[s0] == id) continue;
        std::vector<int64_t> comp{s0};
        dstamp[s0] = id;
        for (size_t h = 0; h < comp.size(); ++h) {
          const int64_t u = comp[h];
          for (int64_t q = aptr[u]; q < aptr[u + 1]; ++q) {
            const int64_t v = adj[q];
            if (own(v) == task && dstamp[v] != id) {
              dstamp[v] = id;
              comp.push_back(v);
            }
          }
        }
        out.comps.push_back(std::move(comp));
      }
      if (out.comps.size() > 1) return;
      out.comps.clear();
    }
    // pseudo-peripheral root
    Levels levels, best;
    bfs(task, *std::min_element(nodes.begin(), nodes.end()), levels);
    for (int it = 0; it < 3; ++it) {
      const int64_t cand = min_degree_last(task, levels);
      std::swap(levels, best);
      bfs(task, cand, levels);
      if (levels.depth() <= best.depth()) {
        std::swap(levels, best);
        break;
      }
    }
    // candidate level structures: from the pseudo-peripheral root and from a
    // minimum-degree node of its last level; in each, every level inside the
    // balance window is scored by its thinned size (nodes with a neighbour in
    // the next level), and the smallest thinned separator wins
    const int64_t N = (int64_t)nodes.size();
    int64_t best_size = -1;
    const int64_t roots[2] = {levels.nodes[0], min_degree_last(task, levels)};
    const int nroots = roots[1] != roots[0] ? 2 : 1;
    std::vector<int64_t> thin;
    for (int ri = 0; ri < nroots; ++ri) {
      // the structure rooted at roots[0] is `levels` itself, and the search above usually built
      // the one rooted at roots[1] already (`best`): a BFS depends only on the part and the root,
      // so stored structures are reused and only dist[] is rewritten
      if (ri == 0) {
        restore_dist(levels);
      } else if (!best.nodes.empty() && best.nodes[0] == roots[1]) {
        std::swap(levels, best);
        restore_dist(levels);
      } else {
        bfs(task, roots[ri], levels);
      }
      const int64_t h = levels.depth();
      if (h < 3) continue;
      // thinned size of level l (nodes with a neighbour in level l + 1), computed only for the
      // levels that are compared: those inside the balance window and the fallback level
      thin.assign(h, -1);
      auto thin_of = [&](int64_t l) {
        if (thin[l] < 0) {
          int64_t c = 0;
          for (const int64_t* it = levels.begin(l); it != levels.end(l); ++it) {
            const int64_t u = *it;
            bool touches = false;
            for (int64_t q = aptr[u]; q < aptr[u + 1] && !touches; ++q) {
              const int64_t v = adj[q];
              touches = own(v) == task && dist[v] == l + 1;
            }
            c += touches;
          }
          thin[l] = c;
        }
        return thin[l];
      };
      int64_t pick = -1;
      for (int64_t l = 1; l + 1 < h; ++l) {
        const int64_t below = levels.start[l], above = N - levels.start[l + 1];
        if ((double)std::min(below, above) >= kBalance * (double)N && (pick < 0 || thin_of(l) < thin_of(pick)))
          pick = l;
      }
      if (pick < 0) {
        pick = 1;
        while (pick + 2 < h && levels.start[pick + 1] < N / 2) ++pick;
      }
      if (best_size >= 0 && thin_of(pick) >= best_size) continue;
      best_size = thin_of(pick);
      out.sep.clear();
      out.rest.clear();
      for (const int64_t* it = levels.begin(pick); it != levels.end(pick); ++it) {
        const int64_t u = *it;
        bool touches = false;
        for (int64_t q = aptr[u]; q < aptr[u + 1] && !touches; ++q) {
          const int64_t v = adj[q];
          touches = own(v) == task && dist[v] == pick + 1;
        }
        (touches ? out.sep : out.rest).push_back(u);
      }
      for (int64_t l = 0; l < h; ++l)
        if (l != pick) out.rest.insert(out.rest.end(), levels.begin(l), levels.end(l));
    }
    if (out.rest.empty()) out.sep.clear();
    std::sort(out.sep.begin(), out.sep.end());
  }

  // Sequential dissection of one part: sides first, separators last.
  void order_seq(std::vector<int64_t> all, std::vector<int64_t>& out) {
    struct Work {
      std::vector<int64_t> nodes;
      bool emit;
    };
    std::vector<Work> stack;
    stack.push_back({std::move(all), false});
    Split sp;
    while (!stack.empty()) {
      Work wk = std::move(stack.back());
      stack.pop_back();
      if (wk.emit) {
        out.insert(out.end(), wk.nodes.begin(), wk.nodes.end());
        continue;
      }
      if ((int64_t)wk.nodes.size() <= kLeaf) {
        emit_amd(wk.nodes, out);
        continue;
      }
      split(wk.nodes, sp);
      if (!sp.comps.empty()) {
        for (size_t c = sp.comps.size(); c-- > 0;) stack.push_back({std::move(sp.comps[c]), false});
      } else if (!sp.sep.empty()) {
        stack.push_back({std::move(sp.sep), true});
        stack.push_back({std::move(sp.rest), false});
      } else {
        emit_amd(wk.nodes, out);
      }
    }
  }

  // The first kParallelDepth splits fan the parts out to threads; each part's
  // ordering is written to its own vector and concatenated in sequential order.
  void order_par(std::vector<int64_t> nodes, std::vector<int64_t>& out, int depth) {
    if (depth >= kParallelDepth || (int64_t)nodes.size() < kParallelMin) {
      order_seq(std::move(nodes), out);
      return;
    }
    Split sp;
    split(nodes, sp);
    if (!sp.comps.empty()) {
      std::vector<std::vector<int64_t>> outs(sp.comps.size());
      std::vector<std::thread> th;
      for (size_t c = 0; c < sp.comps.size(); ++c) {
        if ((int64_t)sp.comps[c].size() >= kParallelMin)
          th.emplace_back([this, &sp, &outs, c, depth] { order_par(std::move(sp.comps[c]), outs[c], depth + 1); });
        else
          order_seq(std::move(sp.comps[c]), outs[c]);
      }
      for (auto& t : th) t.join();
      for (auto& o : outs) out.insert(out.end(), o.begin(), o.end());
    } else if (!sp.sep.empty()) {
      order_par(std::move(sp.rest), out, depth);  // the sides are the components of the rest
      out.insert(out.end(), sp.sep.begin(), sp.sep.end());
    } else {
      emit_amd(nodes, out);
    }
  }
};
}  // namespace

void nd_order(int64_t n, const int64_t* colptr, const int64_t* rowidx, std::vector<int64_t>& perm) {
  NdCtx cx(n);
  // symmetric adjacency (CSR), no self loops, duplicates removed
  std::vector<int64_t> deg(n, 0);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      const int64_t r = rowidx[p];
      if (r == c) continue;
      ++deg[r];
      ++deg[c];
    }
  if (n >= (int64_t)INT32_MAX) throw std::runtime_error("nested dissection: graph too large");
  std::vector<int64_t>& aptr = cx.aptr;
  std::vector<int32_t>& adj = cx.adj;
  aptr.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) aptr[i + 1] = aptr[i] + deg[i];
  adj.assign(aptr[n], 0);
  std::vector<int64_t> fill(aptr.begin(), aptr.end() - 1);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      const int64_t r = rowidx[p];
      if (r == c) continue;
      adj[fill[r]++] = (int32_t)c;
      adj[fill[c]++] = (int32_t)r;
    }
  {
    std::vector<int64_t> nptr(n + 1, 0);
    int64_t w = 0;
    for (int64_t i = 0; i < n; ++i) {
      int32_t* b = adj.data() + aptr[i];
      int32_t* e = adj.data() + aptr[i + 1];
      std::sort(b, e);
      e = std::unique(b, e);
      nptr[i] = w;
      for (int32_t* q = b; q < e; ++q) adj[w++] = *q;
    }
    nptr[n] = w;
    adj.resize(w);
    aptr.swap(nptr);
  }
  perm.clear();
  perm.reserve(n);
  std::vector<int64_t> all(n);
  for (int64_t i = 0; i < n; ++i) all[i] = i;
  cx.order_par(std::move(all), perm, 0);
  if ((int64_t)perm.size() != n) throw std::runtime_error("nested dissection: ordering incomplete");
}

}  // namespace inla
