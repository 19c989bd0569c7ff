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
//     their induced subgraph.
// The reference (faer) has no nested-dissection ordering: this is a GPU-side
// choice of the symbolic analysis; factors, solves and selected inverses
// agree with those under any other ordering up to rounding.
#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "symbolic.hpp"

namespace inla {

namespace {
constexpr int64_t kLeaf = 64;
constexpr double kBalance = 0.45;
}  // namespace

void nd_order(int64_t n, const int64_t* colptr, const int64_t* rowidx, std::vector<int64_t>& perm) {
  // symmetric adjacency (CSR), no self loops, duplicates removed
  std::vector<int64_t> deg(n, 0);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      const int64_t r = rowidx[p];
      if (r == c) continue;
      ++deg[r];
      ++deg[c];
    }
  std::vector<int64_t> aptr(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) aptr[i + 1] = aptr[i] + deg[i];
  std::vector<int64_t> adj(aptr[n]), fill(aptr.begin(), aptr.end() - 1);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      const int64_t r = rowidx[p];
      if (r == c) continue;
      adj[fill[r]++] = c;
      adj[fill[c]++] = r;
    }
  {
    std::vector<int64_t> nptr(n + 1, 0);
    int64_t w = 0;
    for (int64_t i = 0; i < n; ++i) {
      int64_t* b = adj.data() + aptr[i];
      int64_t* e = adj.data() + aptr[i + 1];
      std::sort(b, e);
      e = std::unique(b, e);
      nptr[i] = w;
      for (int64_t* q = b; q < e; ++q) adj[w++] = *q;
    }
    nptr[n] = w;
    adj.resize(w);
    aptr.swap(nptr);
  }

  perm.clear();
  perm.reserve(n);
  std::vector<int64_t> owner(n, -1);  // task stamp of the part a node currently belongs to
  std::vector<int64_t> dist(n, -1), dstamp(n, -1);
  int64_t next_task = 0, bfs_id = 0;

  // rooted level structure of the part `task` from `root`: nodes in BFS order,
  // level l = nodes[start[l] .. start[l+1]); dist[] holds the levels of this BFS
  struct Levels {
    std::vector<int64_t> nodes, start;
    int64_t depth() const { return (int64_t)start.size() - 1; }
    const int64_t* begin(int64_t l) const { return nodes.data() + start[l]; }
    const int64_t* end(int64_t l) const { return nodes.data() + start[l + 1]; }
    int64_t size(int64_t l) const { return start[l + 1] - start[l]; }
  };
  auto bfs = [&](int64_t task, int64_t root, Levels& L) {
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
          if (owner[v] != task || dstamp[v] == id) continue;
          dstamp[v] = id;
          dist[v] = l + 1;
          L.nodes.push_back(v);
        }
      }
      L.start.push_back(lev_end);
      lev_begin = lev_end;
    }
    // start has depth + 1 entries: the last one closes the deepest level
  };
  auto part_degree = [&](int64_t task, int64_t u) {
    int64_t d = 0;
    for (int64_t q = aptr[u]; q < aptr[u + 1]; ++q) d += owner[adj[q]] == task;
    return d;
  };
  auto emit_amd = [&](const std::vector<int64_t>& nodes) {
    if (nodes.size() <= 2) {
      for (int64_t u : nodes) perm.push_back(u);
      return;
    }
    const int64_t m = (int64_t)nodes.size();
    const int64_t task = next_task++;
    for (int64_t i = 0; i < m; ++i) owner[nodes[i]] = task, dist[nodes[i]] = i;
    std::vector<int64_t> cp(m + 1, 0), ri;
    for (int64_t i = 0; i < m; ++i) {
      const int64_t u = nodes[i];
      for (int64_t q = aptr[u]; q < aptr[u + 1]; ++q)
        if (owner[adj[q]] == task) ri.push_back(dist[adj[q]]);
      cp[i + 1] = (int64_t)ri.size();
    }
    std::vector<int64_t> lp;
    amd_order(m, cp.data(), ri.data(), lp);
    for (int64_t k = 0; k < m; ++k) perm.push_back(nodes[lp[k]]);
  };

  // work stack: a part to dissect, or a separator to emit (after both sides)
  struct Work {
    std::vector<int64_t> nodes;
    bool emit;
  };
  std::vector<Work> stack;
  {
    std::vector<int64_t> all(n);
    for (int64_t i = 0; i < n; ++i) all[i] = i;
    stack.push_back({std::move(all), false});
  }
  Levels levels, best_levels;
  while (!stack.empty()) {
    Work wk = std::move(stack.back());
    stack.pop_back();
    if (wk.emit) {
      for (int64_t u : wk.nodes) perm.push_back(u);
      continue;
    }
    std::vector<int64_t>& nodes = wk.nodes;
    if ((int64_t)nodes.size() <= kLeaf) {
      emit_amd(nodes);
      continue;
    }
    const int64_t task = next_task++;
    for (int64_t u : nodes) owner[u] = task;
    // connected components: dissect each separately (pushed in reverse so that
    // the first component is ordered first)
    {
      std::vector<std::vector<int64_t>> comps;
      const int64_t id = bfs_id++;
      for (int64_t s0 : nodes) {
        if (dstamp[s0] == id) continue;
        std::vector<int64_t> comp{s0};
        dstamp[s0] = id;
        for (size_t h = 0; h < comp.size(); ++h) {
          const int64_t u = comp[h];
          for (int64_t q = aptr[u]; q < aptr[u + 1]; ++q) {
            const int64_t v = adj[q];
            if (owner[v] == task && dstamp[v] != id) {
              dstamp[v] = id;
              comp.push_back(v);
            }
          }
        }
        comps.push_back(std::move(comp));
      }
      if (comps.size() > 1) {
        for (size_t c = comps.size(); c-- > 0;) stack.push_back({std::move(comps[c]), false});
        continue;
      }
    }
    // pseudo-peripheral root
    auto min_degree_last = [&](const Levels& L) {
      const int64_t l = L.depth() - 1;
      int64_t cand = *L.begin(l), cd = part_degree(task, cand);
      for (const int64_t* it = L.begin(l); it != L.end(l); ++it) {
        const int64_t d = part_degree(task, *it);
        if (d < cd) cand = *it, cd = d;
      }
      return cand;
    };
    bfs(task, *std::min_element(nodes.begin(), nodes.end()), levels);
    for (int it = 0; it < 3; ++it) {
      const int64_t cand = min_degree_last(levels);
      std::swap(levels, best_levels);
      bfs(task, cand, levels);
      if (levels.depth() <= best_levels.depth()) {
        std::swap(levels, best_levels);
        break;
      }
    }
    // candidate level structures: from the pseudo-peripheral root and from a
    // minimum-degree node of its last level; in each, every level inside the
    // balance window is scored by its thinned size (nodes with a neighbour in
    // the next level), and the smallest thinned separator wins
    const int64_t N = (int64_t)nodes.size();
    std::vector<int64_t> sep, rest;
    int64_t best_size = -1;
    int64_t roots[2] = {levels.nodes[0], min_degree_last(levels)};
    const int nroots = roots[1] != roots[0] ? 2 : 1;
    std::vector<int64_t> thin;
    for (int ri = 0; ri < nroots; ++ri) {
      bfs(task, roots[ri], levels);
      const int64_t h = levels.depth();
      if (h < 3) continue;
      thin.assign(h, 0);
      for (int64_t l = 0; l + 1 < h; ++l)
        for (const int64_t* it = levels.begin(l); it != levels.end(l); ++it) {
          const int64_t u = *it;
          bool touches = false;
          for (int64_t q = aptr[u]; q < aptr[u + 1] && !touches; ++q) {
            const int64_t v = adj[q];
            touches = owner[v] == task && dist[v] == l + 1;
          }
          thin[l] += touches;
        }
      int64_t pick = -1;
      for (int64_t l = 1; l + 1 < h; ++l) {
        const int64_t below = levels.start[l], above = N - levels.start[l + 1];
        if ((double)std::min(below, above) >= kBalance * (double)N && (pick < 0 || thin[l] < thin[pick])) pick = l;
      }
      if (pick < 0) {
        pick = 1;
        while (pick + 2 < h && levels.start[pick + 1] < N / 2) ++pick;
      }
      if (best_size >= 0 && thin[pick] >= best_size) continue;
      best_size = thin[pick];
      sep.clear();
      rest.clear();
      for (const int64_t* it = levels.begin(pick); it != levels.end(pick); ++it) {
        const int64_t u = *it;
        bool touches = false;
        for (int64_t q = aptr[u]; q < aptr[u + 1] && !touches; ++q) {
          const int64_t v = adj[q];
          touches = owner[v] == task && dist[v] == pick + 1;
        }
        (touches ? sep : rest).push_back(u);
      }
      for (int64_t l = 0; l < h; ++l)
        if (l != pick) rest.insert(rest.end(), levels.begin(l), levels.end(l));
    }
    if (sep.empty() || rest.empty()) {
      emit_amd(nodes);
      continue;
    }
    std::sort(sep.begin(), sep.end());
    stack.push_back({std::move(sep), true});
    stack.push_back({std::move(rest), false});
  }
  if ((int64_t)perm.size() != n) throw std::runtime_error("nested dissection: ordering incomplete");
}

}  // namespace inla
