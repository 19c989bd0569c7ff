// Approximate minimum degree ordering on the quotient graph.
//
// The reference calls faer's AMD (crates/inla_math/src/sparse_ldlt.rs:165-170,
// SymmetricOrdering::Amd; faer 0.24 is not vendored). This is an independent
// implementation of the published algorithm (Amestoy, Davis & Duff, "An
// approximate minimum degree ordering algorithm", SIAM J. Matrix Anal. Appl.
// 17(4), 1996): quotient graph with element absorption, approximate external
// degrees d_i = min(n-k, d_i + |Lp\i|, |A_i| + |Lp\i| + sum_e |Le\Lp|),
// aggressive absorption, mass elimination and hash-based supervariable
// detection. Tie-breaking differs from faer, so the permutation is not
// bit-identical to the reference's; fill quality is comparable.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

#include "symbolic.hpp"

namespace inla {

namespace {

struct DegreeLists {
  std::vector<int64_t> head, next, prev, deg;
  int64_t mindeg = 0;
  explicit DegreeLists(int64_t n) : head(n + 1, -1), next(n, -1), prev(n, -1), deg(n, 0) {}
  void insert(int64_t i, int64_t d) {
    deg[i] = d;
    next[i] = head[d];
    prev[i] = -1;
    if (head[d] != -1) prev[head[d]] = i;
    head[d] = i;
    if (d < mindeg) mindeg = d;
  }
  void remove(int64_t i) {
    int64_t d = deg[i];
    if (prev[i] != -1) next[prev[i]] = next[i];
    else head[d] = next[i];
    if (next[i] != -1) prev[next[i]] = prev[i];
    next[i] = prev[i] = -1;
  }
};

}  // namespace

void amd_order(int64_t n, const int64_t* colptr, const int64_t* rowidx, std::vector<int64_t>& perm) {
  perm.clear();
  perm.reserve(n);
  // status: 0 = variable, 1 = element (alive), 2 = dead (absorbed element or
  // non-principal variable)
  std::vector<char> status(n, 0);
  std::vector<std::vector<int32_t>> E(n), A(n), L(n), members(n);
  std::vector<int64_t> nv(n, 1), esize(n, 0);
  for (int64_t c = 0; c < n; ++c)
    for (int64_t p = colptr[c]; p < colptr[c + 1]; ++p) {
      int64_t r = rowidx[p];
      if (r == c) continue;
      A[c].push_back((int32_t)r);
      A[r].push_back((int32_t)c);
    }
  DegreeLists dl(n);
  dl.mindeg = n;
  for (int64_t i = 0; i < n; ++i) {
    auto& a = A[i];
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
    members[i].push_back((int32_t)i);
    dl.insert(i, (int64_t)a.size());
  }

  std::vector<int64_t> wmark(n, -1), wval(n, 0), inlp(n, -1);
  int64_t nel = 0;
  int64_t step = 0;
  std::vector<int32_t> Lp;
  std::vector<std::pair<uint64_t, int32_t>> hashes;

  while (nel < n) {
    // ---- pick the minimum-degree principal variable --------------------------
    while (dl.mindeg <= n && dl.head[dl.mindeg] == -1) ++dl.mindeg;
    if (dl.mindeg > n) break;  // cannot happen for a consistent graph
    int64_t p = dl.head[dl.mindeg];
    dl.remove(p);
    ++step;

    // ---- form the new element Lp -----------------------------------------------
    Lp.clear();
    inlp[p] = step;
    for (int32_t e : E[p]) {
      if (status[e] != 1) continue;
      for (int32_t i : L[e])
        if (status[i] == 0 && nv[i] > 0 && inlp[i] != step) {
          inlp[i] = step;
          Lp.push_back(i);
        }
      status[e] = 2;  // absorbed into p
      L[e].clear();
      L[e].shrink_to_fit();
    }
    for (int32_t i : A[p])
      if (status[i] == 0 && nv[i] > 0 && inlp[i] != step) {
        inlp[i] = step;
        Lp.push_back(i);
      }
    E[p].clear();
    A[p].clear();
    E[p].shrink_to_fit();
    A[p].shrink_to_fit();
    status[p] = 1;
    for (int32_t m : members[p]) perm.push_back(m);
    nel += nv[p];

    // ---- prune the lists of every variable in Lp -------------------------------
    for (int32_t i : Lp) {
      dl.remove(i);
      auto& Ei = E[i];
      size_t w = 0;
      for (int32_t e : Ei)
        if (status[e] == 1 && e != p) Ei[w++] = e;
      Ei.resize(w);
      Ei.push_back((int32_t)p);
      auto& Ai = A[i];
      w = 0;
      for (int32_t j : Ai)
        if (status[j] == 0 && nv[j] > 0 && inlp[j] != step && j != p) Ai[w++] = j;
      Ai.resize(w);
    }

    // ---- |Le \ Lp| for the other elements touching Lp ------------------------
    for (int32_t i : Lp)
      for (int32_t e : E[i]) {
        if (e == p) continue;
        if (wmark[e] != step) {
          wmark[e] = step;
          wval[e] = esize[e];
        }
        wval[e] -= nv[i];
      }

    // ---- aggressive absorption, mass elimination -------------------------------
    int64_t lp_size = 0;
    for (int32_t i : Lp) lp_size += nv[i];
    for (int32_t i : Lp)
      for (int32_t e : E[i])
        if (e != p && status[e] == 1 && wmark[e] == step && wval[e] <= 0) {
          status[e] = 2;  // Le ⊆ Lp: absorb into p
          L[e].clear();
        }
    std::vector<int32_t> keep;
    keep.reserve(Lp.size());
    for (int32_t i : Lp) {
      auto& Ei = E[i];
      size_t w = 0;
      for (int32_t e : Ei)
        if (status[e] == 1) Ei[w++] = e;
      Ei.resize(w);
      if (Ei.size() == 1 && A[i].empty()) {
        // adjacent only to the new element: eliminate together with p
        for (int32_t m : members[i]) perm.push_back(m);
        nel += nv[i];
        lp_size -= nv[i];
        nv[i] = 0;
        status[i] = 2;
        E[i].clear();
        continue;
      }
      keep.push_back(i);
    }
    Lp.swap(keep);

    // ---- supervariable detection -------------------------------------------------
    hashes.clear();
    for (int32_t i : Lp) {
      uint64_t h = 0;
      for (int32_t e : E[i]) h += (uint64_t)e * 2654435761ULL + 1;
      for (int32_t j : A[i]) h += (uint64_t)j * 40503ULL + 7;
      hashes.push_back({h ^ ((uint64_t)E[i].size() << 48) ^ ((uint64_t)A[i].size() << 32), i});
    }
    std::sort(hashes.begin(), hashes.end());
    for (size_t a = 0; a < hashes.size();) {
      size_t b = a;
      while (b < hashes.size() && hashes[b].first == hashes[a].first) ++b;
      if (b - a > 1) {
        for (size_t x = a; x < b; ++x) {
          int32_t i = hashes[x].second;
          if (nv[i] == 0) continue;
          std::vector<int32_t> ei = E[i], ai = A[i];
          std::sort(ei.begin(), ei.end());
          std::sort(ai.begin(), ai.end());
          for (size_t y = x + 1; y < b; ++y) {
            int32_t j = hashes[y].second;
            if (nv[j] == 0) continue;
            if (E[j].size() != ei.size() || A[j].size() != ai.size()) continue;
            std::vector<int32_t> ej = E[j], aj = A[j];
            std::sort(ej.begin(), ej.end());
            std::sort(aj.begin(), aj.end());
            if (ej != ei || aj != ai) continue;
            // j is indistinguishable from i: merge
            nv[i] += nv[j];
            nv[j] = 0;
            status[j] = 2;
            members[i].insert(members[i].end(), members[j].begin(), members[j].end());
            members[j].clear();
            E[j].clear();
            A[j].clear();
          }
        }
      }
      a = b;
    }
    {
      size_t w = 0;
      for (int32_t i : Lp)
        if (nv[i] > 0) Lp[w++] = i;
      Lp.resize(w);
    }
    L[p].assign(Lp.begin(), Lp.end());
    esize[p] = lp_size;

    // ---- approximate degrees -----------------------------------------------------
    for (int32_t i : Lp) {
      int64_t ext = 0;
      for (int32_t e : E[i])
        if (e != p && wmark[e] == step) ext += std::max<int64_t>(wval[e], 0);
        else if (e != p) ext += esize[e];
      int64_t adeg = 0;
      for (int32_t j : A[i]) adeg += nv[j];
      int64_t lpi = lp_size - nv[i];
      int64_t d = adeg + lpi + ext;
      d = std::min<int64_t>(d, dl.deg[i] + lpi);
      d = std::min<int64_t>(d, n - nel - nv[i]);
      if (d < 0) d = 0;
      dl.insert(i, d);
    }
  }
}

}  // namespace inla
