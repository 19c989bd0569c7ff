#include "mesh.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <numeric>
#include <tuple>

namespace inla {

namespace {

inline double signed_area2(double ax, double ay, double bx, double by, double cx, double cy) {
  return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

// Triplets summed per (row, col) in insertion order after a stable sort by (row, col), as
// SparseTriplet::coalesce does, then laid out column-major.
CscBlock coalesce(int64_t n, std::vector<std::tuple<int64_t, int64_t, double>>& t) {
  std::stable_sort(t.begin(), t.end(), [](const auto& a, const auto& b) {
    return std::get<0>(a) != std::get<0>(b) ? std::get<0>(a) < std::get<0>(b) : std::get<1>(a) < std::get<1>(b);
  });
  std::vector<std::tuple<int64_t, int64_t, double>> merged;
  merged.reserve(t.size());
  for (const auto& e : t) {
    if (!merged.empty() && std::get<0>(merged.back()) == std::get<0>(e) && std::get<1>(merged.back()) == std::get<1>(e))
      std::get<2>(merged.back()) += std::get<2>(e);
    else
      merged.push_back(e);
  }
  CscBlock b;
  b.n = n;
  b.colptr.assign(n + 1, 0);
  for (const auto& e : merged) ++b.colptr[std::get<1>(e) + 1];
  for (int64_t j = 0; j < n; ++j) b.colptr[j + 1] += b.colptr[j];
  b.rowidx.resize(merged.size());
  b.val.resize(merged.size());
  std::vector<int64_t> next(b.colptr.begin(), b.colptr.end() - 1);
  for (const auto& e : merged) {  // rows arrive ascending, so each column stays sorted
    const int64_t q = next[std::get<1>(e)]++;
    b.rowidx[q] = std::get<0>(e);
    b.val[q] = std::get<2>(e);
  }
  return b;
}

}  // namespace

std::string build_mesh2d(int64_t nv, const double* xy, int64_t ntri, const int64_t* tri, Mesh2D& m) {
  if (nv < 3) return "need at least three vertices";
  m = Mesh2D();
  m.x.resize(nv);
  m.y.resize(nv);
  for (int64_t i = 0; i < nv; ++i) {
    m.x[i] = xy[2 * i];
    m.y[i] = xy[2 * i + 1];
  }
  m.tri.resize(ntri);
  for (int64_t t = 0; t < ntri; ++t) {
    const int64_t a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv)
      return "triangle " + std::to_string(t) + " has vertex out of range: [" + std::to_string(a) + ", " +
             std::to_string(b) + ", " + std::to_string(c) + "] with " + std::to_string(nv) + " vertices";
    if (a == b || b == c || a == c) return "triangle " + std::to_string(t) + " is degenerate (duplicate indices)";
    if (std::fabs(signed_area2(m.x[a], m.y[a], m.x[b], m.y[b], m.x[c], m.y[c])) <= kGeomEps)
      return "triangle " + std::to_string(t) + " has near-zero area";
    m.tri[t] = {a, b, c};
  }
  // directed edge (a, b) of edge e of triangle t is (tri[e+1], tri[e+2]); a triangle that has
  // (b, a) is the neighbour; a second (a, b) is a non-manifold edge
  m.nbr.assign(ntri, {-1, -1, -1});
  std::map<std::pair<int64_t, int64_t>, std::pair<int64_t, int>> open;
  for (int64_t t = 0; t < ntri; ++t)
    for (int e = 0; e < 3; ++e) {
      const int64_t a = m.tri[t][(e + 1) % 3], b = m.tri[t][(e + 2) % 3];
      auto it = open.find({b, a});
      if (it != open.end()) {
        m.nbr[t][e] = it->second.first;
        m.nbr[it->second.first][it->second.second] = t;
        open.erase(it);
      } else if (!open.emplace(std::make_pair(a, b), std::make_pair(t, e)).second) {
        return "non-manifold edge detected between vertices " + std::to_string(a) + " and " + std::to_string(b);
      }
    }
  return std::string();
}

std::string assemble_fem(const Mesh2D& m, const std::vector<double>& triangle_scale, double hxx, double hxy,
                         double hyy, FemBlocks& out) {
  const int64_t ntri = (int64_t)m.tri.size(), nv = (int64_t)m.x.size();
  if (!triangle_scale.empty() && (int64_t)triangle_scale.size() != ntri)
    return "diffusion scale length " + std::to_string(triangle_scale.size()) + " != n_triangles " +
           std::to_string(ntri);
  if (!std::isfinite(hxx) || !std::isfinite(hxy) || !std::isfinite(hyy))
    return "diffusion tensor entries must be finite";
  const double det = hxx * hyy - hxy * hxy;
  if (det <= 0.0) return "diffusion tensor must be SPD";
  std::vector<std::tuple<int64_t, int64_t, double>> c0, c1, g1, b1;
  c0.reserve(3 * ntri);
  c1.reserve(9 * ntri);
  g1.reserve(9 * ntri);
  out.area.resize(ntri);
  for (int64_t t = 0; t < ntri; ++t) {
    const auto& tv = m.tri[t];
    const double s0x = m.x[tv[0]], s0y = m.y[tv[0]], s1x = m.x[tv[1]], s1y = m.y[tv[1]], s2x = m.x[tv[2]],
                 s2y = m.y[tv[2]];
    // edge vectors e_i opposite vertex i: e0 = s2 - s1, e1 = s0 - s2, e2 = s1 - s0
    const double ex[3] = {s2x - s1x, s0x - s2x, s1x - s0x}, ey[3] = {s2y - s1y, s0y - s2y, s1y - s0y};
    const double area = 0.5 * std::fabs(signed_area2(s0x, s0y, s1x, s1y, s2x, s2y));
    out.area[t] = area;
    double fa = 0.5 * std::fabs(ex[0] * ey[1] - ey[0] * ex[1]);
    if (fa <= kGeomEps) fa = area;
    const double scale = triangle_scale.empty() ? 1.0 : triangle_scale[t];
    // eij = (H g_i) . g_j with g = e rotated by -90 degrees: (e.y, -e.x)
    double eij[3][3];
    for (int i = 0; i < 3; ++i) {
      const double gix = ey[i], giy = -ex[i];
      for (int j = i; j < 3; ++j) {
        const double gjx = ey[j], gjy = -ex[j];
        const double hx = hxx * gix + hxy * giy, hy = hxy * gix + hyy * giy;
        eij[i][j] = hx * gjx + hy * gjy;
        eij[j][i] = eij[i][j];
      }
    }
    for (int i = 0; i < 3; ++i) {
      c0.emplace_back(tv[i], tv[i], area / 3.0);
      c1.emplace_back(tv[i], tv[i], area / 6.0);
      g1.emplace_back(tv[i], tv[i], scale * eij[i][i] / (4.0 * fa));
      for (int j = i + 1; j < 3; ++j) {
        c1.emplace_back(tv[i], tv[j], area / 12.0);
        c1.emplace_back(tv[j], tv[i], area / 12.0);
        const double vij = scale * eij[i][j] / (4.0 * fa);
        g1.emplace_back(tv[i], tv[j], vij);
        g1.emplace_back(tv[j], tv[i], vij);
      }
    }
    const bool bnd[3] = {m.nbr[t][0] < 0, m.nbr[t][1] < 0, m.nbr[t][2] < 0};
    if (bnd[0] || bnd[1] || bnd[2]) {
      const double vij = -1.0 / (4.0 * fa);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k)
            if (bnd[k] && i != k) b1.emplace_back(tv[i], tv[j], scale * eij[k][j] * vij);
    }
  }
  out.c0 = coalesce(nv, c0);
  out.c1 = coalesce(nv, c1);
  out.g1 = coalesce(nv, g1);
  out.b1 = coalesce(nv, b1);
  return std::string();
}

int64_t locate_point(const Mesh2D& m, int64_t start, double px, double py, double bary[3]) {
  const int64_t ntri = (int64_t)m.tri.size();
  if (ntri == 0 || start < 0 || start >= ntri) return -1;
  int64_t cur = start;
  for (int64_t remaining = std::max<int64_t>(ntri * 3, 1); remaining > 0; --remaining) {
    const auto& tv = m.tri[cur];
    const double ax = m.x[tv[0]], ay = m.y[tv[0]], bx = m.x[tv[1]], by = m.y[tv[1]], cx = m.x[tv[2]],
                 cy = m.y[tv[2]];
    const double orient = signed_area2(ax, ay, bx, by, cx, cy) >= 0.0 ? 1.0 : -1.0;
    double most_negative = 0.0;
    int leaving = -1;
    for (int e = 0; e < 3; ++e) {
      const int64_t va = tv[(e + 1) % 3], vb = tv[(e + 2) % 3];
      const double side = orient * signed_area2(m.x[va], m.y[va], m.x[vb], m.y[vb], px, py);
      if (side < most_negative) {
        most_negative = side;
        leaving = e;
      }
    }
    if (most_negative >= -kGeomEps) {
      const double den = signed_area2(ax, ay, bx, by, cx, cy);
      if (std::fabs(den) <= kGeomEps) {
        bary[0] = bary[1] = bary[2] = NAN;
      } else {
        bary[0] = signed_area2(bx, by, cx, cy, px, py) / den;
        bary[1] = signed_area2(cx, cy, ax, ay, px, py) / den;
        bary[2] = 1.0 - bary[0] - bary[1];
      }
      return cur;
    }
    if (leaving < 0 || m.nbr[cur][leaving] < 0) return -1;
    cur = m.nbr[cur][leaving];
  }
  return -1;
}

std::string projector(const Mesh2D& m, int64_t npts, const double* xy, std::vector<int64_t>& rowptr,
                      std::vector<int64_t>& colidx, std::vector<double>& val) {
  rowptr.assign(npts + 1, 0);
  colidx.clear();
  val.clear();
  colidx.reserve(3 * npts);
  val.reserve(3 * npts);
  int64_t start = 0;
  for (int64_t r = 0; r < npts; ++r) {
    double w[3];
    const int64_t t = locate_point(m, start, xy[2 * r], xy[2 * r + 1], w);
    if (t < 0) {
      char buf[128];
      std::snprintf(buf, sizeof(buf), "observation point (%.17g, %.17g) is outside the mesh", xy[2 * r],
                    xy[2 * r + 1]);
      return buf;
    }
    start = t;
    std::array<std::pair<int64_t, double>, 3> e;
    int ne = 0;
    for (int k = 0; k < 3; ++k)
      if (std::fabs(w[k]) > kGeomEps) e[ne++] = {m.tri[t][k], w[k]};
    std::sort(e.begin(), e.begin() + ne);
    for (int k = 0; k < ne; ++k) {
      colidx.push_back(e[k].first);
      val.push_back(e[k].second);
    }
    rowptr[r + 1] = (int64_t)colidx.size();
  }
  return std::string();
}

std::string check_mesh1d(int64_t n, const double* loc) {
  if (n < 2) return "1D mesh requires at least two knots";
  for (int64_t i = 0; i < n; ++i) {
    if (!std::isfinite(loc[i])) return "1D mesh knot " + std::to_string(i) + " is not finite";
    if (i > 0 && loc[i] <= loc[i - 1]) return "1D mesh knots must be strictly increasing";
  }
  return std::string();
}

void assemble_fem1d(int64_t n, const double* loc, FemBlocks& out) {
  std::vector<std::tuple<int64_t, int64_t, double>> c0, c1, g1, b1;
  out.area.clear();
  for (int64_t i = 0; i + 1 < n; ++i) {
    const double h = loc[i + 1] - loc[i];
    out.area.push_back(h);
    c0.emplace_back(i, i, h / 2.0);
    c0.emplace_back(i + 1, i + 1, h / 2.0);
    c1.emplace_back(i, i, h / 3.0);
    c1.emplace_back(i + 1, i + 1, h / 3.0);
    c1.emplace_back(i, i + 1, h / 6.0);
    c1.emplace_back(i + 1, i, h / 6.0);
    const double inv_h = 1.0 / h;
    g1.emplace_back(i, i, inv_h);
    g1.emplace_back(i + 1, i + 1, inv_h);
    g1.emplace_back(i, i + 1, -inv_h);
    g1.emplace_back(i + 1, i, -inv_h);
  }
  out.c0 = coalesce(n, c0);
  out.c1 = coalesce(n, c1);
  out.g1 = coalesce(n, g1);
  out.b1 = coalesce(n, b1);
}

std::string projector1d(int64_t n, const double* loc, int64_t npts, const double* s, std::vector<int64_t>& rowptr,
                        std::vector<int64_t>& colidx, std::vector<double>& val) {
  rowptr.assign(npts + 1, 0);
  colidx.clear();
  val.clear();
  for (int64_t r = 0; r < npts; ++r) {
    const double x = s[r];
    if (!std::isfinite(x)) return "1D observation location " + std::to_string(r) + " is not finite";
    int64_t i;
    double w;
    if (x <= loc[0]) {
      i = 0;
      w = 0.0;
    } else if (x >= loc[n - 1]) {
      i = n - 2;
      w = 1.0;
    } else {  // bisection for loc[lo] <= x < loc[lo + 1]
      int64_t lo = 0, hi = n - 1;
      while (lo + 1 < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (loc[mid] <= x) lo = mid;
        else hi = mid;
      }
      i = lo;
      w = (x - loc[lo]) / (loc[lo + 1] - loc[lo]);
    }
    if (std::fabs(w) <= kGeomEps) {
      colidx.push_back(i);
      val.push_back(1.0);
    } else if (std::fabs(w - 1.0) <= kGeomEps) {
      colidx.push_back(i + 1);
      val.push_back(1.0);
    } else {
      colidx.push_back(i);
      val.push_back(1.0 - w);
      colidx.push_back(i + 1);
      val.push_back(w);
    }
    rowptr[r + 1] = (int64_t)colidx.size();
  }
  return std::string();
}

std::string spde_components(int64_t n, const double* c0, const int64_t* gcp, const int64_t* gri, const double* gv,
                            CscBlock& pat, std::vector<double>& comp) {
  if (n <= 0) return "SPDE requires non-empty FEM blocks";
  std::vector<double> cinv(n);
  for (int64_t i = 0; i < n; ++i) {
    if (std::fabs(c0[i]) < 1e-15) return "Zero entry in mass matrix c0 diagonal";
    cinv[i] = 1.0 / c0[i];
  }
  pat = CscBlock();
  pat.n = n;
  pat.colptr.assign(n + 1, 0);
  std::vector<double> vc, vg, vgcg;            // the three components, aligned with pat.rowidx
  std::vector<double> acc(n, 0.0), gcol(n, 0.0);
  std::vector<char> mark(n, 0);
  std::vector<int64_t> rows;
  std::vector<std::pair<int64_t, double>> kcol;
  for (int64_t j = 0; j < n; ++j) {
    rows.clear();
    auto touch = [&](int64_t i) {
      if (!mark[i]) {
        mark[i] = 1;
        rows.push_back(i);
      }
    };
    touch(j);
    kcol.clear();
    for (int64_t p = gcp[j]; p < gcp[j + 1]; ++p) {
      touch(gri[p]);
      gcol[gri[p]] += gv[p];
      kcol.push_back({gri[p], gv[p]});
    }
    std::stable_sort(kcol.begin(), kcol.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    // column j of G1 C0^-1 G1: for each G1_kj (k ascending) add (G1_ik cinv_k) G1_kj, with G1_ik
    // read from column k (G1 is symmetric)
    for (const auto& kv : kcol) {
      const int64_t k = kv.first;
      for (int64_t p = gcp[k]; p < gcp[k + 1]; ++p) {
        touch(gri[p]);
        acc[gri[p]] += (gv[p] * cinv[k]) * kv.second;
      }
    }
    std::sort(rows.begin(), rows.end());
    for (int64_t i : rows) {
      pat.rowidx.push_back(i);
      vc.push_back(i == j ? c0[j] : 0.0);
      vg.push_back(gcol[i]);
      vgcg.push_back(acc[i]);
      acc[i] = gcol[i] = 0.0;
      mark[i] = 0;
    }
    pat.colptr[j + 1] = (int64_t)pat.rowidx.size();
  }
  const size_t nnz = pat.rowidx.size();
  pat.val.assign(nnz, 1.0);
  comp.resize(3 * nnz);
  std::copy(vc.begin(), vc.end(), comp.begin());
  std::copy(vg.begin(), vg.end(), comp.begin() + nnz);
  std::copy(vgcg.begin(), vgcg.end(), comp.begin() + 2 * nnz);
  return std::string();
}

}  // namespace inla
