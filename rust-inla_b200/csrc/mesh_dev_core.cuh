// Arithmetic of the device mesh tools, written once for host and device. On the device every
// multiply, add and divide is a separately rounded IEEE operation (no contraction into fused
// multiply-adds), so each value equals the host assembly's (mesh.cpp) bit for bit; on the host
// the same expressions compile to the same operations.
#pragma once
#include <cmath>
#include <cstdint>

namespace inla {
namespace meshdev {

constexpr double kEps = 1e-15;  // GEOM_EPSILON (fmesher.rs:5)

__host__ __device__ __forceinline__ double rmul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
__host__ __device__ __forceinline__ double radd(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
__host__ __device__ __forceinline__ double rsub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
__host__ __device__ __forceinline__ double rdiv(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}

__host__ __device__ __forceinline__ bool finite_d(double v) { return rsub(v, v) == 0.0; }

// (b - a) x (c - a): twice the signed area of (a, b, c)
__host__ __device__ __forceinline__ double sa2(double ax, double ay, double bx, double by, double cx, double cy) {
  return rsub(rmul(rsub(bx, ax), rsub(cy, ay)), rmul(rsub(by, ay), rsub(cx, ax)));
}

struct MeshView {
  const double* x;
  const double* y;
  const int* tri;   // [ntri][3]
  const int* nbr;   // [ntri][3], -1 on the boundary
  int64_t ntri;
};

// Per-triangle quantities of assemble_fem (fmesher.rs:544-626): area, the stiffness
// denominator's area fa, the diffusion scale and e[i][j] = (H g_i) . g_j with g_i the edge
// opposite vertex i rotated by -90 degrees (computed for i <= j and mirrored).
struct TriGeom {
  double area, fa, scale;
  double e[3][3];
};

__host__ __device__ inline void tri_geom(const MeshView& m, int64_t t, const double* tscale, double hxx, double hxy,
                                         double hyy, TriGeom& g) {
  const int v0 = m.tri[3 * t], v1 = m.tri[3 * t + 1], v2 = m.tri[3 * t + 2];
  const double s0x = m.x[v0], s0y = m.y[v0], s1x = m.x[v1], s1y = m.y[v1], s2x = m.x[v2], s2y = m.y[v2];
  const double ex[3] = {rsub(s2x, s1x), rsub(s0x, s2x), rsub(s1x, s0x)};
  const double ey[3] = {rsub(s2y, s1y), rsub(s0y, s2y), rsub(s1y, s0y)};
  g.area = rmul(0.5, fabs(sa2(s0x, s0y, s1x, s1y, s2x, s2y)));
  double fa = rmul(0.5, fabs(rsub(rmul(ex[0], ey[1]), rmul(ey[0], ex[1]))));
  if (fa <= kEps) fa = g.area;
  g.fa = fa;
  g.scale = tscale ? tscale[t] : 1.0;
  for (int i = 0; i < 3; ++i) {
    const double gix = ey[i], giy = -ex[i];
    const double hx = radd(rmul(hxx, gix), rmul(hxy, giy)), hy = radd(rmul(hxy, gix), rmul(hyy, giy));
    for (int j = i; j < 3; ++j) {
      const double gjx = ey[j], gjy = -ex[j];
      g.e[i][j] = radd(rmul(hx, gjx), rmul(hy, gjy));
      g.e[j][i] = g.e[i][j];
    }
  }
}

// Slots of the c1 / g1 pairs of one triangle in the host's append order: (a[s], b[s]).
// a = {0, 0, 1, 0, 2, 1, 1, 2, 2}, b = {0, 1, 0, 2, 0, 1, 2, 1, 2}, one hex digit per slot from the right
__host__ __device__ __forceinline__ int slot_a(int s) { return (int)((0x221120100ULL >> (4 * s)) & 0xFULL); }
__host__ __device__ __forceinline__ int slot_b(int s) { return (int)((0x212102010ULL >> (4 * s)) & 0xFULL); }

// Value of one contribution (see FemMap for the codes); which: 0 c0, 1 c1, 2 g1, 3 b1.
__host__ __device__ inline double fem_contrib(int which, int64_t code, const MeshView& m, const double* tscale,
                                              double hxx, double hxy, double hyy) {
  TriGeom g;
  if (which == 0) {
    tri_geom(m, code / 3, tscale, hxx, hxy, hyy, g);
    return rdiv(g.area, 3.0);
  }
  if (which == 1 || which == 2) {
    const int64_t t = code / 9;
    const int s = (int)(code - 9 * t), a = slot_a(s), b = slot_b(s);
    tri_geom(m, t, tscale, hxx, hxy, hyy, g);
    if (which == 1) return a == b ? rdiv(g.area, 6.0) : rdiv(g.area, 12.0);
    return rdiv(rmul(g.scale, g.e[a][b]), rmul(4.0, g.fa));
  }
  const int64_t t = code / 27;
  const int r = (int)(code - 27 * t), j = (r / 3) % 3, k = r % 3;
  tri_geom(m, t, tscale, hxx, hxy, hyy, g);
  const double vij = rdiv(-1.0, rmul(4.0, g.fa));
  return rmul(rmul(g.scale, g.e[k][j]), vij);
}

// The reference's walk (fmesher.rs:221-263) from `start`, at most `maxsteps` triangles. Returns
// the accepting triangle with its barycentric weights, or -1 when the walk left the mesh or ran
// out of steps. certified: every edge test in that triangle exceeds delta and the weights are
// finite (the point lies inside by a margin, so every walk ends there).
__host__ __device__ inline int walk_locate(const MeshView& m, int start, double px, double py, int maxsteps,
                                           double delta, double w[3], bool& certified) {
  certified = false;
  int cur = start;
  for (int step = 0; step < maxsteps; ++step) {
    const int* tv = m.tri + 3 * (int64_t)cur;
    const double ax = m.x[tv[0]], ay = m.y[tv[0]], bx = m.x[tv[1]], by = m.y[tv[1]], cx = m.x[tv[2]],
                 cy = m.y[tv[2]];
    const double den = sa2(ax, ay, bx, by, cx, cy);
    const double orient = den >= 0.0 ? 1.0 : -1.0;
    double most_negative = 0.0;
    int leaving = -1;
    bool inside = true;
    for (int e = 0; e < 3; ++e) {
      const int va = tv[(e + 1) % 3], vb = tv[(e + 2) % 3];
      const double side = rmul(orient, sa2(m.x[va], m.y[va], m.x[vb], m.y[vb], px, py));
      if (side < most_negative) {
        most_negative = side;
        leaving = e;
      }
      inside = inside && side > delta;
    }
    if (most_negative >= -kEps) {
      if (fabs(den) <= kEps) {
        w[0] = w[1] = w[2] = NAN;
        return cur;
      }
      w[0] = rdiv(sa2(bx, by, cx, cy, px, py), den);
      w[1] = rdiv(sa2(cx, cy, ax, ay, px, py), den);
      w[2] = rsub(rsub(1.0, w[0]), w[1]);
      certified = inside && finite_d(w[0]) && finite_d(w[1]) && finite_d(w[2]);
      return cur;
    }
    if (leaving < 0) return -1;
    const int next = m.nbr[3 * (int64_t)cur + leaving];
    if (next < 0) return -1;
    cur = next;
  }
  return -1;
}

}  // namespace meshdev
}  // namespace inla
