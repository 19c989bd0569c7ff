// Device mesh tools (see mesh_dev.hpp): host plans, kernels and their drivers.
#include "mesh_dev.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>

#include "capi_common.hpp"
#include "mesh_dev_core.cuh"

namespace inla {

using namespace meshdev;

namespace {

// Buckets (row, code) by column in append order (a stable counting sort), orders each column by
// row (codes rise with the append order, so equal rows keep it) and groups equal rows.
template <class Emit>
void build_map(int64_t nv, Emit emit, FemMap& f) {
  std::vector<int64_t> start(nv + 1, 0);
  emit([&](int64_t r, int64_t c, int64_t code) {
    (void)r;
    (void)code;
    ++start[c + 1];
  });
  for (int64_t j = 0; j < nv; ++j) start[j + 1] += start[j];
  const int64_t total = start[nv];
  std::vector<std::pair<int64_t, int64_t>> rc(total);
  std::vector<int64_t> next(start.begin(), start.end() - 1);
  emit([&](int64_t r, int64_t c, int64_t code) { rc[next[c]++] = {r, code}; });
  f.colptr.assign(nv + 1, 0);
  f.rowidx.clear();
  f.cptr.clear();
  f.code.resize(total);
  for (int64_t j = 0; j < nv; ++j) {
    std::sort(rc.begin() + start[j], rc.begin() + start[j + 1]);
    for (int64_t p = start[j]; p < start[j + 1]; ++p) {
      if (p == start[j] || rc[p].first != rc[p - 1].first) {
        f.rowidx.push_back(rc[p].first);
        f.cptr.push_back(p);
      }
      f.code[p] = rc[p].second;
    }
    f.colptr[j + 1] = (int64_t)f.rowidx.size();
  }
  f.cptr.push_back(total);
}

}  // namespace

std::string build_fem_maps(const Mesh2D& m, MeshDevPlan& p) {
  const int64_t nv = (int64_t)m.x.size(), ntri = (int64_t)m.tri.size();
  if (nv > INT_MAX || ntri > INT_MAX / 3) return "mesh too large for the device forms (2^31 vertices or triangles)";
  // c0: (v_i, v_i) per triangle vertex
  build_map(nv,
            [&](auto&& put) {
              for (int64_t t = 0; t < ntri; ++t)
                for (int i = 0; i < 3; ++i) put(m.tri[t][i], m.tri[t][i], 3 * t + i);
            },
            p.c0);
  // c1 / g1: the nine pairs of each triangle in append order
  build_map(nv,
            [&](auto&& put) {
              for (int64_t t = 0; t < ntri; ++t)
                for (int s = 0; s < 9; ++s) put(m.tri[t][slot_a(s)], m.tri[t][slot_b(s)], 9 * t + s);
            },
            p.c1g1);
  // b1: triangles with a boundary edge k, pairs (v_i, v_j) for every i != k
  build_map(nv,
            [&](auto&& put) {
              for (int64_t t = 0; t < ntri; ++t) {
                const bool bnd[3] = {m.nbr[t][0] < 0, m.nbr[t][1] < 0, m.nbr[t][2] < 0};
                if (!(bnd[0] || bnd[1] || bnd[2])) continue;
                for (int i = 0; i < 3; ++i)
                  for (int j = 0; j < 3; ++j)
                    for (int k = 0; k < 3; ++k)
                      if (bnd[k] && i != k) put(m.tri[t][i], m.tri[t][j], 27 * t + 9 * i + 3 * j + k);
              }
            },
            p.b1);
  return std::string();
}

void build_locator(const Mesh2D& m, MeshDevPlan& p) {
  const int64_t nv = (int64_t)m.x.size(), ntri = (int64_t)m.tri.size();
  double xmin = INFINITY, xmax = -INFINITY, ymin = INFINITY, ymax = -INFINITY, amax = 0.0;
  for (int64_t i = 0; i < nv; ++i) {
    xmin = std::min(xmin, m.x[i]);
    xmax = std::max(xmax, m.x[i]);
    ymin = std::min(ymin, m.y[i]);
    ymax = std::max(ymax, m.y[i]);
    amax = std::max(amax, std::max(std::fabs(m.x[i]), std::fabs(m.y[i])));
  }
  // about four triangles per cell
  const int g = (int)std::max<int64_t>(1, std::min<int64_t>(4096, (int64_t)std::sqrt((double)ntri / 4.0)));
  p.grid = g;
  p.xmin = xmin;
  p.ymin = ymin;
  p.inv_wx = xmax > xmin ? g / (xmax - xmin) : 0.0;
  p.inv_wy = ymax > ymin ? g / (ymax - ymin) : 0.0;
  p.seed.assign((size_t)g * g, -1);
  for (int64_t t = 0; t < ntri; ++t) {
    const double cx = (m.x[m.tri[t][0]] + m.x[m.tri[t][1]] + m.x[m.tri[t][2]]) / 3.0;
    const double cy = (m.y[m.tri[t][0]] + m.y[m.tri[t][1]] + m.y[m.tri[t][2]]) / 3.0;
    if (!std::isfinite(cx) || !std::isfinite(cy)) continue;
    const int ix = std::min(g - 1, std::max(0, (int)((cx - xmin) * p.inv_wx)));
    const int iy = std::min(g - 1, std::max(0, (int)((cy - ymin) * p.inv_wy)));
    int& s = p.seed[(size_t)iy * g + ix];
    if (s < 0) s = (int)t;
  }
  // a walk from a seed in the point's cell crosses a few cells; a longer one goes to the host
  p.maxsteps = (int)std::min<int64_t>(std::max<int64_t>(3 * ntri, 1), 8 * (int64_t)g + 256);
  // edge tests above delta cannot change sign under rounding (|error| ~ 30 u amax^2) and clear
  // the acceptance threshold 1e-15 by three orders of magnitude
  p.delta = std::max(1e-12 * amax * amax, 1e-12);
}

// -- kernels --------------------------------------------------------------------------------

namespace {

constexpr int kNT = 256;

inline int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + kNT - 1) / kNT, 148 * 16)); }

__global__ void __launch_bounds__(kNT) k_fem_area(MeshView m, double* __restrict__ area) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < m.ntri; t += (int64_t)gridDim.x * blockDim.x) {
    const int v0 = m.tri[3 * t], v1 = m.tri[3 * t + 1], v2 = m.tri[3 * t + 2];
    area[t] = rmul(0.5, fabs(sa2(m.x[v0], m.y[v0], m.x[v1], m.y[v1], m.x[v2], m.y[v2])));
  }
}

// One output entry per thread: its contributions summed in the host's append order.
__global__ void __launch_bounds__(kNT) k_fem_entries(int which, int64_t nnz, const int64_t* __restrict__ cptr,
                                                    const int64_t* __restrict__ code, MeshView m,
                                                    const double* __restrict__ tscale, double hxx, double hxy,
                                                    double hyy, double* __restrict__ out) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p0 = cptr[e], p1 = cptr[e + 1];
    double acc = fem_contrib(which, code[p0], m, tscale, hxx, hxy, hyy);
    for (int64_t p = p0 + 1; p < p1; ++p) acc = radd(acc, fem_contrib(which, code[p], m, tscale, hxx, hxy, hyy));
    out[e] = acc;
  }
}

struct Locator {
  const int* seed;
  int grid, maxsteps;
  double xmin, ymin, inv_wx, inv_wy, delta;
};

__device__ __forceinline__ int cell_of(double v, double lo, double inv_w, int g) {
  const double f = rmul(rsub(v, lo), inv_w);
  if (!(f >= 0.0)) return 0;
  if (f >= (double)g) return g - 1;
  return (int)f;
}

// One point per thread: walk from the seed of the point's cell; flag 1 when certified.
__global__ void __launch_bounds__(kNT) k_locate(MeshView m, Locator L, int64_t npts, const double* __restrict__ xy,
                                               int* __restrict__ tri_out, double* __restrict__ w_out,
                                               unsigned char* __restrict__ flag, unsigned char* __restrict__ cnt) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < npts; r += (int64_t)gridDim.x * blockDim.x) {
    const double px = xy[2 * r], py = xy[2 * r + 1];
    int start = 0;
    if (finite_d(px) && finite_d(py)) {
      const int s = L.seed[(int64_t)cell_of(py, L.ymin, L.inv_wy, L.grid) * L.grid + cell_of(px, L.xmin, L.inv_wx, L.grid)];
      if (s >= 0) start = s;
    }
    double w[3] = {0.0, 0.0, 0.0};
    bool cert = false;
    const int t = m.ntri > 0 ? walk_locate(m, start, px, py, L.maxsteps, L.delta, w, cert) : -1;
    tri_out[r] = t;
    flag[r] = (t >= 0 && cert) ? 1 : 0;
    for (int k = 0; k < 3; ++k) w_out[3 * r + k] = w[k];
    cnt[r] = (unsigned char)((fabs(w[0]) > kEps) + (fabs(w[1]) > kEps) + (fabs(w[2]) > kEps));
  }
}

__global__ void __launch_bounds__(kNT) k_apply_fix(int64_t nfix, const int64_t* __restrict__ idx,
                                                  const int* __restrict__ tri, const double* __restrict__ w,
                                                  int* __restrict__ tri_out, double* __restrict__ w_out) {
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nfix; f += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx[f];
    tri_out[r] = tri[f];
    for (int k = 0; k < 3; ++k) w_out[3 * r + k] = w[3 * f + k];
  }
}

// Row r of the projector: weights with |w| > 1e-15, columns ascending.
__global__ void __launch_bounds__(kNT) k_proj_write(MeshView m, int64_t npts, const int* __restrict__ tri,
                                                   const double* __restrict__ w, const int64_t* __restrict__ rowptr,
                                                   int64_t* __restrict__ colidx, double* __restrict__ vals) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < npts; r += (int64_t)gridDim.x * blockDim.x) {
    const int t = tri[r];
    int col[3];
    double val[3];
    int ne = 0;
    for (int k = 0; k < 3; ++k) {
      const double wk = w[3 * r + k];
      if (fabs(wk) > kEps) {
        col[ne] = m.tri[3 * (int64_t)t + k];
        val[ne] = wk;
        ++ne;
      }
    }
    for (int a = 1; a < ne; ++a)  // insertion sort by column (the three vertices differ)
      for (int b = a; b > 0 && col[b] < col[b - 1]; --b) {
        const int c = col[b];
        col[b] = col[b - 1];
        col[b - 1] = c;
        const double v = val[b];
        val[b] = val[b - 1];
        val[b - 1] = v;
      }
    const int64_t q = rowptr[r];
    for (int k = 0; k < ne; ++k) {
      colidx[q + k] = col[k];
      vals[q + k] = val[k];
    }
  }
}

__global__ void __launch_bounds__(kNT) k_spde_cinv(int64_t n, const double* __restrict__ c0, double* __restrict__ cinv,
                                                  int* __restrict__ status) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double c = c0[i];
    cinv[i] = rdiv(1.0, c);
    if (fabs(c) < 1e-15 && status) *status = 1;
  }
}

// position of row i in column k of G (rows strictly ascending), or -1
__device__ __forceinline__ int64_t find_row(const int64_t* gcp, const int* gri, int64_t k, int i) {
  int64_t lo = gcp[k], hi = gcp[k + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    const int r = gri[mid];
    if (r == i) return mid;
    if (r < i) lo = mid + 1;
    else hi = mid;
  }
  return -1;
}

// Entry (i, j) of the three components: C0 (diagonal), G1, and sum over ascending k of
// (G1_ik / c0_k) G1_kj, each sum started from 0.0 as the host's accumulators are.
__global__ void __launch_bounds__(kNT) k_spde_comp(int64_t nnz, const int* __restrict__ prow,
                                                  const int* __restrict__ pcol, const int64_t* __restrict__ gcp,
                                                  const int* __restrict__ gri, const double* __restrict__ gv,
                                                  const double* __restrict__ c0, const double* __restrict__ cinv,
                                                  double* __restrict__ comp) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
    const int i = prow[e], j = pcol[e];
    const int64_t pij = find_row(gcp, gri, j, i);
    double acc = 0.0;
    for (int64_t p = gcp[j]; p < gcp[j + 1]; ++p) {
      const int k = gri[p];
      const int64_t q = find_row(gcp, gri, k, i);
      if (q >= 0) acc = radd(acc, rmul(rmul(gv[q], cinv[k]), gv[p]));
    }
    comp[e] = i == j ? c0[j] : 0.0;
    comp[nnz + e] = pij >= 0 ? radd(0.0, gv[pij]) : 0.0;
    comp[2 * nnz + e] = acc;
  }
}

}  // namespace

namespace {

// throws CudaError (INLA_ERR_CUDA at the C ABI) when no device is usable
std::string current_device(int& dev) {
  INLA_CUDA(cudaGetDevice(&dev));
  return std::string();
}

// Patterns, locator and device copies of the mesh, made once (on the device current then).
std::string ensure_mesh_device(const Mesh2D& m, MeshDevPlan& p, cudaStream_t st) {
  int dev = 0;
  std::string err = current_device(dev);
  if (!err.empty()) return err;
  if (p.uploaded) {
    if (dev != p.device)
      return "the mesh's device data live on device " + std::to_string(p.device) + ", not on the current device " +
             std::to_string(dev);
    return std::string();
  }
  if (!p.maps) {
    err = build_fem_maps(m, p);
    if (!err.empty()) return err;
    p.maps = true;
  }
  if (!p.locator) {
    build_locator(m, p);
    p.locator = true;
  }
  const int64_t ntri = (int64_t)m.tri.size();
  std::vector<int> tri(3 * ntri), nbr(3 * ntri);
  for (int64_t t = 0; t < ntri; ++t)
    for (int e = 0; e < 3; ++e) {
      tri[3 * t + e] = (int)m.tri[t][e];
      nbr[3 * t + e] = (int)m.nbr[t][e];
    }
  p.x.upload(m.x, st);
  p.y.upload(m.y, st);
  p.tri.upload(tri, st);
  p.nbr.upload(nbr, st);
  p.dseed.upload(p.seed, st);
  const FemMap* maps[3] = {&p.c0, &p.c1g1, &p.b1};
  for (int b = 0; b < 3; ++b) {
    p.cptr[b].upload(maps[b]->cptr, st);
    p.code[b].upload(maps[b]->code, st);
  }
  INLA_CUDA(cudaStreamSynchronize(st));
  p.device = dev;
  p.uploaded = true;
  return std::string();
}

MeshView view_of(const MeshDevPlan& p, int64_t ntri) {
  MeshView v;
  v.x = p.x.p;
  v.y = p.y.p;
  v.tri = p.tri.p;
  v.nbr = p.nbr.p;
  v.ntri = ntri;
  return v;
}

}  // namespace

std::string fem_device(const Mesh2D& m, MeshDevPlan& p, const double* d_scale, double hxx, double hxy, double hyy,
                       double* d_area, double* d_c0, double* d_c1, double* d_g1, double* d_b1, cudaStream_t st) {
  if (!std::isfinite(hxx) || !std::isfinite(hxy) || !std::isfinite(hyy))
    return "diffusion tensor entries must be finite";
  if (hxx * hyy - hxy * hxy <= 0.0) return "diffusion tensor must be SPD";
  const std::string err = ensure_mesh_device(m, p, st);
  if (!err.empty()) return err;
  const int64_t ntri = (int64_t)m.tri.size();
  const MeshView mv = view_of(p, ntri);
  if (d_area && ntri > 0) {
    k_fem_area<<<grid_for(ntri), kNT, 0, st>>>(mv, d_area);
    INLA_CUDA(cudaGetLastError());
    ++g_launches;
  }
  double* outs[4] = {d_c0, d_c1, d_g1, d_b1};
  const int map_of[4] = {0, 1, 1, 2};
  const FemMap* maps[3] = {&p.c0, &p.c1g1, &p.b1};
  for (int which = 0; which < 4; ++which) {
    const int b = map_of[which];
    const int64_t nnz = (int64_t)maps[b]->rowidx.size();
    if (!outs[which] || nnz == 0) continue;
    k_fem_entries<<<grid_for(nnz), kNT, 0, st>>>(which, nnz, p.cptr[b].p, p.code[b].p, mv, d_scale, hxx, hxy, hyy,
                                                 outs[which]);
    INLA_CUDA(cudaGetLastError());
    ++g_launches;
  }
  return std::string();
}

std::string projector_device(const Mesh2D& m, MeshDevPlan& p, int64_t npts, const double* d_xy, int64_t* d_rowptr,
                             int64_t* d_colidx, double* d_vals, int64_t* nnz_out, cudaStream_t st) {
  std::string err = ensure_mesh_device(m, p, st);
  if (!err.empty()) return err;
  std::vector<int64_t> rp(npts + 1, 0);
  if (npts == 0) {
    INLA_CUDA(cudaMemcpyAsync(d_rowptr, rp.data(), sizeof(int64_t), cudaMemcpyHostToDevice, st));
    INLA_CUDA(cudaStreamSynchronize(st));
    if (nnz_out) *nnz_out = 0;
    return std::string();
  }
  const int64_t ntri = (int64_t)m.tri.size();
  const MeshView mv = view_of(p, ntri);
  p.ptri.alloc(npts);
  p.pw.alloc(3 * npts);
  p.pflag.alloc(npts);
  p.pcnt.alloc(npts);
  Locator L;
  L.seed = p.dseed.p;
  L.grid = p.grid;
  L.maxsteps = p.maxsteps;
  L.xmin = p.xmin;
  L.ymin = p.ymin;
  L.inv_wx = p.inv_wx;
  L.inv_wy = p.inv_wy;
  L.delta = p.delta;
  k_locate<<<grid_for(npts), kNT, 0, st>>>(mv, L, npts, d_xy, p.ptri.p, p.pw.p, p.pflag.p, p.pcnt.p);
  INLA_CUDA(cudaGetLastError());
  ++g_launches;
  std::vector<unsigned char> flag(npts), cnt(npts);
  std::vector<int> tri(npts);
  INLA_CUDA(cudaMemcpyAsync(flag.data(), p.pflag.p, npts, cudaMemcpyDeviceToHost, st));
  INLA_CUDA(cudaMemcpyAsync(cnt.data(), p.pcnt.p, npts, cudaMemcpyDeviceToHost, st));
  INLA_CUDA(cudaMemcpyAsync(tri.data(), p.ptri.p, npts * sizeof(int), cudaMemcpyDeviceToHost, st));
  INLA_CUDA(cudaStreamSynchronize(st));
  // points without a certified location: the reference's walk in point order, each from the
  // previous point's triangle, as the host projector runs it
  std::vector<int64_t> fidx;
  std::vector<int> ftri;
  std::vector<double> fw;
  std::vector<double> xy;
  for (int64_t r = 0; r < npts; ++r) {
    if (flag[r]) continue;
    if (xy.empty()) {
      xy.resize(2 * npts);
      INLA_CUDA(cudaMemcpyAsync(xy.data(), d_xy, 2 * npts * sizeof(double), cudaMemcpyDeviceToHost, st));
      INLA_CUDA(cudaStreamSynchronize(st));
    }
    double w[3];
    const int64_t t = locate_point(m, r == 0 ? 0 : tri[r - 1], xy[2 * r], xy[2 * r + 1], w);
    if (t < 0) {
      char buf[128];
      std::snprintf(buf, sizeof(buf), "observation point (%.17g, %.17g) is outside the mesh", xy[2 * r],
                    xy[2 * r + 1]);
      return buf;
    }
    tri[r] = (int)t;
    fidx.push_back(r);
    ftri.push_back((int)t);
    fw.insert(fw.end(), w, w + 3);
    cnt[r] = (unsigned char)((std::fabs(w[0]) > kEps) + (std::fabs(w[1]) > kEps) + (std::fabs(w[2]) > kEps));
  }
  if (!fidx.empty()) {
    const int64_t nfix = (int64_t)fidx.size();
    p.fix_idx.upload(fidx, st);
    p.fix_tri.upload(ftri, st);
    p.fix_w.upload(fw, st);
    k_apply_fix<<<grid_for(nfix), kNT, 0, st>>>(nfix, p.fix_idx.p, p.fix_tri.p, p.fix_w.p, p.ptri.p, p.pw.p);
    INLA_CUDA(cudaGetLastError());
    ++g_launches;
  }
  for (int64_t r = 0; r < npts; ++r) rp[r + 1] = rp[r] + cnt[r];
  INLA_CUDA(cudaMemcpyAsync(d_rowptr, rp.data(), (npts + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
  k_proj_write<<<grid_for(npts), kNT, 0, st>>>(mv, npts, p.ptri.p, p.pw.p, d_rowptr, d_colidx, d_vals);
  INLA_CUDA(cudaGetLastError());
  ++g_launches;
  INLA_CUDA(cudaStreamSynchronize(st));
  if (nnz_out) *nnz_out = rp[npts];
  return std::string();
}

std::string spde_plan_build(int64_t n, const int64_t* gcp, const int64_t* gri, SpdePlan& p) {
  if (n <= 0) return "SPDE requires non-empty FEM blocks";
  if (n > INT_MAX) return "SPDE plan: more than 2^31 - 1 nodes";
  if (gcp[0] != 0) return "SPDE plan: colptr[0] must be 0";
  for (int64_t j = 0; j < n; ++j) {
    if (gcp[j + 1] < gcp[j]) return "SPDE plan: colptr not monotone";
    for (int64_t q = gcp[j]; q < gcp[j + 1]; ++q) {
      if (gri[q] < 0 || gri[q] >= n) return "SPDE plan: row index out of range";
      if (q > gcp[j] && gri[q] <= gri[q - 1]) return "SPDE plan: rows must be strictly ascending within each column";
    }
  }
  p.n = n;  // p is a fresh plan
  p.rowidx.clear();
  p.gcp.assign(gcp, gcp + n + 1);
  p.gri.assign(gri, gri + gcp[n]);
  // pattern of column j: j, the rows of G1 column j and of G1 column k for each of those rows k
  p.colptr.assign(n + 1, 0);
  std::vector<char> mark(n, 0);
  std::vector<int64_t> rows;
  for (int64_t j = 0; j < n; ++j) {
    rows.clear();
    auto touch = [&](int64_t i) {
      if (!mark[i]) {
        mark[i] = 1;
        rows.push_back(i);
      }
    };
    touch(j);
    for (int64_t q = gcp[j]; q < gcp[j + 1]; ++q) touch(gri[q]);
    for (int64_t q = gcp[j]; q < gcp[j + 1]; ++q)
      for (int64_t r = gcp[gri[q]]; r < gcp[gri[q] + 1]; ++r) touch(gri[r]);
    std::sort(rows.begin(), rows.end());
    for (int64_t i : rows) {
      p.rowidx.push_back(i);
      mark[i] = 0;
    }
    p.colptr[j + 1] = (int64_t)p.rowidx.size();
  }
  return std::string();
}

std::string spde_components_device(SpdePlan& p, const double* d_c0, const double* d_gv, double* d_comp, int* d_status,
                                   cudaStream_t st) {
  int dev = 0;
  std::string err = current_device(dev);
  if (!err.empty()) return err;
  const int64_t nnz = (int64_t)p.rowidx.size();
  if (!p.uploaded) {
    std::vector<int> prow(nnz), pcol(nnz);
    for (int64_t j = 0; j < p.n; ++j)
      for (int64_t q = p.colptr[j]; q < p.colptr[j + 1]; ++q) {
        prow[q] = (int)p.rowidx[q];
        pcol[q] = (int)j;
      }
    p.d_gcp.upload(p.gcp, st);
    p.d_gri.upload(p.gri, st);
    p.d_prow.upload(prow, st);
    p.d_pcol.upload(pcol, st);
    p.d_cinv.alloc(p.n);
    INLA_CUDA(cudaStreamSynchronize(st));
    p.device = dev;
    p.uploaded = true;
  } else if (dev != p.device) {
    return "the SPDE plan's device data live on device " + std::to_string(p.device) + ", not on the current device " +
           std::to_string(dev);
  }
  if (d_status) INLA_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), st));
  k_spde_cinv<<<grid_for(p.n), kNT, 0, st>>>(p.n, d_c0, p.d_cinv.p, d_status);
  INLA_CUDA(cudaGetLastError());
  k_spde_comp<<<grid_for(nnz), kNT, 0, st>>>(nnz, p.d_prow.p, p.d_pcol.p, p.d_gcp.p, p.d_gri.p, d_gv, d_c0, p.d_cinv.p,
                                             d_comp);
  INLA_CUDA(cudaGetLastError());
  g_launches += 2;
  return std::string();
}

}  // namespace inla
