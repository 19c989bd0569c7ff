// C ABI of the mesh tools: mesh topology, FEM blocks, point location and the observation
// projector (crates/inla_fmesher/src/fmesher.rs) on the host, and their device forms
// (mesh_dev.cu) with the SPDE components (crates/inla_stats/src/spde.rs:70-140).
#include <cstring>
#include <memory>

#include "capi_common.hpp"
#include "inla_b200.h"
#include "mesh.hpp"
#include "mesh_dev.hpp"

using namespace inla;

struct inla_mesh {
  Mesh2D m;
  std::unique_ptr<FemBlocks> fem;
  std::unique_ptr<MeshDevPlan> dev;  // patterns, contribution lists and device copies (first use)
};

struct inla_spde_plan {
  SpdePlan p;
};

namespace {

MeshDevPlan& dev_plan(inla_mesh* h) {
  if (!h->dev) h->dev.reset(new MeshDevPlan());
  return *h->dev;
}

}  // namespace

extern "C" {

int inla_mesh_create(int64_t nv, const double* xy, int64_t ntri, const int64_t* tri, inla_mesh** out) {
  try {
    if (!out || nv < 0 || ntri < 0 || (nv > 0 && !xy) || (ntri > 0 && !tri))
      return fail(INLA_ERR_INVALID, "inla_mesh_create: invalid argument");
    std::unique_ptr<inla_mesh> h(new inla_mesh());
    const std::string err = build_mesh2d(nv, xy, ntri, tri, h->m);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    *out = h.release();
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

void inla_mesh_free(inla_mesh* h) { delete h; }

int inla_mesh_neighbors(const inla_mesh* h, int64_t* nbr) {
  if (!h || !nbr) return fail(INLA_ERR_INVALID, "inla_mesh_neighbors: invalid argument");
  for (size_t t = 0; t < h->m.nbr.size(); ++t)
    for (int e = 0; e < 3; ++e) nbr[3 * t + e] = h->m.nbr[t][e];
  return INLA_OK;
}

int inla_mesh_fem(inla_mesh* h, const double* triangle_scale, const double* diffusion, double* areas) {
  try {
    if (!h) return fail(INLA_ERR_INVALID, "inla_mesh_fem: invalid argument");
    std::vector<double> scale;
    if (triangle_scale) scale.assign(triangle_scale, triangle_scale + h->m.tri.size());
    const double hxx = diffusion ? diffusion[0] : 1.0, hxy = diffusion ? diffusion[1] : 0.0,
                 hyy = diffusion ? diffusion[2] : 1.0;
    std::unique_ptr<FemBlocks> f(new FemBlocks());
    const std::string err = assemble_fem(h->m, scale, hxx, hxy, hyy, *f);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    if (areas) std::memcpy(areas, f->area.data(), sizeof(double) * f->area.size());
    h->fem = std::move(f);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_mesh_fem_block(const inla_mesh* h, int which, int64_t* nnz, int64_t* colptr, int64_t* rowidx,
                        double* vals) {
  if (!h || !h->fem || which < 0 || which > 3) return fail(INLA_ERR_INVALID, "inla_mesh_fem_block: no such block");
  const CscBlock& b = which == 0 ? h->fem->c0 : which == 1 ? h->fem->c1 : which == 2 ? h->fem->g1 : h->fem->b1;
  if (nnz) *nnz = (int64_t)b.rowidx.size();
  if (colptr) std::memcpy(colptr, b.colptr.data(), sizeof(int64_t) * b.colptr.size());
  if (rowidx) std::memcpy(rowidx, b.rowidx.data(), sizeof(int64_t) * b.rowidx.size());
  if (vals) std::memcpy(vals, b.val.data(), sizeof(double) * b.val.size());
  return INLA_OK;
}

int inla_mesh_locate(const inla_mesh* h, int64_t npts, const double* xy, int64_t* tri, double* bary) {
  if (!h || npts < 0 || (npts > 0 && (!xy || !tri))) return fail(INLA_ERR_INVALID, "inla_mesh_locate: invalid argument");
  for (int64_t r = 0; r < npts; ++r) {
    double w[3];
    tri[r] = locate_point(h->m, 0, xy[2 * r], xy[2 * r + 1], w);
    if (bary)
      for (int k = 0; k < 3; ++k) bary[3 * r + k] = tri[r] >= 0 ? w[k] : NAN;
  }
  return INLA_OK;
}

int inla_mesh_projector(const inla_mesh* h, int64_t npts, const double* xy, int64_t* rowptr, int64_t* colidx,
                        double* vals) {
  try {
    if (!h || npts < 0 || (npts > 0 && !xy) || !rowptr || !colidx || !vals)
      return fail(INLA_ERR_INVALID, "inla_mesh_projector: invalid argument");
    std::vector<int64_t> rp, ci;
    std::vector<double> v;
    const std::string err = projector(h->m, npts, xy, rp, ci, v);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    std::memcpy(rowptr, rp.data(), sizeof(int64_t) * rp.size());
    std::memcpy(colidx, ci.data(), sizeof(int64_t) * ci.size());
    std::memcpy(vals, v.data(), sizeof(double) * v.size());
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_mesh1d_fem(int64_t n, const double* loc, int which, int64_t* nnz, int64_t* colptr, int64_t* rowidx,
                    double* vals) {
  try {
    if (!loc || which < 0 || which > 3) return fail(INLA_ERR_INVALID, "inla_mesh1d_fem: invalid argument");
    const std::string err = check_mesh1d(n, loc);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    FemBlocks f;
    assemble_fem1d(n, loc, f);
    const CscBlock& b = which == 0 ? f.c0 : which == 1 ? f.c1 : which == 2 ? f.g1 : f.b1;
    if (nnz) *nnz = (int64_t)b.rowidx.size();
    if (colptr) std::memcpy(colptr, b.colptr.data(), sizeof(int64_t) * b.colptr.size());
    if (rowidx) std::memcpy(rowidx, b.rowidx.data(), sizeof(int64_t) * b.rowidx.size());
    if (vals) std::memcpy(vals, b.val.data(), sizeof(double) * b.val.size());
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_mesh1d_projector(int64_t n, const double* loc, int64_t npts, const double* s, int64_t* rowptr,
                          int64_t* colidx, double* vals) {
  try {
    if (!loc || npts < 0 || (npts > 0 && !s) || !rowptr || !colidx || !vals)
      return fail(INLA_ERR_INVALID, "inla_mesh1d_projector: invalid argument");
    std::string err = check_mesh1d(n, loc);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    std::vector<int64_t> rp, ci;
    std::vector<double> v;
    err = projector1d(n, loc, npts, s, rp, ci, v);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    std::memcpy(rowptr, rp.data(), sizeof(int64_t) * rp.size());
    std::memcpy(colidx, ci.data(), sizeof(int64_t) * ci.size());
    std::memcpy(vals, v.data(), sizeof(double) * v.size());
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_spde_components(int64_t n, const double* c0, const int64_t* g_colptr, const int64_t* g_rowidx,
                         const double* g_vals, int64_t* nnz, int64_t* colptr, int64_t* rowidx, double* comp) {
  try {
    if (n <= 0 || !c0 || !g_colptr || !g_rowidx || !g_vals)
      return fail(INLA_ERR_INVALID, "SPDE requires non-empty FEM blocks");
    if (g_colptr[0] != 0) return fail(INLA_ERR_INVALID, "inla_spde_components: colptr[0] must be 0");
    for (int64_t j = 0; j < n; ++j) {
      if (g_colptr[j + 1] < g_colptr[j]) return fail(INLA_ERR_INVALID, "inla_spde_components: colptr not monotone");
      for (int64_t p = g_colptr[j]; p < g_colptr[j + 1]; ++p)
        if (g_rowidx[p] < 0 || g_rowidx[p] >= n)
          return fail(INLA_ERR_INVALID, "inla_spde_components: row index out of range");
    }
    CscBlock pat;
    std::vector<double> cv;
    const std::string err = spde_components(n, c0, g_colptr, g_rowidx, g_vals, pat, cv);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    if (nnz) *nnz = (int64_t)pat.rowidx.size();
    if (colptr) std::memcpy(colptr, pat.colptr.data(), sizeof(int64_t) * pat.colptr.size());
    if (rowidx) std::memcpy(rowidx, pat.rowidx.data(), sizeof(int64_t) * pat.rowidx.size());
    if (comp) std::memcpy(comp, cv.data(), sizeof(double) * cv.size());
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_mesh_fem_pattern(inla_mesh* h, int which, int64_t* nnz, int64_t* colptr, int64_t* rowidx) {
  try {
    if (!h || which < 0 || which > 3) return fail(INLA_ERR_INVALID, "inla_mesh_fem_pattern: invalid argument");
    MeshDevPlan& p = dev_plan(h);
    if (!p.maps) {
      const std::string err = build_fem_maps(h->m, p);
      if (!err.empty()) return fail(INLA_ERR_INVALID, err);
      p.maps = true;
    }
    const FemMap& f = which == 0 ? p.c0 : which == 3 ? p.b1 : p.c1g1;
    if (nnz) *nnz = (int64_t)f.rowidx.size();
    if (colptr) std::memcpy(colptr, f.colptr.data(), sizeof(int64_t) * f.colptr.size());
    if (rowidx) std::memcpy(rowidx, f.rowidx.data(), sizeof(int64_t) * f.rowidx.size());
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_mesh_fem_dev(inla_mesh* h, const double* d_triangle_scale, const double* diffusion, double* d_areas,
                      double* d_c0, double* d_c1, double* d_g1, double* d_b1, void* stream) {
  try {
    if (!h) return fail(INLA_ERR_INVALID, "inla_mesh_fem_dev: invalid argument");
    const double hxx = diffusion ? diffusion[0] : 1.0, hxy = diffusion ? diffusion[1] : 0.0,
                 hyy = diffusion ? diffusion[2] : 1.0;
    const std::string err = fem_device(h->m, dev_plan(h), d_triangle_scale, hxx, hxy, hyy, d_areas, d_c0, d_c1, d_g1,
                                       d_b1, (cudaStream_t)stream);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_mesh_projector_dev(inla_mesh* h, int64_t npts, const double* d_xy, int64_t* d_rowptr, int64_t* d_colidx,
                            double* d_vals, int64_t* nnz, void* stream) {
  try {
    if (!h || npts < 0 || (npts > 0 && (!d_xy || !d_colidx || !d_vals)) || !d_rowptr)
      return fail(INLA_ERR_INVALID, "inla_mesh_projector_dev: invalid argument");
    if (npts > INT32_MAX) return fail(INLA_ERR_INVALID, "inla_mesh_projector_dev: more than 2^31 - 1 points");
    const std::string err =
        projector_device(h->m, dev_plan(h), npts, d_xy, d_rowptr, d_colidx, d_vals, nnz, (cudaStream_t)stream);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

int inla_spde_plan_create(int64_t n, const int64_t* g_colptr, const int64_t* g_rowidx, inla_spde_plan** out) {
  try {
    if (!out || !g_colptr || (n > 0 && g_colptr[n] > 0 && !g_rowidx))
      return fail(INLA_ERR_INVALID, "inla_spde_plan_create: invalid argument");
    std::unique_ptr<inla_spde_plan> h(new inla_spde_plan());
    const std::string err = spde_plan_build(n, g_colptr, g_rowidx, h->p);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    *out = h.release();
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

void inla_spde_plan_free(inla_spde_plan* h) { delete h; }

int inla_spde_plan_pattern(const inla_spde_plan* h, int64_t* nnz, int64_t* colptr, int64_t* rowidx) {
  if (!h) return fail(INLA_ERR_INVALID, "inla_spde_plan_pattern: invalid argument");
  if (nnz) *nnz = (int64_t)h->p.rowidx.size();
  if (colptr) std::memcpy(colptr, h->p.colptr.data(), sizeof(int64_t) * h->p.colptr.size());
  if (rowidx) std::memcpy(rowidx, h->p.rowidx.data(), sizeof(int64_t) * h->p.rowidx.size());
  return INLA_OK;
}

int inla_spde_components_dev(inla_spde_plan* h, const double* d_c0, const double* d_g_vals, double* d_comp,
                             int* d_status, void* stream) {
  try {
    if (!h || !d_c0 || (!d_g_vals && !h->p.gri.empty()) || !d_comp)
      return fail(INLA_ERR_INVALID, "inla_spde_components_dev: invalid argument");
    const std::string err = spde_components_device(h->p, d_c0, d_g_vals, d_comp, d_status, (cudaStream_t)stream);
    if (!err.empty()) return fail(INLA_ERR_INVALID, err);
    return INLA_OK;
  } catch (...) {
    return map_exception();
  }
}

}  // extern "C"
