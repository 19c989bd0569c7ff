// Device forms of the mesh tools: P1 finite-element blocks, the SPDE precision components and
// the observation projector, computed on the GPU with results equal bit for bit to the host
// forms in mesh.cpp (crates/inla_fmesher/src/fmesher.rs:168-263, 544-626;
// crates/inla_stats/src/spde.rs:70-140).
//
// FEM: the blocks' patterns depend on the mesh topology only, so they are built once per mesh
// on the host together with, for every output entry, the list of its per-triangle
// contributions in the order the host assembly appends them (triangle order, then the order
// inside a triangle). One thread per output entry recomputes each contribution from the
// vertex coordinates and sums the list in that order. Multiplies and adds are kept apart
// (__dmul_rn / __dadd_rn) so that no fused multiply-add changes a rounding; the host compiler
// emits none either (plain x86-64 without FMA), so both sides round every operation alike.
//
// Projector: one thread per point walks from a triangle near the point (a bucket grid of
// triangle centroids) with the reference's acceptance test and barycentric formulas. A point
// whose three edge tests in its triangle all exceed `delta` lies inside that triangle by a
// margin no rounding can cross, so no other triangle passes the acceptance test and the
// reference's walk (from the previous point's triangle) ends in the same triangle with the
// same weights. Points that miss the margin (on or near an edge or a vertex), whose walk left
// the mesh or ran past its step limit are located again on the host in point order by the
// reference's walk from the previous point's triangle, exactly as the host projector does.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "gpu_factor.hpp"
#include "mesh.hpp"

namespace inla {

// Contribution lists of one FEM block: the CSC pattern (rows ascending in each column) and,
// per entry e, the contribution codes code[cptr[e] .. cptr[e+1]) in the host's append order.
// Codes: c0 3t + i; c1 and g1 9t + s (s the slot of the pair (i, j) in append order); b1
// 27t + 9i + 3j + k (vertex i, column vertex j, boundary edge k).
struct FemMap {
  std::vector<int64_t> colptr, rowidx, cptr, code;
};

// Host-side plan of a mesh's device forms (topology only) plus its device copies, built on
// the first device call and tied to the device current then.
struct MeshDevPlan {
  int device = -1;
  bool maps = false, locator = false, uploaded = false;
  FemMap c0, c1g1, b1;            // c1 and g1 share pattern and contribution lists
  double xmin = 0, ymin = 0, inv_wx = 0, inv_wy = 0, delta = 0;
  int grid = 1, maxsteps = 1;
  std::vector<int> seed;          // grid x grid: a triangle whose centroid lies in the cell, or -1
  DBuf<double> x, y;
  DBuf<int> tri, nbr, dseed;
  DBuf<int64_t> cptr[3], code[3];
  // projector scratch, reused across calls
  DBuf<int> ptri;
  DBuf<double> pw;
  DBuf<unsigned char> pflag, pcnt;
  DBuf<int64_t> fix_idx;
  DBuf<int> fix_tri;
  DBuf<double> fix_w;
};

// Patterns and contribution lists of the four blocks (no device use).
std::string build_fem_maps(const Mesh2D& m, MeshDevPlan& p);
// Bucket grid and walk bounds of the device locator (no device use).
void build_locator(const Mesh2D& m, MeshDevPlan& p);

// Device FEM values on the plan's patterns; any output may be null. diffusion {hxx, hxy, hyy}.
std::string fem_device(const Mesh2D& m, MeshDevPlan& p, const double* d_scale, double hxx, double hxy, double hyy,
                       double* d_area, double* d_c0, double* d_c1, double* d_g1, double* d_b1, cudaStream_t st);

// Device projector in CSR; synchronizes the stream. nnz_out: entries written.
std::string projector_device(const Mesh2D& m, MeshDevPlan& p, int64_t npts, const double* d_xy, int64_t* d_rowptr,
                             int64_t* d_colidx, double* d_vals, int64_t* nnz_out, cudaStream_t st);

// SPDE components on a fixed G1 pattern.
struct SpdePlan {
  int64_t n = 0;
  std::vector<int64_t> colptr, rowidx;   // components' pattern (host)
  int device = -1;
  bool uploaded = false;
  std::vector<int64_t> gcp;
  std::vector<int> gri;
  DBuf<int64_t> d_gcp;
  DBuf<int> d_gri, d_prow, d_pcol;
  DBuf<double> d_cinv;
};

std::string spde_plan_build(int64_t n, const int64_t* gcp, const int64_t* gri, SpdePlan& p);
std::string spde_components_device(SpdePlan& p, const double* d_c0, const double* d_gv, double* d_comp, int* d_status,
                                   cudaStream_t st);

}  // namespace inla
