// 2-D triangle meshes for SPDE models: topology, P1 finite-element blocks and the barycentric
// observation projector, host code.
//
// Reference: crates/inla_fmesher/src/fmesher.rs:119-158 (build_mesh2d: validation and
// edge neighbours), 168-263 (observation_projector_triplets, locate_point_from: a walk across
// edge neighbours from the previous point's triangle), 544-626 (P1 blocks c0 / c1 / g1 / b1
// with a per-triangle diffusion scale and a global tensor H), 782-831 (barycentric
// classification), 870-893 (triangle validation). GEOM_EPSILON = 1e-15 (fmesher.rs:5).
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace inla {

constexpr double kGeomEps = 1e-15;

struct Mesh2D {
  std::vector<double> x, y;
  std::vector<std::array<int64_t, 3>> tri;
  std::vector<std::array<int64_t, 3>> nbr;  // neighbour across the edge opposite vertex e (-1: boundary)
};

// One assembled block in CSC (rows sorted within a column).
struct CscBlock {
  int64_t n = 0;
  std::vector<int64_t> colptr, rowidx;
  std::vector<double> val;
};

struct FemBlocks {
  CscBlock c0, c1, g1, b1;
  std::vector<double> area;
};

// Empty string on success, else the reference's error message.
std::string build_mesh2d(int64_t nv, const double* xy, int64_t ntri, const int64_t* tri, Mesh2D& m);

// triangle_scale: [ntri] or empty (all 1); H = [[hxx, hxy], [hxy, hyy]] symmetric positive definite.
std::string assemble_fem(const Mesh2D& m, const std::vector<double>& triangle_scale, double hxx, double hxy,
                         double hyy, FemBlocks& out);

// Triangle containing (px, py) by the reference's walk from `start` (-1: outside), with the
// barycentric weights of the point in that triangle.
int64_t locate_point(const Mesh2D& m, int64_t start, double px, double py, double bary[3]);

// Projector rows (up to three entries each, weights with |w| > 1e-15, columns ascending).
// Empty string on success, else the reference's error for the first point outside the mesh.
std::string projector(const Mesh2D& m, int64_t npts, const double* xy, std::vector<int64_t>& rowptr,
                      std::vector<int64_t>& colidx, std::vector<double>& val);

// 1-D meshes (crates/inla_fmesher/src/mesh1d.rs): knots strictly increasing and finite;
// blocks c0 / c1 / g1 (b1 empty) summed like the 2-D ones; projector rows (1 - w) x_i + w x_{i+1}
// with locations outside the knot range clamped to the end knots.
std::string check_mesh1d(int64_t n, const double* loc);
void assemble_fem1d(int64_t n, const double* loc, FemBlocks& out);
std::string projector1d(int64_t n, const double* loc, int64_t npts, const double* s, std::vector<int64_t>& rowptr,
                        std::vector<int64_t>& colidx, std::vector<double>& val);

// spde_precision_csc (crates/inla_stats/src/spde.rs:70-140) as components on one pattern:
// Q = tau^2 kappa^4 C0 + 2 tau^2 kappa^2 G1 + tau^2 G1 C0^-1 G1. c0: lumped mass diagonal;
// G1 in CSC with both triangles. The pattern is the union of the diagonal, G1 and
// G1 C0^-1 G1 (rows sorted); comp [3][nnz]. Entry (i, j) of G1 C0^-1 G1 is
// sum_k (G1_ik (1 / c0_k)) G1_kj over ascending k, the order of the reference's sparse
// products. Empty string on success, else the reference's error.
std::string spde_components(int64_t n, const double* c0, const int64_t* gcp, const int64_t* gri, const double* gv,
                            CscBlock& pattern, std::vector<double>& comp);

}  // namespace inla
