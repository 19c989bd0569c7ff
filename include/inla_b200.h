/*
 * inla_b200 — C ABI of the B200-native INLA inner hot path (CUDA sm_100a, FP64).
 *
 * Drop-in seam for rust-inla's faer-backed solver path. Every entry point takes
 * plain host pointers and sizes (caller-owned, copied by the call) or, in the
 * `_dev` variants, device pointers; no C++ exceptions cross this boundary and
 * each call returns an INLA_* status code. Device memory is owned by handles.
 *
 * Matrix convention (same as the reference): a square CSC matrix with int64
 * column pointers and row indices holding BOTH triangles of a symmetric
 * matrix; only entries with row >= col are read as values
 * (crates/inla_math/src/sparse_ldlt.rs:82-92). Explicit zeros stay structural.
 */
#ifndef INLA_B200_H
#define INLA_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. They map 1:1 onto the reference's error enums
 * (crates/inla_math/src/solver.rs:10-27, crates/inla_math/src/error.rs:7-38). */
enum {
  INLA_OK = 0,
  INLA_ERR_SINGULAR = 1,       /* SolverError::Singular (|D_j| < 1e-14 or non-finite) */
  INLA_ERR_NOT_PD = 2,         /* SolverError::NotPositiveDefinite */
  INLA_ERR_DIM_MISMATCH = 3,   /* MathError::DimensionMismatch / NotSquare -> SolveFailure */
  INLA_ERR_OOM = 4,            /* MathError::OutOfMemory */
  INLA_ERR_NONCONVERGED = 5,   /* "Newton-Raphson did not converge" */
  INLA_ERR_CANCELLED = 6,      /* "Operation cancelled by user" */
  INLA_ERR_INVALID = 7,        /* invalid argument or pattern */
  INLA_ERR_NOT_FACTORED = 8,   /* "Factorization not computed yet" (solver.rs:78-80) */
  INLA_ERR_CUDA = 9,           /* CUDA runtime error (no device, launch failure) */
  INLA_ERR_INTERNAL = 10
};

/* Fill-reducing ordering selector. INLA_ORDER_REFERENCE restates
 * choose_symmetric_order (crates/inla_math/src/ordering.rs:149-162):
 * time-major Kronecker -> RCM -> AMD (the RCM branch yields a path-like
 * elimination tree with no level parallelism). INLA_ORDER_ND (nested
 * dissection; no reference counterpart) is the default of the batched
 * engines: a shallower elimination tree with fewer pivots on its longest path
 * than INLA_ORDER_AMD.
 * Numeric results do not depend on the ordering beyond rounding. */
enum {
  INLA_ORDER_REFERENCE = 0,
  INLA_ORDER_AMD = 1,
  INLA_ORDER_RCM = 2,
  INLA_ORDER_NATURAL = 3,
  INLA_ORDER_CUSTOM = 4,
  INLA_ORDER_TIME_MAJOR = 5,
  INLA_ORDER_ND = 6
};

/* Last error message of the calling thread ("" if none). */
const char* inla_last_error(void);

/* Number of kernels this library has launched in the calling process. */
int64_t inla_kernel_launches(void);

/* Device memory released by freed handles is kept per device and reused by later
 * handles (creating and freeing handles in a loop then maps no memory); the cache
 * holds at most half of a device's memory and is emptied automatically when an
 * allocation fails. This call returns all cached blocks to the driver (for other
 * users of the GPU in the same process). INLA_NO_MEMORY_CACHE in the environment
 * disables the cache. Symbolic analyses are cached the same way, per exact pattern,
 * ordering, options and permutation (at most 1 GiB of host memory; handles on the
 * same pattern reuse the analysis), and this call empties that cache too, together with the
 * engine tables derived from each cached analysis (panel map, front positions: at most 1 GiB);
 * INLA_NO_SYMBOLIC_CACHE disables both. No reference counterpart. */
int inla_release_cached_memory(void);

/* ------------------------------------------------------------------------
 * Ordering restatement (crates/inla_math/src/ordering.rs:149-162).
 * Writes fwd (old -> new) when a custom branch is taken; returns the branch
 * (INLA_ORDER_TIME_MAJOR, INLA_ORDER_RCM or INLA_ORDER_AMD). Host only.
 * ---------------------------------------------------------------------- */
int inla_choose_symmetric_order(int64_t n, const int64_t* colptr, const int64_t* rowidx, int64_t* fwd);

/* ------------------------------------------------------------------------
 * InlaSolver seam: one solver per thread, holds one factor
 * (trait InlaSolver, crates/inla_math/src/solver.rs:29-44; FaerCpuSolver 48-99).
 * ---------------------------------------------------------------------- */
typedef struct inla_solver inla_solver;

/* FaerCpuSolver::new (solver.rs:54-56). `ordering` is an INLA_ORDER_* value. */
int inla_solver_new(int ordering, inla_solver** out);
void inla_solver_free(inla_solver* s);

/* Use the permutation perm[new] = old (INLA_ORDER_CUSTOM) for the next analysis. */
int inla_solver_set_perm(inla_solver* s, int64_t n, const int64_t* perm);

/* Host-only symbolic analysis of a pattern (the symbolic half of factorize,
 * sparse_ldlt.rs:159-186); needs no GPU. */
int inla_solver_analyze(inla_solver* s, int64_t n, const int64_t* colptr, const int64_t* rowidx);

/* InlaSolver::factorize (solver.rs:31, impl 71-75 -> sparse_ldlt.rs:196-241).
 * Symbolic analysis when the pattern differs from the cached one, numeric only
 * when it matches exactly (scratch.rs:90-103). */
int inla_solver_factorize(inla_solver* s, int64_t n, const int64_t* colptr, const int64_t* rowidx,
                          const double* values);

/* InlaSolver::solve (solver.rs:34, impl 77-85 -> sparse_ldlt.rs:243-265). x may alias rhs. */
int inla_solver_solve(inla_solver* s, const double* rhs, double* x);

/* InlaSolver::diag_inv (solver.rs:40, impl 87-93 -> sparse_ldlt.rs:438-444): Takahashi
 * selected inverse on the filled pattern of L, diag(Q^-1) in original order. */
int inla_solver_diag_inv(inla_solver* s, double* diag);

/* InlaSolver::log_abs_det (solver.rs:43, impl 95-99 -> ldlt.rs:65-67). */
int inla_solver_log_abs_det(const inla_solver* s, double* out);

/* Selected inverse Sigma on the lower entries (row >= col) of the factorized
 * input pattern, in input order (upper entries written as 0). Needed by the
 * adjoint; the reference computes these entries and drops them
 * (sparse_ldlt.rs:376-432). */
int inla_solver_selinv_pattern(inla_solver* s, double* sigma);

/* Symbolic summary of the current factor: info[0]=n, [1]=nnz(L) (true),
 * [2]=stored panel entries, [3]=supernodes, [4]=etree levels, [5]=max front
 * rows, [6]=ordering branch used, [7]=front buffer doubles per problem. */
int inla_solver_info(const inla_solver* s, int64_t* info);
/* perm[new] = old of the current factor (after postordering). */
int inla_solver_perm(const inla_solver* s, int64_t* perm);
/* Column elimination tree (permuted indices, -1 = root) and supernode
 * partition (first column of each supernode, nsuper+1 entries). */
int inla_solver_etree(const inla_solver* s, int64_t* parent);
int inla_solver_supernodes(const inla_solver* s, int64_t* first, int64_t* count);
/* nnz of each column of L incl. the diagonal (permuted order). */
int inla_solver_colcounts(const inla_solver* s, int64_t* counts);

/* ------------------------------------------------------------------------
 * 2-D meshes for SPDE models (crates/inla_fmesher/src/fmesher.rs), host forms.
 * ---------------------------------------------------------------------- */
typedef struct inla_mesh inla_mesh;
/* build_mesh2d (fmesher.rs:119-158, validation 870-893): xy [nv][2], tri [ntri][3] (0-based).
 * INLA_ERR_INVALID with the reference's message for fewer than three vertices, an index out of
 * range, duplicate indices, a near-zero area (|2A| <= 1e-15) or a non-manifold edge. */
int inla_mesh_create(int64_t nv, const double* xy, int64_t ntri, const int64_t* tri, inla_mesh** out);
void inla_mesh_free(inla_mesh* m);
/* nbr [ntri][3]: triangle across the edge opposite vertex e of each triangle, -1 on the boundary. */
int inla_mesh_neighbors(const inla_mesh* m, int64_t* nbr);
/* assemble_fem_blocks_diffusion (fmesher.rs:515-626): lumped mass c0, consistent mass c1,
 * stiffness g1 and boundary term b1, summed per entry in triangle order. triangle_scale [ntri]
 * (NULL = 1; barrier triangles of range fraction f take f^2, fmesher.rs:913-934) multiplies the
 * diffusion tensor diffusion = {hxx, hxy, hyy} (NULL = identity). areas [ntri] may be NULL. */
int inla_mesh_fem(inla_mesh* m, const double* triangle_scale, const double* diffusion, double* areas);
/* One block of the last inla_mesh_fem in CSC: which 0 c0, 1 c1, 2 g1, 3 b1. Call with NULL
 * arrays to read nnz first; colptr has nv + 1 entries. */
int inla_mesh_fem_block(const inla_mesh* m, int which, int64_t* nnz, int64_t* colptr, int64_t* rowidx,
                        double* vals);
/* locate_point (fmesher.rs:161-263): triangle of each point by the walk from triangle 0 (-1
 * outside), bary [npts][3] its barycentric weights (may be NULL). */
int inla_mesh_locate(const inla_mesh* m, int64_t npts, const double* xy, int64_t* tri, double* bary);
/* observation_projector_triplets (fmesher.rs:168-219): A (npts x nv) in CSR, each walk starting
 * from the previous point's triangle, weights with |w| > 1e-15, columns ascending; rowptr
 * [npts + 1], colidx and vals at most 3 npts. INLA_ERR_INVALID for a point outside the mesh. */
int inla_mesh_projector(const inla_mesh* m, int64_t npts, const double* xy, int64_t* rowptr, int64_t* colidx,
                        double* vals);

/* 1-D meshes (crates/inla_fmesher/src/mesh1d.rs): loc [n] strictly increasing finite knots.
 * inla_mesh1d_fem: block `which` (0 c0, 1 c1, 2 g1, 3 b1 = empty) in CSC, nnz first with NULL
 * arrays. inla_mesh1d_projector: A (npts x n) in CSR, rows (1 - w) x_i + w x_{i+1}, locations
 * outside [loc_0, loc_{n-1}] clamped to the end knots; colidx / vals at most 2 npts. */
int inla_mesh1d_fem(int64_t n, const double* loc, int which, int64_t* nnz, int64_t* colptr, int64_t* rowidx,
                    double* vals);
int inla_mesh1d_projector(int64_t n, const double* loc, int64_t npts, const double* s, int64_t* rowptr,
                          int64_t* colidx, double* vals);

/* spde_precision_csc (crates/inla_stats/src/spde.rs:70-140) as the three components of
 * inla_laplace_create on one pattern: Q(theta) = c_0 C0 + c_1 G1 + c_2 G1 C0^-1 G1 with
 * (c_0, c_1, c_2) = tau^2 (kappa^4, 2 kappa^2, 1) (inla_theta_map_spde). c0: the lumped mass
 * diagonal [n]; G1 in CSC with both triangles (e.g. from inla_mesh_fem_block). Call with
 * colptr / rowidx / comp NULL to read nnz; the pattern (diagonal, G1 and G1 C0^-1 G1, rows
 * sorted) goes to colptr [n + 1] / rowidx [nnz], the components to comp [3][nnz].
 * INLA_ERR_INVALID for |c0_i| < 1e-15 ("Zero entry in mass matrix c0 diagonal"). */
int inla_spde_components(int64_t n, const double* c0, const int64_t* g_colptr, const int64_t* g_rowidx,
                         const double* g_vals, int64_t* nnz, int64_t* colptr, int64_t* rowidx, double* comp);

/* ------------------------------------------------------------------------
 * Device forms of the mesh tools, equal bit for bit to the host forms above.
 * The first device call on a mesh builds its patterns and per-entry contribution lists on the
 * host (topology only) and copies the mesh to the current device; later calls must run on that
 * device. Calls on one mesh (or one SPDE plan) must not overlap: they share its scratch.
 * ---------------------------------------------------------------------- */
/* Pattern of FEM block `which` (0 c0, 1 c1, 2 g1, 3 b1) in CSC, the same as inla_mesh_fem_block's
 * after inla_mesh_fem: it depends on the topology only (c1 and g1 share it). Host only; call
 * with NULL arrays to read nnz; colptr has nv + 1 entries. */
int inla_mesh_fem_pattern(inla_mesh* m, int which, int64_t* nnz, int64_t* colptr, int64_t* rowidx);
/* assemble_fem_blocks_diffusion (fmesher.rs:515-626) on the device: the values of c0 / c1 / g1 / b1
 * on inla_mesh_fem_pattern's patterns (device arrays of nnz doubles; any may be NULL) and d_areas
 * [ntri] (may be NULL), queued on `stream` without synchronizing. d_triangle_scale: device
 * [ntri] or NULL (all 1); diffusion: host {hxx, hxy, hyy} or NULL (identity). One thread per
 * entry sums the entry's per-triangle contributions in triangle order with separately rounded
 * operations, so every value equals inla_mesh_fem's. INLA_ERR_INVALID for a non-finite or
 * non-SPD diffusion tensor (the host form's messages). */
int inla_mesh_fem_dev(inla_mesh* m, const double* d_triangle_scale, const double* diffusion, double* d_areas,
                      double* d_c0, double* d_c1, double* d_g1, double* d_b1, void* stream);
/* observation_projector_triplets (fmesher.rs:168-219) on the device: d_xy [npts][2] (device);
 * A in CSR into d_rowptr [npts + 1], d_colidx / d_vals (at most 3 npts each); *nnz (host) the
 * entries written. Each point is located by a walk from a triangle near it; a point inside its
 * triangle by more than rounding can move an edge test keeps that triangle, which every walk
 * reaches, and the others (on or near edges and vertices, or whose walk left the mesh) are
 * located again on the host in point order from the previous point's triangle, as
 * inla_mesh_projector does; the result equals inla_mesh_projector's bit for bit, with the same
 * INLA_ERR_INVALID for the first point outside the mesh. Synchronizes the stream. */
int inla_mesh_projector_dev(inla_mesh* m, int64_t npts, const double* d_xy, int64_t* d_rowptr, int64_t* d_colidx,
                            double* d_vals, int64_t* nnz, void* stream);
/* spde_precision_csc's components (spde.rs:70-140) on the device for a fixed G1 pattern (host
 * CSC, rows strictly ascending in each column, e.g. inla_mesh_fem_pattern(m, 2, ...)).
 * inla_spde_plan_pattern gives the components' pattern, the same as inla_spde_components'
 * (NULL arrays to read nnz). inla_spde_components_dev: d_c0 [n] the lumped mass diagonal and
 * d_g_vals the G1 values on its pattern (device) -> d_comp [3][nnz] (C0, G1, G1 C0^-1 G1), equal
 * to inla_spde_components' bit for bit, queued on `stream`; d_status (device int, may be NULL) is
 * set to 0, or to 1 when some |c0_i| < 1e-15 (the host form's "Zero entry in mass matrix c0
 * diagonal"). */
typedef struct inla_spde_plan inla_spde_plan;
int inla_spde_plan_create(int64_t n, const int64_t* g_colptr, const int64_t* g_rowidx, inla_spde_plan** out);
void inla_spde_plan_free(inla_spde_plan* p);
int inla_spde_plan_pattern(const inla_spde_plan* p, int64_t* nnz, int64_t* colptr, int64_t* rowidx);
int inla_spde_components_dev(inla_spde_plan* p, const double* d_c0, const double* d_g_vals, double* d_comp,
                             int* d_status, void* stream);

/* scale_model_csc (crates/inla_math/src/design.rs:150-195): fac = exp(mean(log d_i)) over the
 * positive finite d = diag(Q^+) (Moore-Penrose inverse), Q_scaled = fac Q. The reference
 * diagonalizes the dense matrix (O(n^3)); here d comes from the sparse LDL^T and selected
 * inverse of the bordered matrix [[Q, U^T], [U, 0]] on the GPU, whose leading block of the
 * inverse is Q^+ when the rows of U span null(Q). k = -1 derives U: one constant row per
 * connected component whose rows sum to ~0 (Besag, rw1, ...); k >= 0 takes the caller's
 * k x n row-major null_basis (rw2: constant and linear trend). Nodes whose column holds no
 * nonzero have d = 0 (left out of the mean, as the reference's zero eigenvalues are). n = 1
 * follows the reference: Q_scaled = [1]. Outputs (each may be NULL): fac; scaled: the values
 * of fac Q in the input pattern; ginv_diag: d [n]. INLA_ERR_INVALID when a basis row is not in
 * the null space (|Q u| > 1e-8 |Q|max |u|max) or no d is positive; INLA_ERR_SINGULAR when U
 * misses part of the null space. */
int inla_scale_model(int64_t n, const int64_t* colptr, const int64_t* rowidx, const double* values, int k,
                     const double* null_basis, int ordering, double* fac, double* scaled, double* ginv_diag);

/* ------------------------------------------------------------------------
 * Batched engine: B problems sharing one symbolic analysis (numeric values
 * differ), factorized / solved / selectively inverted in one launch sequence.
 * ---------------------------------------------------------------------- */
typedef struct inla_batch inla_batch;

int inla_batch_create(int64_t n, const int64_t* colptr, const int64_t* rowidx, int ordering, int max_batch,
                      inla_batch** out);
void inla_batch_free(inla_batch* h);
/* values: [B][nnz] in input-pattern order. logdet, status: [B]. */
int inla_batch_factorize(inla_batch* h, int B, const double* values, double* logdet, int* status);
/* rhs, x: [B][n] (x may alias rhs). */
int inla_batch_solve(inla_batch* h, int B, const double* rhs, double* x);
/* diag: [B][n]. */
int inla_batch_diag_inv(inla_batch* h, int B, double* diag);
/* sigma: [B][nnz] (see inla_solver_selinv_pattern). */
int inla_batch_selinv_pattern(inla_batch* h, int B, double* sigma);

/* Device-pointer variants, ordered on `stream` (a cudaStream_t; NULL = the
 * legacy default stream): the work starts after everything already queued on
 * `stream` and later work queued on `stream` waits for it. The calls do not
 * synchronize the host. Inputs/outputs live in device memory. */
int inla_batch_factorize_dev(inla_batch* h, int B, const double* d_values, double* d_logdet, int* d_status,
                             void* stream);
/* Schedule of the numeric factorization (no reference counterpart; the reference runs faer's
 * factorization per theta-point): *persistent = 1 when the handle factorizes every front of
 * every batch member in ONE persistent launch (a task queue in elimination-tree order with
 * bounded dependency waits), 0 when it launches the kernels level by level (fronts too wide
 * for the persistent kernel's shared memory, or INLA_NO_PERSIST set). Results are the same
 * bit for bit; *persistent = 1 means the schedule is available (with mode 1 each batch size
 * then uses the faster of the two). A persistent launch whose dependency wait ran out (2 s; INLA_PERSIST_WAIT_MS)
 * ends early and the call that synchronizes after it returns INLA_ERR_CUDA (status bit 4 in
 * the _dev status words). */
int inla_batch_schedule(inla_batch* h, int* persistent);
/* Host-only check of the persistent schedule of a solver's symbolic analysis (after
 * inla_solver_analyze; no device use): walking the task queue in order, every task's
 * dependencies are complete when it is reached and every front ends complete.
 * info3 = {tasks per problem, shared memory bytes, 1 if the schedule fits}. INLA_ERR_INTERNAL
 * with the first violation otherwise. */
int inla_solver_check_schedule(const inla_solver* s, int64_t* info3);
/* Process-wide choice for engines (solver, batch, Laplace, many-model handles) created after
 * the call: 0 the level launches; 1 (default) measured per batch size -- on its first
 * factorization at a batch size an engine times both schedules and keeps the faster for that
 * structure and size; 2 the persistent schedule wherever it fits. */
int inla_set_persistent_schedule(int mode);
/* Process-wide panel form of the level launches for engines created after the call: -1
 * (default) the autotuner's per-level choice (on the first factorization at a batch size the
 * level sequence is timed in each form and every level keeps the fastest); 0 split (diagonal
 * block, rows, trailing update: three launches per 64-column step); 1 fused (every row CTA
 * factors the diagonal block: two launches); 2 look-ahead (rows, then the trailing update
 * whose first tile also factors the next diagonal block: two launches). All forms give
 * bit-identical factors. */
int inla_set_panel_form(int form);
/* Diagnostic of the bounded waits: runs the persistent factorization once with completion
 * counts that can never be reached and a wait limit of limit_ms, and returns in *code what
 * the launch recorded (1: a wait ran out and the launch ended). The handle stays usable;
 * factorize again before solving. */
int inla_batch_wait_limit_selftest(inla_batch* h, double limit_ms, int* code);
int inla_batch_solve_dev(inla_batch* h, int B, double* d_x, void* stream);
int inla_batch_diag_inv_dev(inla_batch* h, int B, double* d_diag, void* stream);
int inla_batch_selinv_pattern_dev(inla_batch* h, int B, double* d_sigma, void* stream);

/* ------------------------------------------------------------------------
 * Laplace engine: find_latent_mode_a_with_solver (crates/inla_stats/src/
 * inference.rs:776-975) for B theta-points at once. The latent precision is
 * a linear combination of fixed-pattern components,
 *   Q(theta_b) = sum_t coef[b][t] * comp[t]      (value refresh, no re-assembly),
 * on a full symmetric pattern that must contain A^T A and the diagonal.
 * A is the n_obs x n projector in CSR (a_rowptr == NULL: identity, eta = x).
 * family: 0 gaussian/identity (p1 = precision), 1 poisson/log (p1 = exposure),
 * 2 binomial/logit (p1 = trials), 3 negative binomial/log (p1 = size,
 * p2 = exposure) (inference.rs:170-311). p1 is multiplied by p1scale[b].
 * ---------------------------------------------------------------------- */
typedef struct inla_laplace inla_laplace;

/* INLA_LAP_NO_PRIOR_SHARING: evaluate every member's prior on its own. By default
 * members whose prior coefficient vectors are proportional (c_b = s c_r, s > 0)
 * share one prior factorization and selected inverse (log|Q_b| = log|Q_r| +
 * n log s, tr(Q_b^-1 M_t) = tr(Q_r^-1 M_t) / s; the 1e-12 log-det jitter then acts
 * as 1e-12 / s on the member). No reference counterpart (the reference
 * evaluates one theta-point at a time). */
enum { INLA_LAP_VARIANCES = 1, INLA_LAP_GRADIENT = 2, INLA_LAP_NO_PRIOR_SHARING = 8 };

int inla_laplace_create(int64_t n, const int64_t* colptr, const int64_t* rowidx, int ncomp, const double* comp,
                        int64_t nobs, const int64_t* a_rowptr, const int64_t* a_colidx, const double* a_vals,
                        int family, const double* y, const double* p1, const double* p2, int ordering,
                        int max_batch, inla_laplace** out);
void inla_laplace_free(inla_laplace* h);
/* Hard linear constraints C x = e for every later evaluation and fit: the
 * Augmented method of find_latent_mode_a_with_solver (inference.rs:804-830,
 * 867-869, 902-904, 949-951; constraints.rs:268-353). The working prior is
 * Q + kappa C^T C with kappa = 3.059023205018258e6 (HARD_CONSTRAINT_KAPPA); the
 * prior log-determinant is log|Q + kappa C^T C| without the 1e-12 jitter;
 * Newton trial points and the mode are projected onto C x = e. c: [k][n]
 * row-major dense (ConstraintSpec.a), e: [k] (ConstraintSpec.e); k = 0 removes
 * the constraints. Both methods below give the reference's results; they
 * differ in how Q + kappa C^T C is held (a new symbolic analysis either way):
 *  INLA_CONSTR_AUGMENTED: as the reference, kappa C^T C added on the pattern
 *    widened by its support (sum over rows of nnz(row)^2 <= 2^26 entries);
 *  INLA_CONSTR_BORDERED (no reference counterpart): the sparse bordered matrix
 *    [[Q, C^T], [C, -I/kappa]] of order n + k, whose Schur complement is
 *    Q + kappa C^T C, so no constrained block densifies;
 *  INLA_CONSTR_AUTO: augmented up to 2^22 added entries, else bordered.
 * Limits: k <= 1024, at most 7 model components. INLA_ERR_INVALID for a singular
 * C C^T (pivot below 1e-14, constraints.rs:369-371); the previous constraints
 * then stay. */
enum { INLA_CONSTR_AUTO = 0, INLA_CONSTR_AUGMENTED = 1, INLA_CONSTR_BORDERED = 2 };
int inla_laplace_set_constraints(inla_laplace* h, int k, const double* c, const double* e, int method);
/* scalars: [B][8] = {mlik, log|Q+1e-12 I|, log|Q_post|, loglik, x'Qx, newton iterations,
 * status (0 ok, 1 singular prior, 2 singular posterior, 3 invalid likelihood, 4 non-finite
 * step, 5 not converged), d loglik / d log p1scale}. x, var: [B][n] or NULL (modes and
 * Takahashi marginal variances). grad_terms: [B][4][ncomp+1] or NULL = {tr(S_prior M_t),
 * tr(S_post M_t) + [tr(S_post A^T W A)], x'M_t x, z'M_t x (implicit GLM term)}. */
int inla_laplace_eval(inla_laplace* h, int B, const double* coef, const double* p1scale, int flags,
                      double* scalars, double* x, double* var, double* grad_terms);

/* ------------------------------------------------------------------------
 * Independent models of uneven size in one engine (no reference counterpart:
 * the reference fits each model on its own). G models are given as one
 * block-diagonal latent field: model g owns latent nodes [lat_off[g],
 * lat_off[g+1]) and observations [obs_off[g], obs_off[g+1]); the pattern,
 * components and the projector A (CSR) must not couple models. One symbolic
 * analysis (an elimination forest with one tree per model, each model's block
 * ordered on its own) serves every evaluation; each level launch works on the
 * fronts of all models. Per theta-set and model the evaluation is
 * find_latent_mode_a_with_solver (inference.rs:776-975) with that model's
 * coefficients and family scale.
 * ---------------------------------------------------------------------- */
typedef struct inla_multi inla_multi;
int inla_multi_create(int G, const int64_t* lat_off, const int64_t* obs_off, const int64_t* colptr,
                      const int64_t* rowidx, int ncomp, const double* comp, const int64_t* a_rowptr,
                      const int64_t* a_colidx, const double* a_vals, int family, const double* y, const double* p1,
                      const double* p2, int ordering, int max_batch, inla_multi** out);
void inla_multi_free(inla_multi* h);
/* coef: [B][G][ncomp]; p1scale: [B][G] or NULL; scalars: [B][G][8] (layout of
 * inla_laplace_eval); x, var: [B][n] or NULL; grad_terms: [B][G][4][ncomp+1] or NULL. */
int inla_multi_eval(inla_multi* h, int B, const double* coef, const double* p1scale, int flags, double* scalars,
                    double* x, double* var, double* grad_terms);

/* Fit of every model (run_inla_inference_a_cancellable, inference.rs:1116-1466, per
 * model), all models in lockstep: per model the batched Newton mode search on adjoint
 * gradients of inla_fit (mode_search 2), the Hessian (hessian 0: the reference's FD of
 * values with h = max(1e-4, 0.05 max|theta_g|); 1: central FD of adjoint gradients),
 * CCD nodes with f0 and the per-model mixture moments. Batch b of every evaluation holds
 * point b of every model. map/prior get the model index g. theta0, mode: [G][m];
 * hessian: [G][m][m]; mlik, mode_iters, status: [G] (status 0 ok, 1 no finite CCD node,
 * 2 singular Hessian); latent_mean, latent_var: [n]; info: [3] = {seconds, batches,
 * model evaluations}. */
typedef int (*inla_multi_theta_map_fn)(int g, const double* theta, int m, double* coef, double* dcoef,
                                       double* p1scale, double* dp1scale, void* user);
typedef double (*inla_multi_log_prior_fn)(int g, const double* theta, int m, double* grad, void* user);
/* Cancellation poll (the check_cancel callback of run_inla_inference_a_cancellable,
 * inference.rs:1116-1130): called before every batched evaluation; a nonzero return stops the
 * fit, which returns INLA_ERR_CANCELLED ("Operation cancelled by user") and leaves its outputs
 * unwritten. */
typedef int (*inla_cancel_fn)(void* cancel_user);
typedef struct {
  int hessian;    /* 0 FD of values (reference), 1 FD of adjoint gradients */
  double f0;      /* CCD f0 (0 = 1.0) */
  int max_iter;   /* Newton iterations per model (0 = 100) */
  double tol;     /* gradient infinity-norm tolerance (0 = 1e-4) */
  inla_cancel_fn cancel; /* NULL: never cancelled */
  void* cancel_user;
} inla_multi_fit_options;
int inla_multi_fit(inla_multi* h, int m, const double* theta0, inla_multi_theta_map_fn map,
                   inla_multi_log_prior_fn prior, void* user, const inla_multi_fit_options* opt, double* mode,
                   double* hessian, double* mlik, double* latent_mean, double* latent_var, int* mode_iters,
                   int* status, double* info);
/* Linear predictor of the last inla_multi_fit: per model the mixture mean and variance of
 * eta = A x over that model's CCD nodes (inference.rs:1451-1466), [nobs] each (NULL allowed). */
int inla_multi_fit_predictor(inla_multi* h, double* pred_mean, double* pred_var);
/* Model-selection criteria of model g of the last inla_multi_fit (as inla_fit_model_selection for a
 * single model: the model's observations at its mode, its node weights, D(theta*) at the node
 * with the smallest |z|; crit[6] from its own Hessian). cpo, pit: that model's [nobs_g]
 * observations. INLA_ERR_NONCONVERGED for a model without a finite node. */
int inla_multi_fit_model_selection(inla_multi* h, int g, int what, double* crit, double* cpo, double* pit);
/* Built-in map of AR1 + iid + intercept models: theta = [log tau, logit-type rho, log tau_iid],
 * components [intercept precision, AR1 pieces K0, K1, K2, iid] with coefficients
 * [1, tau, tau rho^2, -tau rho, tau_iid] (ar1.rs:9-69, structured.rs:348-356). */
int inla_multi_theta_map_ar1_iid(int g, const double* theta, int m, double* coef, double* dcoef, double* p1scale,
                                 double* dp1scale, void* user);
/* One prior stack (user = inla_prior_set*) for every model. */
double inla_multi_log_prior_set(int g, const double* theta, int m, double* grad, void* user);

/* ------------------------------------------------------------------------
 * Hyperpriors (crates/inla_stats/src/priors.rs): log pi(theta) and gradient.
 * ---------------------------------------------------------------------- */
enum {
  INLA_PRIOR_PC_PREC = 1,   /* p = {u, alpha}: priors.rs:532-548 */
  INLA_PRIOR_LOGGAMMA = 2,  /* p = {shape, rate}: priors.rs:836-855 */
  INLA_PRIOR_PC_SPDE = 3,   /* p = {r0, alpha_r, s0, alpha_s}, slots (log tau, log kappa): priors.rs:127-147,813-834 */
  INLA_PRIOR_GAUSSIAN = 4,  /* p = {mean, precision} */
  INLA_PRIOR_PC_COR1 = 5    /* p = {u, alpha}, theta = logit-type ((1 + rho) / 2): priors.rs:611-704 */
};
typedef struct {
  int kind;
  int slot;
  double p[4];
} inla_prior_spec;
double inla_prior_log_density(const inla_prior_spec* specs, int nspec, const double* theta, int m, double* grad);

/* A prior stack usable directly as the inla_fit prior callback (user = inla_prior_set*). */
typedef struct {
  int nspec;
  inla_prior_spec specs[8];
} inla_prior_set;
double inla_log_prior_set(const double* theta, int m, double* grad, void* user);

/* ------------------------------------------------------------------------
 * INLA fit: run_inla_inference_a_cancellable (inference.rs:1116-1466).
 * map(theta) gives coef[ncomp], dcoef[m][ncomp], p1scale, dp1scale[m]
 * (the build_prior / build_obs callbacks of the reference, as value
 * refreshes); prior(theta) gives log pi(theta) and its gradient.
 * ---------------------------------------------------------------------- */
typedef int (*inla_theta_map_fn)(const double* theta, int m, double* coef, double* dcoef, double* p1scale,
                                 double* dp1scale, void* user);
typedef double (*inla_log_prior_fn)(const double* theta, int m, double* grad, void* user);

typedef struct {
  int mode_search; /* 0 Nelder-Mead on values (reference), 1 BFGS on adjoint gradients,
                      2 batched Newton (adjoint gradients + central FD-of-gradient Hessians, 2m + 1 points
                      per batch), 3 the same with forward differences (m + 1 points per batch) */
  int batched;     /* 0 one theta-point per evaluation (plain drop-in), 1 batched theta-sets */
  int strategy;    /* 0 CCD, 1 grid (m <= 2; CCD f0 = 2.5 above) */
  double f0;       /* CCD f0 / grid step (0 = 1.0) */
  int hessian;     /* 0 FD of log-posterior values (reference stencil), 1 FD of adjoint gradients */
  int max_iter;    /* 0 = 200 (NM) / 100 (BFGS) */
  double tol;      /* 0 = 1e-6 (NM f-spread) / 1e-4 (BFGS gradient inf-norm) */
  double nm_step;  /* 0 = 0.1 */
  inla_cancel_fn cancel; /* polled before every evaluation (NULL: never cancelled) */
  void* cancel_user;
} inla_fit_options;

/* node_theta: up to [64][m]; node_weight: up to [64]; info: [6] = {mlik, seconds,
 * theta-evaluations, batches, mode-search iterations, integration nodes}.
 * m = 0 (no hyperparameters, inference.rs:1135-1239): one Laplace evaluation at the empty
 * theta with marginal variances, no mode search, Hessian or integration design; mlik is the
 * Laplace marginal likelihood (no prior term), info[5] = 0 integration nodes (node_theta and
 * node_weight are not written), the predictor, model selection and marginals of the fit use
 * that single node with weight 1, and a failed Laplace evaluation is an error. theta0, mode
 * and hessian may be NULL then. */
int inla_fit(inla_laplace* h, int m, const double* theta0, inla_theta_map_fn map, inla_log_prior_fn prior,
             void* user, const inla_fit_options* opt, double* mode, double* hessian, double* latent_mean,
             double* latent_var, double* node_theta, double* node_weight, double* info);

/* Linear predictor of the last inla_fit on h: mixture mean and variance of eta = A x
 * (predictor_means / predictor_variances of the reference's result, inference.rs:1451-1466),
 * length nobs each (either pointer may be NULL). INLA_ERR_INVALID before the first fit. */
int inla_fit_predictor(inla_laplace* h, double* pred_mean, double* pred_var);
/* Wall seconds of the phases of the last inla_fit on h (no reference counterpart): out4 =
 * {mode search, Hessian, integration design + node evaluations, aggregation}; they add up to
 * info[1] of inla_fit up to the host bookkeeping between them. */
int inla_fit_phase_seconds(inla_laplace* h, double* out4);

/* Model-selection criteria of the last inla_fit on h, as the reference computes them at the
 * end of a fit (inference.rs:1470-1514; model_selection.rs): DIC (compute_dic, 101-150) and
 * WAIC (compute_waic, 152-211) from the per-node predictors, CPO / PIT (compute_cpo_pit,
 * 222-325, with the failure heuristic check_cpo_failure_for_obs, 327-396) from the predictors
 * and their variances, all with the observations rebuilt at the mode (the theta map's p1 scale
 * there) and D(theta*) at the node with the smallest |z|. what: INLA_MS_* bits (criteria not
 * asked for are NaN). crit: [8] = {DIC, mean deviance, DIC effective parameters, WAIC, lppd,
 * WAIC effective parameters, Gaussian-approximation log marginal likelihood
 * (compute_marginal_log_lik_gaussian, model_selection.rs:25-73; NaN when -H is not positive
 * definite), CPO failures}; cpo, pit: [nobs], NaN where the reference gives None (either may be
 * NULL). INLA_ERR_INVALID (with the reference's message) where the reference returns an error:
 * a likelihood that cannot be evaluated, a non-finite WAIC predictive density. */
enum { INLA_MS_DIC = 1, INLA_MS_WAIC = 2, INLA_MS_CPO = 4, INLA_MS_ALL = 7 };
int inla_fit_model_selection(inla_laplace* h, int what, double* crit, double* cpo, double* pit);

/* Posterior precision at the mode (posterior_precision_at, inference.rs:1027-1058, as the
 * reference's result carries it, 1565-1570): Q(theta*) [+ kappa C^T C with constraints] +
 * A^T W A, W = -d2 log p(y | eta) at eta = A x of the node nearest the mode, with the
 * observations as given to inla_laplace_create. CSC on the model's pattern united with the
 * entries the likelihood and constraint terms add; call with NULL arrays to read nnz first
 * (colptr has n + 1 entries). */
int inla_fit_posterior_precision(inla_laplace* h, int64_t* nnz, int64_t* colptr, int64_t* rowidx, double* vals);
/* Host-only form: Q = sum_t coef_t comp_t on the given pattern, A (NULL = identity), the
 * observations, the latent point x [n] and kc x n constraint rows c (kc = 0: none). */
int inla_posterior_precision(int64_t n, const int64_t* colptr, const int64_t* rowidx, int ncomp, const double* comp,
                             const double* coef, int64_t nobs, const int64_t* a_rowptr, const int64_t* a_colidx,
                             const double* a_vals, int family, const double* y, const double* p1, const double* p2,
                             const double* x, int kc, const double* c, int64_t* nnz, int64_t* colptr_out,
                             int64_t* rowidx_out, double* vals);

/* Marginal densities of the last inla_fit on h on a uniform grid (marginals.rs): kind 0 the
 * latent entry `index`, 1 the predictor entry `index` (gaussian_mixture_marginal over the nodes,
 * 73-135), 2 the hyperparameter `index` on the internal scale (hyperpar_marginal_from_nodes,
 * 137-162). x, y: [n_points] (n_points >= 5); the grid spans mean +- max(n_sd, 1) sd and y has
 * unit trapezoid mass. The reference's defaults are 201 points and n_sd = 4. */
int inla_fit_marginal(inla_laplace* h, int kind, int64_t index, int n_points, double n_sd, double* x, double* y);
/* Host-only forms: a mixture from the caller's node means / variances / weights, a hyperparameter
 * kernel density from node values, and quantiles of a gridded density (marginal_quantiles,
 * marginals.rs:202-226; probabilities in (0, 1)). */
int inla_mixture_marginal(int K, const double* means, const double* vars, const double* weights, int n_points,
                          double n_sd, double* x, double* y);
int inla_hyperpar_marginal(int K, const double* theta, const double* weights, int n_points, double n_sd, double* x,
                           double* y);
int inla_marginal_quantiles(int n, const double* x, const double* y, int np, const double* probs, double* q);

/* Host-only: the same criteria from a caller's node results (crit[6] is NaN). family: as in
 * inla_laplace_create (0 gaussian, 1 poisson, 2 binomial, 3 negative binomial); y, p1, p2: [nobs] (p1 gaussian precision / poisson exposure / binomial trials /
 * nb size, p2 nb exposure; NULL = 1); weight: [K] normalised; mode_index: the node of D(theta*);
 * cond_eta, cond_eta_var: [K][nobs]. */
int inla_model_selection(int family, int64_t nobs, const double* y, const double* p1, const double* p2, int K,
                         const double* weight, int mode_index, const double* cond_eta, const double* cond_eta_var,
                         int what, double* crit, double* cpo, double* pit);
/* Device forms of the two entry points above: every array is a device pointer, the work is
 * queued on `stream` (NULL = default stream). inla_predictor_moments_dev also returns the
 * per-node predictor d_cond_eta / d_cond_eta_var [K][nobs] (A in CSR with int64 row pointers
 * and int32 column indices; d_a_rowptr NULL means eta = x, nobs = n); it does not
 * synchronize. inla_model_selection_dev takes the node weights on the host, synchronizes the
 * stream and writes crit / cpo / pit on the host; its sums over observations use a fixed
 * reduction order (identical run to run, equal to the host form to rounding). The predictor
 * moments equal the host form bit for bit. */
int inla_predictor_moments_dev(int64_t nobs, int64_t n, const int64_t* d_a_rowptr, const int* d_a_colidx,
                               const double* d_a_vals, int K, const double* d_weight, const double* d_cond_mean,
                               const double* d_cond_var, double* d_cond_eta, double* d_cond_eta_var,
                               double* d_pred_mean, double* d_pred_var, void* stream);
int inla_model_selection_dev(int family, int64_t nobs, const double* d_y, const double* d_p1, const double* d_p2,
                             int K, const double* weight, int mode_index, const double* d_cond_eta,
                             const double* d_cond_eta_var, int what, double* crit, double* cpo, double* pit,
                             void* stream);
/* compute_marginal_log_lik_gaussian (model_selection.rs:25-73): log_post_mode + m/2 log(2 pi)
 * - 1/2 log det(neg_hessian), neg_hessian row-major m x m; INLA_ERR_NOT_PD when it is not
 * positive definite. */
int inla_mlik_gaussian(double log_post_mode, int m, const double* neg_hessian, double* out);
/* observation_cdf (model_selection.rs:398-448): F(y | eta, variance) of one observation;
 * INLA_ERR_INVALID where the reference gives None (negative binomial, invalid rate), and for a
 * non-finite y or a count above 1e15 (whose term-by-term CDF sum the reference would loop over). */
int inla_observation_cdf(int family, double y, double p1, double eta, double variance, double* out);
/* check_cpo_failure_for_obs (model_selection.rs:327-396): 1 when the CPO of this observation is
 * flagged unreliable at posterior mean mu and variance var of its predictor, else 0. */
int inla_cpo_failure(int family, double y, double p1, double p2, double mu, double var);

/* Host-only mixture of the linear predictor over K integration nodes (no device use):
 * per node eta_k = A x_k (matvec_csc, design.rs:52-70: columns with x_kj = 0 skipped) and
 * eta-var_k = sum_j A_ij^2 var_kj (predictor_variances_diag, design.rs:198-210), then
 * mean = sum_k w_k eta_k and var = sum_k w_k (eta-var_k + (eta_k - mean)^2)
 * (inference.rs:1451-1466). A is nobs x n in CSR, each row summed in stored order
 * (ascending columns give the reference's order); a_rowptr NULL means eta = x (nobs = n).
 * weight: [K] normalised node weights; cond_mean, cond_var: [K][n]; pred_*: [nobs]. */
int inla_predictor_moments(int64_t nobs, int64_t n, const int64_t* a_rowptr, const int64_t* a_colidx,
                           const double* a_vals, int K, const double* weight, const double* cond_mean,
                           const double* cond_var, double* pred_mean, double* pred_var);

/* ------------------------------------------------------------------------
 * Dense LDL^T + log|Q| + solve that allocates no device memory.
 * No counterpart in the reference: it exists for host programs that embed
 * this library but must own every device allocation themselves (pool
 * allocators, framework plugins handed pre-sized buffers, code where a
 * cudaMalloc/cudaFree would synchronize the device or is not allowed while
 * other work is captured or scheduled). All pointers are caller-owned device
 * memory: d_q is the n x n matrix (column-major, both triangles; the lower
 * one is read), d_rhs / d_x are length n (both NULL to skip the solve),
 * d_logdet / d_status receive log|Q| and the pivot status (0 ok, nonzero =
 * singular or non-finite pivot). Work is queued on `stream` (NULL = default
 * stream) without synchronizing. Limit: n <= 1024 (larger n returns
 * INLA_ERR_DIM_MISMATCH). The factor lives in a fixed 8 MiB static device
 * scratch per GPU, shared by every call and kept until process exit: calls
 * whose GPU work overlaps race on it (calls queued on one stream run in
 * order and do not). The first call on a device resolves the scratch
 * addresses; make it before any stream capture (a first call on a capturing
 * stream returns INLA_ERR_INVALID).
 * ---------------------------------------------------------------------- */
int inla_dense_ldlt_solve_noalloc(int n, const double* d_q, const double* d_rhs, double* d_x, double* d_logdet,
                                  int* d_status, void* stream);

/* Built-in theta map of the SPDE Gaussian model: theta = [log prec_eps, log tau, log kappa],
 * components [C~, G, G C~^-1 G] (crates/inla_stats/src/spde.rs:70-140). */
int inla_theta_map_spde(const double* theta, int m, double* coef, double* dcoef, double* p1scale,
                        double* dp1scale, void* user);

#ifdef __cplusplus
}
#endif

#endif /* INLA_B200_H */
