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
 * time-major Kronecker -> RCM -> AMD. INLA_ORDER_AMD is the GPU default:
 * the RCM branch yields a path-like elimination tree with no level
 * parallelism. Numeric results do not depend on the ordering beyond rounding. */
enum {
  INLA_ORDER_REFERENCE = 0,
  INLA_ORDER_AMD = 1,
  INLA_ORDER_RCM = 2,
  INLA_ORDER_NATURAL = 3,
  INLA_ORDER_CUSTOM = 4,
  INLA_ORDER_TIME_MAJOR = 5
};

/* Last error message of the calling thread ("" if none). */
const char* inla_last_error(void);

/* Number of kernels this library has launched in the calling process. */
int64_t inla_kernel_launches(void);

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
 * handle's own stream). Inputs/outputs live in device memory. */
int inla_batch_factorize_dev(inla_batch* h, int B, const double* d_values, double* d_logdet, int* d_status,
                             void* stream);
int inla_batch_solve_dev(inla_batch* h, int B, double* d_x, void* stream);
int inla_batch_diag_inv_dev(inla_batch* h, int B, double* d_diag, void* stream);
int inla_batch_selinv_pattern_dev(inla_batch* h, int B, double* d_sigma, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* INLA_B200_H */
