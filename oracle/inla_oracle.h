/*
 * CPU ORACLE — test infrastructure only. A plain-C restatement of
 * rust-inla's INLA inner path, used by tests/ (to check the library) and by
 * bench.py's cpu_baseline / --impl reference leg (as the timed CPU path).
 * It is never linked into, called by or shipped with the product library.
 *
 * Pinning: the reference (Rust + faer 0.24, unvendored) cannot be built in
 * this environment, so this oracle is pinned against the reference's own
 * known-answer tests for the path (sparse vs dense LDL^T / Takahashi on the
 * AR1, Besag and tridiagonal fixtures of sparse_ldlt.rs:613-665 and
 * ldlt.rs:522-544, the identity solver test solver.rs:106-121, the
 * Gaussian-identity mode = linear solve test inference.rs:2845-2929) and
 * against dense numpy references; see tests/test_oracle.py.
 */
#ifndef INLA_ORACLE_H
#define INLA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- ordering.rs restatement ---- */
int64_t orc_lower_bandwidth(int64_t n, const int64_t* cp, const int64_t* ri);
int64_t orc_bandwidth_with_fwd(int64_t n, const int64_t* cp, const int64_t* ri, const int64_t* fwd);
int orc_try_time_major(int64_t n, const int64_t* cp, const int64_t* ri, int64_t* fwd);
void orc_rcm(int64_t n, const int64_t* cp, const int64_t* ri, int64_t* fwd);
/* 5 = time-major, 2 = RCM (fwd written), 1 = AMD */
int orc_choose_order(int64_t n, const int64_t* cp, const int64_t* ri, int64_t* fwd);
/* Minimum-degree order for the AMD branch (perm[new] = old); not faer's AMD. */
void orc_min_degree(int64_t n, const int64_t* cp, const int64_t* ri, int64_t* perm);

/* ---- sparse LDL^T (simplicial, up-looking) ---- */
typedef struct orc_factor orc_factor;
/* perm[new] = old (NULL = natural). Returns 0, or 1 when a pivot is tiny /
 * non-finite (sparse_ldlt.rs:117-120). Only entries with row >= col are read. */
int orc_factor_create(int64_t n, const int64_t* cp, const int64_t* ri, const double* vals, const int64_t* perm,
                      orc_factor** out);
/* The same factor by a supernodal LDL^T (dense panels, left-looking over the supernodal tree), equal to
 * orc_factor_create's to rounding; the CPU baseline's factorization. */
int orc_factor_create_sn(int64_t n, const int64_t* cp, const int64_t* ri, const double* vals, const int64_t* perm,
                         orc_factor** out);
/* 1: the Laplace functions below factorize with orc_factor_create_sn (set before any thread
 * uses the oracle); 0 (default): with orc_factor_create, the form the parity tests pin. */
void orc_set_supernodal(int on);
/* OpenMP threads inside one supernodal factorization (default 1). */
void orc_set_threads(int t);
void orc_factor_free(orc_factor* f);
int64_t orc_factor_nnz(const orc_factor* f);
double orc_logdet(const orc_factor* f);                      /* ldlt.rs:65-67, sequential */
void orc_solve(const orc_factor* f, const double* b, double* x);
/* Takahashi selected inverse (sparse_ldlt.rs:376-432): diag in original order. */
int orc_takahashi_diag(const orc_factor* f, double* diag);
/* Sigma at the lower entries of a pattern (0 for upper entries). */
int orc_takahashi_pattern(const orc_factor* f, const int64_t* cp, const int64_t* ri, double* out);

/* ---- likelihoods (inference.rs:170-311) ----
 * family 0 gaussian/identity (p1 = precision), 1 poisson/log (p1 = exposure),
 * 2 binomial/logit (p1 = trials), 3 negative binomial/log (p1 = size, p2 = exposure) */
int orc_eval_lik(int family, double eta, double y, double p1, double p2, double* logp, double* grad,
                 double* hess);
double orc_log_gamma(double z);

/* ---- Laplace mode (inference.rs:776-975) ----
 * Q: full symmetric CSC; A: CSR n_obs x n (acp == NULL => identity);
 * constraints: kc rows of dense cA (kc x n) and ce (kc), kc = 0 for none. */
/* constraints.rs:316-353: x <- x - C^T (C C^T)^-1 (C x - e); nonzero when C C^T is singular. */
int orc_project_constraints(int64_t n, double* x, int kc, const double* cA, const double* ce);
int orc_laplace(int64_t n, const int64_t* qcp, const int64_t* qri, const double* qv, int64_t nobs,
                const int64_t* acp, const int64_t* aci, const double* av, int family, const double* y,
                const double* p1, const double* p2, int kc, const double* cA, const double* ce, int max_iter,
                double tol, const int64_t* perm, double* x_out, double* out4 /* mlik, ldprior, ldpost, iters */,
                double* var_out /* optional diag(Q_post^-1) */);

#ifdef __cplusplus
}
#endif
#endif
