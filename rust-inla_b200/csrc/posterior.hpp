// Posterior precision at the mode, host code: Q_post = Q(theta) [+ kappa C^T C] + A^T W A with
// W = -d2 log p(y | eta) at eta = A x.
//
// Reference: crates/inla_stats/src/inference.rs:1027-1058 (posterior_precision_at, called at
// 1565-1570 with the prior at the mode, the observations as passed in and the latent mode of the
// node nearest the mode), crates/inla_math/src/ldlt.rs:373-453 (laplace_newton_system_a),
// design.rs:94-139 (at_diag_a: rows with d = 0 or non-finite d and zero products are skipped;
// add_csc), constraints.rs:275-313 (kappa C^T C).
#pragma once
#include <cstdint>
#include <string>

#include "mesh.hpp"  // CscBlock

namespace inla {

// Pattern: the input pattern united with the entries A^T W A and kappa C^T C add; values summed
// per entry as Q first, then the likelihood terms in observation order, then the constraint
// terms. acp == nullptr: A = I (nobs == n). C: kc x n row-major (kc = 0: none).
std::string posterior_precision(int64_t n, const int64_t* cp, const int64_t* ri, int ncomp, const double* comp,
                                const double* coef, int64_t nobs, const int64_t* acp, const int64_t* aci,
                                const double* av, int family, const double* y, const double* p1, const double* p2,
                                const double* x, int kc, const double* c, CscBlock& out);

}  // namespace inla
