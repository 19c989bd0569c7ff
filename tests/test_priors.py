"""Hyperprior densities of the library's host code (inla_prior_log_density, no GPU) and of
the oracle, pinned on the reference's prior tests (crates/inla_stats/src/priors.rs:950-1114)."""
import math

import numpy as np

import oracle as O
from inla_b200.laplace import PRIOR_GAUSSIAN, PRIOR_LOGGAMMA, PRIOR_PC_PREC, PRIOR_PC_SPDE, log_prior, prior_set


def lib_prior(specs, theta):
    return log_prior(prior_set(specs), np.asarray(theta, dtype=float))


def test_pc_prec_matches_closed_form():
    """priors.rs:950-966: u = 1, alpha = 0.01, theta = 0.5 (1e-12); gradient vs central FD (1e-5)."""
    lam = -math.log(0.01) / 1.0
    theta = 0.5
    expect = math.log(lam) - math.log(2.0) - lam * math.exp(-0.5 * theta) - 0.5 * theta
    v, g = lib_prior([(PRIOR_PC_PREC, 0, (1.0, 0.01))], [theta])
    assert abs(v - expect) < 1e-12
    assert abs(O.pc_prec_log_dens(theta, 1.0, 0.01) - expect) < 1e-12
    eps = 1e-6
    fd = (lib_prior([(PRIOR_PC_PREC, 0, (1.0, 0.01))], [theta + eps])[0]
          - lib_prior([(PRIOR_PC_PREC, 0, (1.0, 0.01))], [theta - eps])[0]) / (2 * eps)
    assert abs(g[0] - fd) < 1e-5


def test_pc_spde_mapping_from_theta():
    """priors.rs:1078-1093: pc.spde(r0 = 50, alpha_r = 0.05, s0 = 2, alpha_s = 0.01) at
    (log tau, log kappa) = (0, 0) equals the closed form on (log rho, log sigma) (1e-12)."""
    log_rho = 0.5 * math.log(8.0)
    log_sigma = -0.5 * math.log(4.0 * math.pi)
    lam1 = -math.log(0.05) * 50.0
    lam2 = -math.log(0.01) / 2.0
    expect = (math.log(lam1) - log_rho - lam1 * math.exp(-log_rho)) + (
        math.log(lam2) + log_sigma - lam2 * math.exp(log_sigma))
    v, _ = lib_prior([(PRIOR_PC_SPDE, 0, (50.0, 0.05, 2.0, 0.01))], [0.0, 0.0])
    assert abs(v - expect) < 1e-12
    assert abs(O.pc_spde_log_dens(0.0, 0.0, 50.0, 0.05, 2.0, 0.01) - expect) < 1e-12


def test_loggamma_rate_convention():
    """priors.rs:1096-1105: shape 3, rate 0.5 at theta = 0; gradient shape - rate."""
    expect = 3.0 * math.log(0.5) - math.lgamma(3.0) + 0.0 - 0.5
    v, g = lib_prior([(PRIOR_LOGGAMMA, 0, (3.0, 0.5))], [0.0])
    assert abs(v - expect) < 1e-12
    assert abs(g[0] - 2.5) < 1e-12
    assert abs(O.loggamma_log_dens(0.0, 3.0, 0.5) - expect) < 1e-12


def test_gaussian_prior_gradient():
    """priors.rs:1108-1113: N(0, precision 4) at 0.2 has gradient -0.8."""
    _, g = lib_prior([(PRIOR_GAUSSIAN, 0, (0.0, 4.0))], [0.2])
    assert abs(g[0] + 0.8) < 1e-12


def test_prior_stack_sums_slots():
    """A stack adds the densities and gradients of its members, each on its own slots."""
    specs = [(PRIOR_PC_PREC, 0, (1.0, 0.01)), (PRIOR_PC_SPDE, 1, (1.0, 0.05, 1.0, 0.01))]
    th = [0.3, -1.2, 2.1]
    v, g = lib_prior(specs, th)
    v0, g0 = lib_prior(specs[:1], th[:1])
    v1, g1 = lib_prior([(PRIOR_PC_SPDE, 0, (1.0, 0.05, 1.0, 0.01))], th[1:])
    assert abs(v - (v0 + v1)) < 1e-12
    np.testing.assert_allclose(g, np.r_[g0, g1], atol=1e-14)
