"""Posterior precision at the mode (host code of the library, no GPU): posterior_precision_at
(inference.rs:1027-1058) through inla_posterior_precision against a scipy restatement of
Q [+ kappa C^T C] + A^T W A with W from the oracle's likelihoods."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from inla_b200 import InlaError, models
from inla_b200.laplace import posterior_precision

KAPPA = 3.059023205018258e6


def restated(model, coef, x, a, family, y, p1=None, p2=None, c=None):
    q = model.matrix(coef).toarray()
    eta = x if a is None else a @ x
    n_obs = len(y)
    p1 = np.ones(n_obs) if p1 is None else np.broadcast_to(p1, (n_obs,))
    p2 = np.ones(n_obs) if p2 is None else np.broadcast_to(p2, (n_obs,))
    w = np.array([-O.eval_lik(family, eta[i], y[i], p1[i], p2[i])[2] for i in range(n_obs)])
    at = np.eye(len(x)) if a is None else a.toarray()
    q = q + at.T @ (w[:, None] * at)
    if c is not None:
        c = np.atleast_2d(c)
        q = q + KAPPA * c.T @ c
    return q


def test_spde_gaussian_with_projector():
    p = models.make_spde_problem(nx=12, n_obs=80, seed=3)
    coef, _ = models.spde_coefs(-0.5, 1.1)
    x = np.random.default_rng(1).normal(size=p.model.n)
    got = posterior_precision(p.model, coef, x, a=p.a, family="gaussian", y=p.y, p1=7.5).toarray()
    ref = restated(p.model, coef, x, p.a, "gaussian", p.y, p1=7.5)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    assert np.allclose(got, got.T, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_poisson_identity_projector_newton_step_case():
    """ldlt.rs:487-502: Q = I, every observation with Fisher weight 1.2 on the diagonal."""
    n = 4
    model = models.build_latent(n, [sp.identity(n, format="csc")], "iid")
    lam = 1.2
    x = np.full(n, np.log(lam))
    got = posterior_precision(model, [1.0], x, a=None, family="poisson", y=np.ones(n)).toarray()
    np.testing.assert_allclose(got, np.eye(n) * (1.0 + lam), rtol=1e-14)


def test_besag_with_sum_to_zero_constraint():
    b = models.make_besag_problem(nr=6, nc=5, seed=4)
    coef = models.besag_coefs(0.7)[0]
    x = np.random.default_rng(2).normal(scale=0.3, size=b.model.n)
    c, _ = b.constraint
    got = posterior_precision(b.model, coef, x, a=b.a, family="poisson", y=b.y, c=c).toarray()
    ref = restated(b.model, coef, x, b.a, "poisson", b.y, c=c)
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_invalid_observation_is_an_error():
    n = 3
    model = models.build_latent(n, [sp.identity(n, format="csc")], "iid")
    with pytest.raises(InlaError, match="likelihood"):
        posterior_precision(model, [1.0], np.zeros(n), a=None, family="poisson", y=[-1.0, 0.0, 1.0])


class _DenseSolver:
    """A dense stand-in for the GPU solver, to test the lincomb bookkeeping on the CPU."""

    def factorize(self, q):
        self.q = q.toarray()

    def solve(self, b):
        return np.linalg.solve(self.q, b)


def test_lincomb_summaries_bookkeeping():
    """posterior.rs:55-92: mean, sd and the Gaussian quantiles; duplicate indices add up."""
    from inla_b200.laplace import lincomb_summaries

    rng = np.random.default_rng(6)
    b = rng.normal(size=(5, 5))
    q = sp.csc_matrix(b @ b.T + 5 * np.eye(5))
    mean = rng.normal(size=5)
    combs = [("first", [(0, 1.0)]), ("diff", [(1, 1.0), (3, -1.0), (1, 0.5)])]
    res = lincomb_summaries(mean, q, combs, solver=_DenseSolver())
    cov = np.linalg.inv(q.toarray())
    a = np.array([0.0, 1.5, 0.0, -1.0, 0.0])
    assert res[0]["mean"] == mean[0] and abs(res[0]["sd"] - np.sqrt(cov[0, 0])) < 1e-12
    assert abs(res[1]["mean"] - a @ mean) < 1e-14 and abs(res[1]["sd"] - np.sqrt(a @ cov @ a)) < 1e-12
    assert abs(res[1]["q975"] - res[1]["mean"] - 1.96 * res[1]["sd"]) < 1e-14
    with pytest.raises(ValueError, match="out of range"):
        lincomb_summaries(mean, q, [("bad", [(9, 1.0)])], solver=_DenseSolver())
