"""GPU parity of hard linear constraints (the reference's Augmented method,
find_latent_mode_a_with_solver with constraints, inference.rs:804-951), held
either as the reference holds it (kappa C^T C on a widened pattern) or as the
sparse bordered matrix [[Q, C^T], [C, -I/kappa]].

The Poisson Besag GLMM with a sum-to-zero constraint on the region block
(30 x 30 rook lattice, scale.model, fixed effects first) and the binomial
Besag x AR1 group model with one sum-to-zero row per time (downscaled to
8 x 8 x 6, where the oracle's dense augmentation is computable) are compared
per theta-point with the oracle: log-determinants 1e-10 relative, mlik 1e-10 of
|log|Q_post||, modes and marginal variances 1e-8 relative, equal Newton
iteration counts, C x* = e to 1e-12. The full fit (Nelder-Mead + grid
integration) is compared with the oracle's restatement on a 10 x 10 lattice;
the adjoint gradient of the group model with central differences of the
oracle; the full-size group model (n = 200 001, 40 constraint rows, which the
dense augmentation cannot hold) runs bordered and is checked for feasibility.
"""
import math

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from inla_b200 import models
from inla_b200.laplace import PRIOR_PC_PREC, LaplaceModel

pytestmark = pytest.mark.gpu

RT_LD = 1e-10
RT_X = 1e-8


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300)


def besag_model(nr, nc, max_batch=4, method="auto"):
    p = models.make_besag_problem(nr=nr, nc=nc)
    lm = LaplaceModel(p.model, a=p.a, family="poisson", y=p.y, max_batch=max_batch)
    lm.set_constraints(*p.constraint, method=method)
    return p, lm


def check_against_oracle(p, lm, coefs, e=None, family="poisson", **kw):
    c = p.constraint[0]
    e = p.constraint[1] if e is None else e
    out = lm.eval(coefs, variances=True)
    assert np.all(out["status"] == 0), out["status"]
    for b in range(len(coefs)):
        r = O.laplace(p.model.matrix(coefs[b]), p.a, family, p.y, constraints=(c, e), want_var=True, **kw)
        assert out["iters"][b] == r["iters"]
        assert abs(out["logdet_prior"][b] - r["logdet_prior"]) <= RT_LD * abs(r["logdet_prior"])
        assert abs(out["logdet_post"][b] - r["logdet_post"]) <= RT_LD * abs(r["logdet_post"])
        assert abs(out["mlik"][b] - r["mlik"]) <= RT_LD * abs(r["logdet_post"])
        assert rel(out["x"][b], r["x"]) < RT_X
        assert rel(out["var"][b], r["var"]) < RT_X
        assert np.max(np.abs(c @ out["x"][b] - e)) < 1e-12


def besag_coefs(log_taus):
    return np.stack([models.besag_coefs(t)[0] for t in log_taus])


@pytest.mark.parametrize("method", ["augmented", "bordered"])
def test_constrained_besag_poisson_matches_oracle(method):
    p, lm = besag_model(30, 30, method=method)
    check_against_oracle(p, lm, besag_coefs([-1.0, 0.7]))


@pytest.mark.parametrize("method", ["augmented", "bordered"])
def test_nonzero_rhs(method):
    p, lm = besag_model(8, 8, method=method)
    e = np.array([0.4])
    lm.set_constraints(p.constraint[0], e, method=method)
    check_against_oracle(p, lm, besag_coefs([0.2, 1.1]), e=e)


def test_removal_restores_the_unconstrained_engine():
    p, lm = besag_model(8, 8)
    # removing the constraints gives exactly the unconstrained engine
    lm.set_constraints(None)
    fresh = LaplaceModel(p.model, a=p.a, family="poisson", y=p.y, max_batch=4)
    coefs = models.besag_coefs(1.0)[0][None]
    a, b = lm.eval(coefs, variances=True), fresh.eval(coefs, variances=True)
    assert a["mlik"][0] == b["mlik"][0]
    np.testing.assert_array_equal(a["x"], b["x"])
    # unconstrained, the intrinsic prior's log|Q + 1e-12 I| rests on a pivot of ~1e-12 that
    # rounding moves by ~1e-3 relative, so only the posterior side is compared
    r = O.laplace(p.model.matrix(coefs[0]), p.a, "poisson", p.y)
    assert a["iters"][0] == r["iters"]
    assert abs(a["logdet_post"][0] - r["logdet_post"]) <= RT_LD * abs(r["logdet_post"])
    assert rel(a["x"][0], r["x"]) < RT_X


def test_singular_constraint_rows_are_rejected():
    p, lm = besag_model(6, 6)
    c = np.vstack([p.constraint[0], p.constraint[0]])
    with pytest.raises(Exception, match="singular"):
        lm.set_constraints(c, np.zeros(2))
    # the previous constraints stay in force
    out = lm.eval(models.besag_coefs(0.5)[0][None])
    assert out["status"][0] == 0
    assert abs(p.constraint[0] @ out["x"][0]) < 1e-12


def test_rw1_hard_sum_to_zero_holds():
    """inference.rs:2533-2594: RW1 (n = 8) + intercept, Gaussian observations with
    precision 4, hard sum-to-zero on the RW1 block, CCD: the posterior means of the RW1
    block sum to ~0 and the marginal likelihood is finite."""
    n = 8
    y = (np.arange(n) - 3.5) * 0.3
    adj = sp.diags([np.ones(n - 1), np.ones(n - 1)], [-1, 1])
    r = models.besag_structure(adj)
    m0 = sp.block_diag([r, sp.csc_matrix((1, 1))]).tocsc()
    m1 = sp.diags(np.r_[np.zeros(n), 1e-4]).tocsc()
    a = sp.hstack([sp.identity(n), np.ones((n, 1))]).tocsr()
    model = models.build_latent(n + 1, [m0, m1], "rw1", extra_pattern=[(a.T @ a).tocsc()])
    lm = LaplaceModel(model, a=a, family="gaussian", y=y, p1=4.0, max_batch=8)
    c, e = models.sum_to_zero_constraint(n, 1)
    lm.set_constraints(models.embed_constraint(c, n + 1, 0), e)

    def theta_map(t):
        tau = math.exp(t[0])
        return np.array([tau, 1.0]), np.array([[tau, 0.0]]), 1.0, np.array([0.0])

    res = lm.fit(np.array([0.0]), theta_map=theta_map, priors=lambda t: (-0.05 * t[0] ** 2, [-0.1 * t[0]]),
                 mode_search="nm", batched=False, strategy="ccd", f0=1.0)
    assert abs(res["mean"][:n].sum()) < 1e-4
    assert math.isfinite(res["mlik"])


def test_besag_grid_fit_matches_oracle():
    """Nelder-Mead path, FD Hessian and grid integration (step 1) of the Besag GLMM on a
    10 x 10 lattice against the oracle's restatement."""
    p, lm = besag_model(10, 10, max_batch=16)
    c, e = p.constraint

    def theta_map(t):
        coef, dcoef = models.besag_coefs(t[0])
        return coef, dcoef, 1.0, np.array([0.0])

    prior = [(PRIOR_PC_PREC, 0, (1.0, 0.01))]
    res = lm.fit(np.array([0.0]), theta_map=theta_map, priors=prior, mode_search="nm", batched=False,
                 strategy="grid", f0=1.0)

    def laplace(t):
        return O.laplace(p.model.matrix(models.besag_coefs(t[0])[0]), p.a, "poisson", p.y, constraints=(c, e),
                         want_var=True)

    def f(t):
        try:
            return -(laplace(t)["mlik"] + O.pc_prec_log_dens(t[0], 1.0, 0.01))
        except O.OracleError:
            return 1e12

    mode_ref = O.nelder_mead([0.0], 0.1, 200, 1e-6, f)
    np.testing.assert_allclose(res["mode"], mode_ref, atol=1e-6)
    h = max(1e-4, 0.05 * abs(mode_ref[0]))
    np.testing.assert_allclose(res["hessian"], O.fd_hessian(mode_ref, f, h), rtol=1e-5, atol=1e-6)

    def node(t):
        r = laplace(t)
        return r["x"], r["var"], r["mlik"] + O.pc_prec_log_dens(t[0], 1.0, 0.01)

    ref = O.integrate(res["mode"], res["hessian"], node, f0=1.0, strategy="grid")
    np.testing.assert_allclose(np.sort(res["node_theta"].ravel()), np.sort(ref["thetas"].ravel()), atol=1e-8)
    assert rel(res["mean"], ref["mean"]) < RT_X
    assert rel(res["var"], ref["var"]) < RT_X
    assert abs(res["mlik"] - ref["mlik"]) < RT_X * abs(ref["mlik"])
    assert abs(c @ res["mean"] - e).max() < 1e-12


GROUP_THETAS = [np.array([0.0, 0.0, 2.2, 1.4]), np.array([0.3, -0.2, 1.5, 1.0])]


@pytest.mark.parametrize("method", ["augmented", "bordered"])
def test_group_model_matches_oracle(method):
    """Besag 8 x 8 (x) AR1 T = 6 + iid + intercept, binomial(10), sum-to-zero per time."""
    p = models.make_group_problem(nr=8, nc=8, T=6)
    lm = LaplaceModel(p.model, a=p.a, family="binomial", y=p.y, p1=p.ntrials, max_batch=4)
    lm.set_constraints(*p.constraint, method=method)
    coefs = np.stack([models.group_coefs(t)[0] for t in GROUP_THETAS])
    check_against_oracle(p, lm, coefs, family="binomial", p1=p.ntrials)


def test_group_model_adjoint_vs_central_fd():
    """d mlik / d theta of the constrained group model (bordered) against central differences
    (step 1e-4) of the oracle's mlik, Newton tolerance 1e-10 on the oracle side."""
    p = models.make_group_problem(nr=6, nc=6, T=4)
    lm = LaplaceModel(p.model, a=p.a, family="binomial", y=p.y, p1=p.ntrials, max_batch=2)
    lm.set_constraints(*p.constraint, method="bordered")
    t = np.array([0.2, -0.1, 1.8, 1.2])
    c, dc = models.group_coefs(t)
    out = lm.eval(c[None], gradient=True)
    T = len(c)
    g = dc @ (0.5 * out["trP"][0, :T] - 0.5 * out["trQ"][0, :T] - 0.5 * out["xMx"][0, :T] + 0.5 * out["zMx"][0, :T])

    def mlik(tt):
        q = p.model.matrix(models.group_coefs(tt)[0])
        return O.laplace(q, p.a, "binomial", p.y, p1=p.ntrials, constraints=p.constraint, tol=1e-10)["mlik"]

    h = 1e-4
    fd = np.array([(mlik(t + h * e) - mlik(t - h * e)) / (2 * h) for e in np.eye(4)])
    assert np.max(np.abs(g - fd)) <= 2e-3 * max(1.0, np.max(np.abs(fd))), (g, fd)


def test_group_model_full_size_bordered():
    """Besag 50 x 50 (x) AR1 T = 40 + iid + intercept (n = 200 001, 40 constraint rows):
    the dense augmentation would add 2.5e8 entries; bordered it evaluates with variances and
    gradient pieces, and every mode satisfies its constraints."""
    p = models.make_group_problem()
    lm = LaplaceModel(p.model, a=p.a, family="binomial", y=p.y, p1=p.ntrials, max_batch=2)
    with pytest.raises(Exception, match="2\\^26"):
        lm.set_constraints(*p.constraint, method="augmented")
    lm.set_constraints(*p.constraint)  # auto -> bordered
    coefs = np.stack([models.group_coefs(t)[0] for t in GROUP_THETAS])
    out = lm.eval(coefs, variances=True, gradient=True)
    assert np.all(out["status"] == 0), out["status"]
    c, e = p.constraint
    for b in range(2):
        assert np.max(np.abs(c @ out["x"][b] - e)) < 1e-10
        assert np.all(out["var"][b] > 0) and np.all(np.isfinite(out["var"][b]))
        assert np.isfinite(out["mlik"][b]) and np.all(np.isfinite(out["trP"][b]))
    single = lm.eval(coefs[1:], variances=True)
    assert abs(single["mlik"][0] - out["mlik"][1]) <= 1e-12 * abs(out["logdet_post"][1])
