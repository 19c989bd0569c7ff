"""Hard linear constraints on the CPU: the oracle's projection and augmentation pinned
on the reference's own tests (crates/inla_math/src/constraints.rs:391-461,
crates/inla_stats/src/inference.rs:2533-2594), and the constraint / scale.model
input generators."""
import math

import numpy as np
import scipy.sparse as sp

import oracle as O
from inla_b200 import models

KAPPA = 3.059023205018258e6  # HARD_CONSTRAINT_KAPPA, constraints.rs:268


def test_kappa_is_the_reference_literal():
    """The reference's comment calls the constant exp(15); its value (used here, as parity
    requires) is 3.059023205018258e6, while exp(15) = 3.269e6."""
    assert KAPPA == 3.059023205018258e6
    assert abs(KAPPA - math.exp(15.0)) > 1e5


def test_sum_to_zero_projects():
    """constraints.rs:395-402"""
    c, e = models.sum_to_zero_constraint(5, 1)
    x = O.project_constraints([1.0, 2.0, 3.0, 4.0, 5.0], c, e)
    assert abs(x.sum()) < 1e-10


def test_rw2_constraints_kill_constant_and_linear():
    """constraints.rs:404-418"""
    c, e = models.sum_to_zero_constraint(6, 2)
    x = O.project_constraints(2.0 + 0.5 * np.arange(6), c, e)
    assert abs(x.sum()) < 1e-9
    assert abs(np.sum((np.arange(6) - 2.5) * x)) < 1e-9


def test_augment_makes_identity_stiffer():
    """constraints.rs:420-429: Q = I_4 plus kappa A^T A with A = 1/2 (1,1,1,1) has the
    diagonal 1 + kappa/4 and the eigenvalues {1, 1, 1, 1 + kappa}; the oracle's constrained
    prior log-determinant (no jitter, inference.rs:838-840) is therefore log(1 + kappa)."""
    c, e = models.sum_to_zero_constraint(4, 1)
    q = sp.identity(4, format="csc")
    r = O.laplace(q, None, "gaussian", np.zeros(4), p1=1.0, constraints=(c, e))
    assert abs(r["logdet_prior"] - math.log1p(KAPPA)) <= 1e-10 * math.log1p(KAPPA)
    dense = np.eye(4) + KAPPA * c.T @ c
    assert abs(dense[0, 0] - (1.0 + KAPPA / 4.0)) < 1e-6


def test_plane_2d_kills_const_row_col_trends():
    """constraints.rs:431-460"""
    nrow, ncol = 4, 5
    c, e = models.plane_constraint_2d(nrow, ncol)
    assert c.shape == (3, nrow * ncol)
    x = np.zeros(nrow * ncol)
    for j in range(ncol):
        for i in range(nrow):
            x[j * nrow + i] = 1.0 + 0.3 * i + 0.7 * j
    x = O.project_constraints(x, c, e)
    ii = np.tile(np.arange(nrow), ncol) - (nrow - 1) / 2.0
    jj = np.repeat(np.arange(ncol), nrow) - (ncol - 1) / 2.0
    assert abs(x.sum()) < 1e-9
    assert abs(np.sum(ii * x)) < 1e-9
    assert abs(np.sum(jj * x)) < 1e-9


def test_embed_places_block():
    c, _ = models.sum_to_zero_constraint(3, 1)
    full = models.embed_constraint(c, 6, 2)
    assert full.shape == (1, 6)
    np.testing.assert_array_equal(full[0, :2], 0.0)
    np.testing.assert_array_equal(full[0, 5:], 0.0)
    np.testing.assert_allclose(full[0, 2:5], 1 / math.sqrt(3))


def test_scale_model_geometric_mean_is_one():
    """design.rs:140-149: after scaling, the generalized-inverse marginal variances have
    geometric mean 1."""
    r = models.besag_structure(models.lattice_adjacency(6, 7))
    rs, fac = models.scale_model(r)
    assert fac > 0
    g = np.diag(np.linalg.pinv(rs.toarray()))
    assert abs(math.exp(np.mean(np.log(g))) - 1.0) < 1e-10


def test_besag_problem_layout():
    p = models.make_besag_problem(nr=8, nc=9)
    n = 8 * 9 + 2
    assert p.model.n == n and p.a.shape == (72, n)
    c, e = p.constraint
    assert c.shape == (1, n) and np.all(c[0, :2] == 0.0)
    assert abs(c[0] @ np.r_[0.0, 0.0, p.truth["u"]]) < 1e-10  # the sampled field sums to zero
    q = p.model.matrix(models.besag_coefs(0.3)[0])
    np.testing.assert_allclose(q.diagonal()[:2], models.BESAG_FIXED_PREC)
    a = p.a.toarray()
    np.testing.assert_array_equal(a[:, 0], 1.0)
    np.testing.assert_array_equal(a[:, 2:], np.eye(72))


def test_constrained_oracle_mode_is_feasible():
    """The oracle's constrained Poisson mode satisfies C x = e (projection after the last
    Newton step, inference.rs:949-951), also for e != 0."""
    p = models.make_besag_problem(nr=6, nc=6)
    c, _ = p.constraint
    q = p.model.matrix(models.besag_coefs(0.5)[0])
    for e in (np.zeros(1), np.array([0.4])):
        r = O.laplace(q, p.a, "poisson", p.y, constraints=(c, e))
        assert abs(c[0] @ r["x"] - e[0]) < 1e-12
        assert np.isfinite(r["mlik"])


def test_oracle_grid_design_walks_until_threshold():
    """integration.rs:64-102 for m = 1: centre, +k steps, then -k steps while the drop
    from the centre is at most the threshold; weights 1."""
    f = lambda z: -0.5 * z[0] ** 2
    z, w = O.grid_design(1, 1.0, 4.0, f)
    np.testing.assert_array_equal(z.ravel(), [0.0, 1.0, 2.0, -1.0, -2.0])
    np.testing.assert_array_equal(w, 1.0)
    z2, _ = O.grid_design(2, 1.0, 4.0, lambda z: -(z[0] ** 2 + z[1] ** 2))
    assert len(z2) == 13  # the 5 x 5 square minus the 12 points with |z|^2 > 4


def test_pc_prior_goldens():
    """priors.rs:982-1032: pc.cor1(0.5, 0.75) at theta = 0 is -2.381562305990987 (1e-8), its
    analytic gradient agrees with central differences (1e-5); pc.prec(1, 0.01) at 0 is
    log(lam) - log 2 - lam (1e-14). Oracle restatement and the library's host code."""
    from inla_b200.laplace import PRIOR_PC_COR1, PRIOR_PC_PREC, log_prior, prior_set

    assert abs(O.pc_cor1_log_dens(0.0, 0.5, 0.75) - (-2.381562305990987)) < 1e-8
    ps = prior_set([(PRIOR_PC_COR1, 0, (0.5, 0.75))])
    v, _ = log_prior(ps, [0.0])
    assert abs(v - (-2.381562305990987)) < 1e-8
    for th in (0.4, -1.2, 2.5):
        v, g = log_prior(ps, [th])
        assert abs(v - O.pc_cor1_log_dens(th, 0.5, 0.75)) < 1e-12
        eps = 1e-6
        fd = (log_prior(ps, [th + eps])[0] - log_prior(ps, [th - eps])[0]) / (2 * eps)
        assert abs(g[0] - fd) < 1e-5 * max(1.0, abs(fd))
    lam = -math.log(0.01)
    v, _ = log_prior(prior_set([(PRIOR_PC_PREC, 0, (1.0, 0.01))]), [0.0])
    assert abs(v - (math.log(lam) - math.log(2.0) - lam)) < 1e-14


def test_group_problem_layout():
    """Group-major latent order with the spatial index fastest (structured.rs:527-528), one
    sum-to-zero row per time slice that the sampled field satisfies, A = [1 | I | I]."""
    p = models.make_group_problem(nr=4, nc=5, T=3)
    ns, T = p.dims
    n = 1 + 2 * ns * T
    assert p.model.n == n and p.a.shape == (ns * T, n)
    c, e = p.constraint
    assert c.shape == (T, n)
    assert np.max(np.abs(c @ np.r_[0.0, p.truth["u"].ravel(), p.truth["w"]])) < 1e-10
    np.testing.assert_allclose(c @ c.T, np.eye(T), atol=1e-15)
    coef, dcoef = models.group_coefs([0.1, -0.2, 1.3, 0.7])
    q = p.model.matrix(coef).toarray()
    r = models.besag_structure(models.lattice_adjacency(4, 5)).toarray()
    rho = 2.0 / (1.0 + math.exp(-1.3)) - 1.0
    ar = models.ar1_precision(T, rho, math.exp(0.1 - 0.2)).toarray()
    np.testing.assert_allclose(q[1:1 + ns * T, 1:1 + ns * T], np.kron(ar, r), rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(np.diag(q)[1 + ns * T:], math.exp(0.7))
    h = 1e-6
    for i in range(4):
        d = np.zeros(4)
        d[i] = h
        fd = (models.group_coefs(np.array([0.1, -0.2, 1.3, 0.7]) + d)[0]
              - models.group_coefs(np.array([0.1, -0.2, 1.3, 0.7]) - d)[0]) / (2 * h)
        np.testing.assert_allclose(dcoef[i], fd, rtol=1e-7, atol=1e-9)


def test_multi_problem_layout():
    """Independent AR1 + iid + intercept models of uneven size: latent [intercept, AR1,
    iid], A = [1 | I | I], sizes log-uniform in [n_lo, n_hi), coefficient derivatives."""
    p = models.make_multi_problem(G=6, n_lo=20, n_hi=60, seed=3)
    assert len(p.models) == len(p.a) == len(p.y) == 6
    for m, a, y, nk in zip(p.models, p.a, p.y, p.truth["n"]):
        assert 20 <= nk < 60 and m.n == 2 * nk + 1 and a.shape == (nk, m.n) and len(y) == nk
        d = a.toarray()
        np.testing.assert_array_equal(d[:, 0], 1.0)
        np.testing.assert_array_equal(d[:, 1:1 + nk], np.eye(nk))
        np.testing.assert_array_equal(d[:, 1 + nk:], np.eye(nk))
    th = np.array([0.3, 1.1, 2.0])
    c, dc = models.ar1_iid_coefs(th)
    q = p.models[0].matrix(c).toarray()
    nk = p.truth["n"][0]
    rho = 2.0 / (1.0 + math.exp(-1.1)) - 1.0
    np.testing.assert_allclose(q[1:1 + nk, 1:1 + nk], models.ar1_precision(nk, rho, math.exp(0.3)).toarray(),
                               rtol=1e-14, atol=1e-14)
    for i in range(3):
        e = np.zeros(3)
        e[i] = 1e-6
        fd = (models.ar1_iid_coefs(th + e)[0] - models.ar1_iid_coefs(th - e)[0]) / 2e-6
        np.testing.assert_allclose(dc[i], fd, rtol=1e-7, atol=1e-9)


def test_group_block_is_group_major_kronecker():
    """structured.rs grouped_iid_ar1_uses_group_major_kronecker_order: the grouped block of Q is
    kron(Q_group, Q_main) with Q_group the AR1 precision (ar1.rs:9-69: tau at the ends,
    tau (1 + rho^2) inside, -tau rho off the diagonal) and rho = 2 / (1 + e^-theta) - 1."""
    p = models.make_group_problem(nr=3, nc=4, T=3, seed=2)
    theta = [0.2, -0.1, 0.6, 0.3]
    c, _ = models.group_coefs(theta)
    q = p.model.matrix(c).toarray()
    ns, T = p.dims
    rho = 2.0 / (1.0 + np.exp(-theta[2])) - 1.0
    q_group = models.ar1_precision(T, rho, np.exp(theta[1])).toarray()
    assert q_group[0, 0] == np.exp(theta[1]) and q_group[0, 1] == -np.exp(theta[1]) * rho
    r = models.besag_structure(models.lattice_adjacency(3, 4)).toarray()
    expected = np.kron(q_group, np.exp(theta[0]) * r)
    block = q[1:1 + ns * T, 1:1 + ns * T]
    np.testing.assert_allclose(block, expected, rtol=1e-14, atol=1e-14)
    assert q[0, 0] == models.BESAG_FIXED_PREC
    np.testing.assert_allclose(np.diag(q)[1 + ns * T:], np.exp(theta[3]), rtol=1e-15)


def test_besag_precision_reference_cases():
    """besag.rs:177-196 (4-cycle, tau = 1.5: diagonal 3.0, neighbour -1.5, others 0) and
    besag.rs:199-206 (a singleton region gets the diagonal tau)."""
    cyc = sp.csr_matrix(np.array([[0, 1, 0, 1], [1, 0, 1, 0], [0, 1, 0, 1], [1, 0, 1, 0]], dtype=float))
    q = 1.5 * models.besag_structure(cyc).toarray()
    assert abs(q[0, 0] - 3.0) < 1e-12 and abs(q[0, 1] + 1.5) < 1e-12 and abs(q[0, 2]) < 1e-12
    adj = np.zeros((6, 6))
    for i, j in [(0, 1), (1, 2), (3, 4)]:
        adj[i, j] = adj[j, i] = 1.0
    q = 2.0 * models.besag_structure(sp.csr_matrix(adj)).toarray()
    assert q[5, 5] == 2.0 and q[0, 0] == 2.0 and q[1, 1] == 4.0


def test_besag_constraints_follow_connected_components():
    """structured.rs besag_constraints_follow_connected_components: components {0,1,2}, {3,4},
    {5}; two rows, the singleton unconstrained."""
    adj = np.zeros((6, 6))
    for i, j in [(0, 1), (1, 2), (3, 4)]:
        adj[i, j] = adj[j, i] = 1.0
    c, e = models.component_constraints(sp.csr_matrix(adj))
    assert c.shape == (2, 6) and np.all(e == 0.0)
    assert c[0, 5] == 0.0 and c[1, 5] == 0.0
    assert np.all(c[0, :3] > 0) and np.all(c[1, 3:5] > 0)
    np.testing.assert_allclose(c[0, :3], 1 / np.sqrt(3)) and np.testing.assert_allclose(c[1, 3:5], 1 / np.sqrt(2))
    assert models.component_constraints(sp.csr_matrix((3, 3))) is None
