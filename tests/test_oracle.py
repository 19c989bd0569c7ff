"""Pin the CPU oracle against the reference's own known-answer tests.

Each test restates a reference test (file:line) with the same inputs and
tolerance, plus checks against the committed dense golden vectors.
"""
import math
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from fixtures import (KNOWN_ANSWER, identity, mixture_major_fgn_like, mixture_major_path_cliques,
                      tridiagonal8)

GOLDEN = np.load(Path(__file__).parent / "golden" / "golden.npz")


def golden_cases():
    names = sorted({k.split("/")[0] for k in GOLDEN.files})
    return names


def golden_matrix(name):
    n = len(GOLDEN[f"{name}/indptr"]) - 1
    return sp.csc_matrix((GOLDEN[f"{name}/data"], GOLDEN[f"{name}/indices"], GOLDEN[f"{name}/indptr"]), shape=(n, n))


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_matches_dense_golden(name):
    q = golden_matrix(name)
    f = O.Factor(q, perm=O.default_perm(q))
    assert not f.singular
    assert abs(f.logdet() - GOLDEN[f"{name}/logdet"][0]) <= 1e-10 * max(1.0, abs(GOLDEN[f"{name}/logdet"][0]))
    b = np.arange(1, q.shape[0] + 1, dtype=float)
    np.testing.assert_allclose(f.solve(b), GOLDEN[f"{name}/solve"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(f.diag_inv(), GOLDEN[f"{name}/diag_inv"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", list(KNOWN_ANSWER))
def test_takahashi_vs_dense_tolerances(name):
    """sparse_ldlt.rs:640-665: Takahashi diag within the test's own tolerance of dense."""
    mk, tol = KNOWN_ANSWER[name]
    q = mk()
    dense = np.diag(np.linalg.inv(q.toarray()))
    for perm in (None, O.default_perm(q), np.arange(q.shape[0])[::-1].copy()):
        f = O.Factor(q, perm=perm)
        assert np.max(np.abs(f.diag_inv() - dense)) < tol


def test_identity_solver():
    """solver.rs:106-121."""
    f = O.Factor(identity(3, 2.0))
    np.testing.assert_array_equal(f.solve([2.0, 4.0, 6.0]), [1.0, 2.0, 3.0])
    np.testing.assert_array_equal(f.diag_inv(), [0.5, 0.5, 0.5])
    assert abs(f.logdet() - 3 * math.log(2.0)) < 1e-10


def test_tridiagonal_logdet_and_solve():
    """ldlt.rs:522-544: sparse vs dense log-det and solve within 1e-9."""
    q = tridiagonal8()
    f = O.Factor(q)
    sign, ld = np.linalg.slogdet(q.toarray())
    assert abs(f.logdet() - ld) < 1e-9
    b = np.arange(1, 9, dtype=float)
    np.testing.assert_allclose(f.solve(b), np.linalg.solve(q.toarray(), b), atol=1e-9)


def test_fgn_like_factor_is_sparse():
    """sparse_ldlt.rs:549-570: nnz(L) < n^2/8 for the 64x5 FGN-like matrix."""
    q = mixture_major_fgn_like(64, 5)
    n = q.shape[0]
    f = O.Factor(q, perm=O.default_perm(q))
    assert f.nnz() < n * n / 8
    assert np.all(np.isfinite(f.solve(np.ones(n))))


def test_time_major_cuts_envelope():
    """ordering.rs:191-204."""
    q = mixture_major_path_cliques(64, 5)
    assert O.lower_bandwidth(q) >= 63
    kind, fwd = O.choose_order(q)
    assert kind == 5
    n, cp, ri = q.shape[0], q.indptr.astype(np.int64), q.indices.astype(np.int64)
    bw = 0
    for c in range(n):
        for p in range(cp[c], cp[c + 1]):
            bw = max(bw, abs(int(fwd[ri[p]]) - int(fwd[c])))
    assert bw <= 2 * 5


def test_likelihood_derivatives():
    """inference.rs:170-311: grad/hess vs closed forms (1e-12) and finite differences."""
    # gaussian: grad = -prec (eta - y), hess = -prec
    lp, g, h = O.eval_lik("gaussian", 0.3, 1.1, 4.0)
    assert abs(g - (-4.0 * (0.3 - 1.1))) < 1e-12 and abs(h + 4.0) < 1e-12
    assert abs(lp - (-0.9189385332046728 + 0.5 * math.log(4.0) - 0.5 * 4.0 * 0.8 ** 2)) < 1e-12
    # poisson: grad = y - E e^eta, Fisher hess = -E e^eta
    lp, g, h = O.eval_lik("poisson", 0.4, 3.0, 2.0)
    mu = 2.0 * math.exp(0.4)
    assert abs(g - (3.0 - mu)) < 1e-12 and abs(h + mu) < 1e-12
    assert abs(lp - (3.0 * math.log(mu) - mu - math.lgamma(4.0))) < 1e-10
    # binomial: grad = y - n p, Fisher hess = -n p (1-p)
    lp, g, h = O.eval_lik("binomial", -0.2, 3.0, 10.0)
    p = 1 / (1 + math.exp(0.2))
    assert abs(g - (3.0 - 10.0 * p)) < 1e-12 and abs(h + 10.0 * p * (1 - p)) < 1e-12
    # negative binomial: observed hessian == d/deta grad
    eps = 1e-5
    _, g0, h0 = O.eval_lik("nbinomial", 0.7, 4.0, 5.0, 1.0)
    _, gp, _ = O.eval_lik("nbinomial", 0.7 + eps, 4.0, 5.0, 1.0)
    _, gm, _ = O.eval_lik("nbinomial", 0.7 - eps, 4.0, 5.0, 1.0)
    assert abs(h0 - (gp - gm) / (2 * eps)) < 1e-6
    lpp, _, _ = O.eval_lik("nbinomial", 0.7 + eps, 4.0, 5.0, 1.0)
    lpm, _, _ = O.eval_lik("nbinomial", 0.7 - eps, 4.0, 5.0, 1.0)
    assert abs(g0 - (lpp - lpm) / (2 * eps)) < 1e-6


def test_log_gamma():
    for z in (0.3, 1.0, 2.5, 7.0, 31.5, 200.0):
        assert abs(O.log_gamma(z) - math.lgamma(z)) < 1e-10 * max(1.0, abs(math.lgamma(z)))


def test_gaussian_identity_mode_is_linear_solve():
    """inference.rs:2845-2889: mode == (Q + diag(prec))^-1 (prec*y), 1e-10."""
    n = 4
    q = identity(n, 2.0)
    y = np.array([0.5, -1.0, 2.0, 0.25])
    prec = np.array([1.0, 4.0, 0.5, 9.0])
    r = O.laplace(q, None, "gaussian", y, p1=prec, max_iter=50, tol=1e-12)
    x_lin = (prec * y) / (2.0 + prec)
    np.testing.assert_allclose(r["x"], x_lin, atol=1e-10)
    assert r["iters"] == 1 and math.isfinite(r["mlik"])


def test_gaussian_identity_with_projector():
    """inference.rs:2891-2929."""
    n, nobs = 3, 5
    q = identity(n, 1.5)
    a = sp.csc_matrix(([1.0, 0.5, 0.5, 1.0, 0.25, 0.75, 1.0], ([0, 1, 1, 2, 3, 3, 4], [0, 0, 1, 1, 1, 2, 2])),
                      shape=(nobs, n))
    y = np.array([0.2 * i - 0.4 for i in range(nobs)])
    prec = np.array([1.0 + i for i in range(nobs)])
    r = O.laplace(q, a, "gaussian", y, p1=prec, max_iter=50, tol=1e-12)
    ad = a.toarray()
    qpost = 1.5 * np.eye(n) + ad.T @ np.diag(prec) @ ad
    x_lin = np.linalg.solve(qpost, ad.T @ (prec * y))
    np.testing.assert_allclose(r["x"], x_lin, atol=1e-10)
    # mlik = loglik - 1/2 x'Qx + 1/2 log|Q| - 1/2 log|Qpost|
    eta = ad @ x_lin
    ll = np.sum(-0.9189385332046728 + 0.5 * np.log(prec) - 0.5 * prec * (eta - y) ** 2)
    ml = ll - 0.5 * 1.5 * x_lin @ x_lin + 0.5 * n * math.log(1.5 + 1e-12) - 0.5 * np.linalg.slogdet(qpost)[1]
    assert abs(r["mlik"] - ml) < 1e-9


def test_poisson_newton_converges_to_stationary_point():
    """inference.rs:2932-3023: non-Gaussian families iterate to the mode."""
    n = 6
    q = identity(n, 1.0)
    y = np.array([0.0, 1.0, 3.0, 2.0, 5.0, 1.0])
    r = O.laplace(q, None, "poisson", y, p1=np.ones(n), max_iter=200, tol=1e-10)
    assert r["iters"] > 1
    # stationarity: y - exp(x) - x = 0
    np.testing.assert_allclose(y - np.exp(r["x"]) - r["x"], 0.0, atol=1e-8)


def test_ccd_design_weights():
    """integration.rs:1-62 (CCD m=3: 15 points, weights sum to 1)."""
    z, w = O.ccd_design(3, 1.0)
    assert z.shape == (15, 3)
    assert abs(w.sum() - 1.0) < 1e-12
    z, w = O.ccd_design(4, 1.0)
    assert z.shape == (25, 4)


def test_ccd_design_points_reference():
    """integration.rs:328-347: f0 = 2.5 gives 3 / 9 / 15 points for m = 1 / 2 / 3 with weights
    summing to 1; for m = 1 the points are 0, +2.5, -2.5."""
    z, w = O.ccd_design(1, 2.5)
    assert z.shape == (3, 1)
    assert z[0, 0] == 0.0 and abs(z[1, 0] - 2.5) < 1e-12 and abs(z[2, 0] + 2.5) < 1e-12
    assert abs(w.sum() - 1.0) < 1e-12
    for m, npts in ((2, 9), (3, 15)):
        z, w = O.ccd_design(m, 2.5)
        assert z.shape == (npts, m)
        assert abs(w.sum() - 1.0) < 1e-12


def test_grid_design_points_reference():
    """integration.rs:349-369: spherical Gaussian log-density, step 1, threshold 2: five
    points for m = 1; for m = 2 every kept point has z1^2 + z2^2 <= 4."""
    f = lambda z: -0.5 * sum(v * v for v in z)
    z1, _ = O.grid_design(1, 1.0, 2.0, f)
    assert len(z1) == 5
    z2, _ = O.grid_design(2, 1.0, 2.0, f)
    assert len(z2) > 0 and all(p[0] ** 2 + p[1] ** 2 <= 4.0001 for p in z2)


def test_likelihood_known_answers_reference():
    """inference.rs evaluates_{gaussian,poisson,binomial,negative_binomial}_likelihood on the
    oracle, and the library's host likelihood through its Hessian (the posterior precision of
    Q = 0 at eta) and its log-density (a one-node deviance)."""
    import scipy.sparse as sp

    from inla_b200 import models
    from inla_b200.laplace import model_selection, posterior_precision

    lp, g, h = O.eval_lik("gaussian", 1.5, 1.0, 2.0)
    assert abs(g + 1.0) < 1e-12 and abs(h + 2.0) < 1e-12
    for fam, eta, y, p1 in [("poisson", 0.2, 3.0, 2.0), ("binomial", 0.3, 4.0, 10.0)]:
        assert all(np.isfinite(O.eval_lik(fam, eta, y, p1)))
    mu, r, y = 2.0, 3.0, 4.0
    lp, g, h = O.eval_lik("nbinomial", math.log(2.0), y, r, 1.0)
    d1 = y / mu - (y + r) / (mu + r)
    d2 = -y / (mu * mu) + (y + r) / ((mu + r) * (mu + r))
    assert abs(g - d1 * mu) < 1e-12 and abs(h - (d2 * mu * mu + d1 * mu)) < 1e-12
    # the library's host likelihoods (shared with the device kernels) at the same points
    cases = [("gaussian", 1.5, 1.0, 2.0, 1.0), ("poisson", 0.2, 3.0, 2.0, 1.0), ("binomial", 0.3, 4.0, 10.0, 1.0),
             ("nbinomial", math.log(2.0), 4.0, 3.0, 1.0)]
    zero = models.build_latent(1, [sp.identity(1, format="csc")], "iid")
    for fam, eta, yy, p1, p2 in cases:
        lp, g, h = O.eval_lik(fam, eta, yy, p1, p2)
        q = posterior_precision(zero, [0.0], [eta], a=None, family=fam, y=[yy], p1=[p1], p2=[p2]).toarray()
        assert abs(q[0, 0] + h) <= 1e-13 * max(1.0, abs(h)), fam
        dev = model_selection(fam, [yy], [1.0], 0, [[eta]], [[0.1]], p1=[p1], p2=[p2], criteria=["dic"])
        assert abs(dev["mean_deviance"] + 2.0 * lp) <= 1e-12 * max(1.0, abs(lp)), fam


BINOMIAL_YS = [3., 5., 4., 2., 5., 6., 3., 4., 5., 3., 4., 6., 2., 5., 4., 3., 5., 4., 6., 3., 4., 5.,
               3., 4., 5., 2., 6., 4., 3., 5., 4., 3., 5., 4., 6., 3., 4., 5., 3., 4., 5., 2., 6., 4.,
               3., 5., 4., 3., 5., 4., 6., 3., 4., 5.]


def test_binomial_identity_mode_converges():
    """inference.rs binomial_identity_mode_converges: Q = I (n = 20), y alternating 4 / 6 of 10."""
    n = 20
    y = [4.0 if i % 2 == 0 else 6.0 for i in range(n)]
    r = O.laplace(sp.identity(n, format="csc"), None, "binomial", y, p1=10.0, max_iter=100, tol=1e-6)
    assert np.isfinite(r["mlik"]) and np.all(np.isfinite(r["x"]))
    assert abs(np.mean(r["x"])) < 1.0


def test_binomial_mode_across_prior_strengths():
    """inference.rs binomial_mode_across_prior_strengths: the mode search converges for
    tau in {1e-4, 1e-2, 1, 1e2, 1e4} and with an explicit A = I."""
    n = len(BINOMIAL_YS)
    for tau in (1e-4, 1e-2, 1.0, 1e2, 1e4):
        r = O.laplace(tau * sp.identity(n, format="csc"), None, "binomial", BINOMIAL_YS, p1=10.0, max_iter=100)
        assert np.isfinite(r["mlik"])
    r = O.laplace(sp.identity(n, format="csc"), sp.identity(n, format="csr"), "binomial", BINOMIAL_YS, p1=10.0,
                  max_iter=100)
    assert np.isfinite(r["mlik"])


# --- the supernodal form (the CPU baseline's factorization) ----------------------------------------


@pytest.mark.parametrize("name", golden_cases())
def test_supernodal_factor_matches_dense_golden(name):
    """The supernodal form against the same dense LAPACK golden vectors as the simplicial one."""
    q = golden_matrix(name)
    f = O.Factor(q, perm=O.default_perm(q), supernodal=True)
    assert not f.singular
    assert abs(f.logdet() - GOLDEN[f"{name}/logdet"][0]) <= 1e-10 * max(1.0, abs(GOLDEN[f"{name}/logdet"][0]))
    b = np.arange(1, q.shape[0] + 1, dtype=float)
    np.testing.assert_allclose(f.solve(b), GOLDEN[f"{name}/solve"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(f.diag_inv(), GOLDEN[f"{name}/diag_inv"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("name", list(KNOWN_ANSWER))
def test_supernodal_factor_equals_simplicial(name):
    """Same factor to rounding under every ordering, including a singular-pivot report."""
    q = KNOWN_ANSWER[name][0]()
    for perm in (None, O.default_perm(q), np.arange(q.shape[0])[::-1].copy()):
        a, b = O.Factor(q, perm=perm), O.Factor(q, perm=perm, supernodal=True)
        assert a.nnz() == b.nnz() and a.singular == b.singular
        assert abs(a.logdet() - b.logdet()) <= 1e-12 * max(1.0, abs(a.logdet()))
        np.testing.assert_allclose(b.diag_inv(), a.diag_inv(), rtol=1e-11)


def test_supernodal_on_spde_patterns_and_threads():
    """A 60 x 60 SPDE posterior under the reference's order and the natural one (wide relaxed
    supernodes), factorized from eight threads at once on the shared cached analyses."""
    from concurrent.futures import ThreadPoolExecutor

    import inla_b200.models as M

    p = M.make_spde_problem(nx=60, n_obs=1800)
    perm = O.reference_perm(p.model.pattern)
    qs = []
    for lt, lk in ((-1.0, 1.2), (-3.0, 2.5), (0.5, 0.3)):
        c, _ = M.spde_coefs(lt, lk)
        q = (p.model.matrix(c) + 25.0 * (p.a.T @ p.a)).tocsc()
        q.sort_indices()
        qs.append(q)
    ref = [(O.Factor(q, perm=pp).logdet(), O.Factor(q, perm=pp).solve(np.ones(q.shape[0])))
           for q in qs for pp in (perm, None)]

    def run(k):
        q, pp = qs[(k // 2) % 3], (perm, None)[k % 2]
        f = O.Factor(q, perm=pp, supernodal=True)
        return f.logdet(), f.solve(np.ones(q.shape[0]))

    with ThreadPoolExecutor(max_workers=8) as ex:
        got = list(ex.map(run, range(48)))
    for k, (ld, x) in enumerate(got):
        ld_ref, x_ref = ref[((k // 2) % 3) * 2 + k % 2]
        assert abs(ld - ld_ref) <= 1e-12 * abs(ld_ref)
        np.testing.assert_allclose(x, x_ref, rtol=1e-9, atol=1e-12 * np.max(np.abs(x_ref)))


def test_supernodal_laplace_equals_simplicial():
    """The Laplace evaluation the CPU baseline times, with either factorization."""
    import inla_b200.models as M

    p = M.make_spde_problem(nx=30, n_obs=400)
    q = p.model.matrix(O.spde_coefs(-1.0, 1.2))
    perm = O.reference_perm(p.model.pattern)
    a = O.laplace(q, p.a, "gaussian", p.y, p1=25.0, perm=perm, want_var=True)
    O.set_supernodal(True)
    try:
        b = O.laplace(q, p.a, "gaussian", p.y, p1=25.0, perm=perm, want_var=True)
    finally:
        O.set_supernodal(False)
    for key in a:
        va, vb = np.asarray(a[key], dtype=float), np.asarray(b[key], dtype=float)
        np.testing.assert_allclose(vb, va, rtol=1e-10, atol=1e-12 * max(1.0, np.max(np.abs(va))), err_msg=key)


def test_supernodal_threads_inside_one_factorization_give_the_same_bits():
    """orc_set_threads runs independent subtrees as tasks and splits large updates by target
    column; every entry still receives its updates in the same order, so the factor is
    bit-identical for any thread count (minimum-degree order: a bushy tree; natural order: a band
    of ~100 with large updates)."""
    import inla_b200.models as M

    p = M.make_spde_problem(nx=100, n_obs=5000)
    c, _ = M.spde_coefs(-1.0, 1.2)
    q = (p.model.matrix(c) + 25.0 * (p.a.T @ p.a)).tocsc()
    q.sort_indices()
    x = np.linspace(-1.0, 1.0, q.shape[0])
    for perm in (O.reference_perm(p.model.pattern), None):
        base = O.Factor(q, perm=perm, supernodal=True)
        for t in (2, 4, 8):
            try:
                O.set_threads(t)
                f = O.Factor(q, perm=perm, supernodal=True)
            finally:
                O.set_threads(1)
            assert f.logdet() == base.logdet()
            assert np.array_equal(f.solve(x), base.solve(x))


def test_oracle_against_superlu_at_a_realistic_size():
    """An independent pin at n = 10 000 (SPDE 100 x 100 posterior): SuperLU's log|det| (sum of
    log|U_ii|) and solve against both factorizations of the oracle, and 16 marginal variances
    (Q^-1)_ii from SuperLU solves against the oracle's Takahashi diagonal."""
    import scipy.sparse.linalg as spla

    import inla_b200.models as M

    p = M.make_spde_problem(nx=100, n_obs=5000)
    c, _ = M.spde_coefs(-2.0, 2.0)
    q = (p.model.matrix(c) + 50.0 * (p.a.T @ p.a)).tocsc()
    q.sort_indices()
    lu = spla.splu(q, permc_spec="COLAMD")
    ld_ref = float(np.sum(np.log(np.abs(lu.U.diagonal()))))
    b = np.cos(np.arange(q.shape[0]))
    x_ref = lu.solve(b)
    perm = O.reference_perm(p.model.pattern)
    idx = np.random.default_rng(3).choice(q.shape[0], 16, replace=False)
    var_ref = np.array([lu.solve(np.eye(1, q.shape[0], i).ravel())[i] for i in idx])  # (Q^-1 e_i)_i
    for sn in (False, True):
        f = O.Factor(q, perm=perm, supernodal=sn)
        assert abs(f.logdet() - ld_ref) <= 1e-10 * abs(ld_ref)
        np.testing.assert_allclose(f.solve(b), x_ref, rtol=1e-9, atol=1e-12 * np.max(np.abs(x_ref)))
    # the reference's Takahashi recurrence (sparse_ldlt.rs:376-432) on the simplicial factor
    np.testing.assert_allclose(O.Factor(q, perm=perm).diag_inv()[idx], var_ref, rtol=1e-9)
