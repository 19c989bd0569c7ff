"""GPU parity of the multi-model engine: independent AR1 + iid + intercept Poisson
models of uneven size held block-diagonally and evaluated together. Per
(theta-set, model) against the oracle's find_latent_mode_a_with_solver
(inference.rs:776-975) on that model alone: equal Newton iteration counts,
log-determinants 1e-10 relative, mlik 1e-10 of |log|Q_post||, modes and
marginal variances 1e-8 relative; the per-model adjoint pieces against central
differences of the oracle's mlik; the full 512-model batch (1.4 M latent nodes)
checked on sampled models."""
import math

import numpy as np
import pytest

import oracle as O
from inla_b200 import models
from inla_b200.multi import MultiModel

pytestmark = pytest.mark.gpu

RT_LD = 1e-10
RT_X = 1e-8


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300)


def thetas_for(p, rng, B):
    """Per (theta-set, model) hyperparameters scattered around the generating values."""
    G = len(p.models)
    th = np.zeros((B, G, 3))
    rho = p.truth["rho"]
    th[:, :, 0] = np.log(p.truth["tau"])[None, :] + rng.normal(0.0, 0.3, size=(B, G))
    th[:, :, 1] = np.log((1 + rho) / (1 - rho))[None, :] + rng.normal(0.0, 0.3, size=(B, G))
    th[:, :, 2] = math.log(p.truth["tau_iid"]) + rng.normal(0.0, 0.3, size=(B, G))
    return th


def coefs_of(th):
    B, G, _ = th.shape
    return np.stack([[models.ar1_iid_coefs(th[b, g])[0] for g in range(G)] for b in range(B)])


def chain_perm(nk):
    """Elimination order for the oracle (perm[new] = old): iid node, then AR1 node, along the
    chain, intercept last -- O(n) fill, where the oracle's natural-order fallback for the
    AMD branch would eliminate the dense intercept row first and fill the whole matrix."""
    return np.r_[np.stack([1 + nk + np.arange(nk), 1 + np.arange(nk)], axis=1).ravel(), 0].astype(np.int64)


def check_model(out, b, g, mm, p, coef):
    r = O.laplace(p.models[g].matrix(coef), p.a[g], "poisson", p.y[g], want_var=True,
                  perm=chain_perm(p.truth["n"][g]))
    assert out["status"][b, g] == 0
    assert out["iters"][b, g] == r["iters"]
    assert abs(out["logdet_prior"][b, g] - r["logdet_prior"]) <= RT_LD * abs(r["logdet_prior"])
    assert abs(out["logdet_post"][b, g] - r["logdet_post"]) <= RT_LD * abs(r["logdet_post"])
    assert abs(out["mlik"][b, g] - r["mlik"]) <= RT_LD * abs(r["logdet_post"])
    assert rel(mm.split(out["x"][b])[g], r["x"]) < RT_X
    assert rel(mm.split(out["var"][b])[g], r["var"]) < RT_X


@pytest.fixture(scope="module")
def small():
    p = models.make_multi_problem(G=10, n_hi=1500, seed=7)
    mm = MultiModel(p.models, p.a, p.y, family="poisson", max_batch=4)
    return p, mm


def test_multi_matches_oracle_per_model(small):
    p, mm = small
    th = thetas_for(p, np.random.default_rng(1), 2)
    c = coefs_of(th)
    out = mm.eval(c, variances=True)
    for b in range(2):
        for g in range(mm.G):
            check_model(out, b, g, mm, p, c[b, g])


def test_multi_adjoint_vs_central_fd(small):
    p, mm = small
    th = thetas_for(p, np.random.default_rng(2), 1)
    c = coefs_of(th)
    out = mm.eval(c, gradient=True)
    T = 5
    for g in (0, mm.G - 1):
        t = th[0, g]
        dc = models.ar1_iid_coefs(t)[1]
        gr = dc @ (0.5 * out["trP"][0, g, :T] - 0.5 * out["trQ"][0, g, :T] - 0.5 * out["xMx"][0, g, :T]
                   + 0.5 * out["zMx"][0, g, :T])

        def mlik(tt):
            q = p.models[g].matrix(models.ar1_iid_coefs(tt)[0])
            return O.laplace(q, p.a[g], "poisson", p.y[g], tol=1e-10, perm=chain_perm(p.truth["n"][g]))["mlik"]

        h = 1e-4
        fd = np.array([(mlik(t + h * e) - mlik(t - h * e)) / (2 * h) for e in np.eye(3)])
        assert np.max(np.abs(gr - fd)) <= 2e-3 * max(1.0, np.max(np.abs(fd))), (g, gr, fd)


def test_multi_models_are_independent(small):
    """Changing one model's coefficients leaves every other model's results unchanged
    bit for bit (per-model reductions, no cross-model arithmetic)."""
    p, mm = small
    th = thetas_for(p, np.random.default_rng(3), 1)
    c = coefs_of(th)
    a = mm.eval(c, variances=True)
    c2 = c.copy()
    c2[0, 3] = models.ar1_iid_coefs(th[0, 3] + 0.5)[0]
    b = mm.eval(c2, variances=True)
    for g in range(mm.G):
        same = g != 3
        assert (a["mlik"][0, g] == b["mlik"][0, g]) == same
        if same:
            np.testing.assert_array_equal(mm.split(a["x"][0])[g], mm.split(b["x"][0])[g])
            np.testing.assert_array_equal(mm.split(a["var"][0])[g], mm.split(b["var"][0])[g])


def test_config4_512_uneven_models():
    p = models.make_multi_problem()
    mm = MultiModel(p.models, p.a, p.y, family="poisson", max_batch=4)
    th = thetas_for(p, np.random.default_rng(4), 2)
    c = coefs_of(th)
    out = mm.eval(c, variances=True)
    assert np.all(out["status"] == 0)
    assert np.all(out["var"] > 0) and np.all(np.isfinite(out["mlik"]))
    for g in (0, int(np.argmax(p.truth["n"])), 511):
        check_model(out, 1, g, mm, p, c[1, g])


def single_fit(p, g):
    """The same model fitted on its own through the single-model engine (batched Newton on
    adjoint gradients, FD Hessian of values, CCD)."""
    from inla_b200.laplace import LaplaceModel
    from inla_b200.multi import AR1_IID_PRIORS

    lm = LaplaceModel(p.models[g], a=p.a[g], family="poisson", y=p.y[g], max_batch=25)

    def tmap(t):
        c, dc = models.ar1_iid_coefs(t)
        return c, dc, 1.0, np.zeros(3)

    return lm.fit(np.zeros(3), theta_map=tmap, priors=AR1_IID_PRIORS, mode_search="newton", batched=True)


def check_fit(r, s, mm, g):
    np.testing.assert_allclose(r["mode"][g], s["mode"], atol=1e-6)
    np.testing.assert_allclose(r["hessian"][g], s["hessian"], rtol=1e-5, atol=1e-6)
    assert rel(mm.split(r["mean"])[g], s["mean"]) < 1e-6
    assert rel(mm.split(r["var"])[g], s["var"]) < 1e-6
    assert abs(r["mlik"][g] - s["mlik"]) < 1e-6 * abs(s["mlik"])
    # each predictor row sums three latent entries (intercept, AR1, iid), so the 1e-6 bound of
    # the latent moments allows up to about 3e-6 on the predictor
    o0, o1 = int(mm.obs_off[g]), int(mm.obs_off[g + 1])
    assert rel(r["pred_mean"][o0:o1], s["pred_mean"]) < 5e-6
    assert rel(r["pred_var"][o0:o1], s["pred_var"]) < 5e-6


def test_multi_fit_matches_single_model_fits(small):
    """Lockstep fit of all models: each model takes the decisions it takes alone."""
    p, mm = small
    r = mm.fit(np.zeros((mm.G, 3)))
    assert np.all(r["status"] == 0)
    for g in (0, 4, mm.G - 1):
        check_fit(r, single_fit(p, g), mm, g)


def test_config4_fit_512_models():
    """Config 4: per-model mode search on adjoint gradients, Hessian and CCD for 512 uneven
    models in one lockstep fit; two models checked against their own single-model fits."""
    p = models.make_multi_problem()
    mm = MultiModel(p.models, p.a, p.y, family="poisson", max_batch=15)
    r = mm.fit(np.zeros((mm.G, 3)))
    assert np.all(r["status"] == 0)
    # the reference's CCD weights for m = 3, f0 = 1 give the centre node weight 1 - 14 w = -0.68
    # (integration.rs:1-62), so a mixture variance can come out negative where the node
    # variances differ; parity with the single-model fits is the check
    assert np.all(np.isfinite(r["mlik"])) and np.all(np.isfinite(r["var"]))
    print(f"config4 fit: {r['seconds']:.2f} s, {r['n_batches']} batches, {r['n_model_evals']} model evaluations, "
          f"max mode iterations {int(r['mode_iters'].max())}")
    for g in (int(np.argmin(p.truth["n"])), int(np.argmax(p.truth["n"]))):
        check_fit(r, single_fit(p, g), mm, g)


def test_multi_gaussian_closed_form_matches_oracle():
    """Gaussian family (closed-form mode, inference.rs:845-870) with a per-model observation
    precision through p1scale."""
    p = models.make_multi_problem(G=4, n_hi=600, seed=11)
    ys = [np.log1p(y) for y in p.y]  # continuous responses on the same models
    mm = MultiModel(p.models, p.a, ys, family="gaussian", p1=1.0, max_batch=2)
    th = thetas_for(p, np.random.default_rng(5), 2)
    c = coefs_of(th)
    prec = np.array([[2.0, 5.0, 1.5, 3.0], [4.0, 1.0, 2.5, 6.0]])
    out = mm.eval(c, p1scale=prec, variances=True)
    assert np.all(out["status"] == 0) and np.all(out["iters"] == 1)
    for b in range(2):
        for g in range(4):
            r = O.laplace(p.models[g].matrix(c[b, g]), p.a[g], "gaussian", ys[g], p1=prec[b, g], want_var=True,
                          perm=chain_perm(p.truth["n"][g]))
            assert abs(out["logdet_post"][b, g] - r["logdet_post"]) <= RT_LD * abs(r["logdet_post"])
            assert abs(out["mlik"][b, g] - r["mlik"]) <= RT_LD * abs(r["logdet_post"])
            assert rel(mm.split(out["x"][b])[g], r["x"]) < RT_X
            assert rel(mm.split(out["var"][b])[g], r["var"]) < RT_X


def test_multi_fit_python_map_and_gradient_hessian(small):
    """inla_multi_fit with a Python theta map (per-model callback) and the FD-of-gradient
    Hessian against the single-model fits with the same options."""
    from inla_b200.laplace import LaplaceModel
    from inla_b200.multi import AR1_IID_PRIORS

    p, mm = small

    def tmap_g(g, t):
        cc, dc = models.ar1_iid_coefs(t)
        return cc, dc, 1.0, np.zeros(3)

    r = mm.fit(np.zeros((mm.G, 3)), theta_map=tmap_g, hessian="grad")
    assert np.all(r["status"] == 0)
    for g in (1, mm.G - 2):
        lm = LaplaceModel(p.models[g], a=p.a[g], family="poisson", y=p.y[g], max_batch=25)
        s = lm.fit(np.zeros(3), theta_map=lambda t: tmap_g(g, t), priors=AR1_IID_PRIORS, mode_search="newton",
                   batched=True, hessian="grad")
        np.testing.assert_allclose(r["mode"][g], s["mode"], atol=1e-6)
        np.testing.assert_allclose(r["hessian"][g], s["hessian"], rtol=1e-5, atol=1e-6)
        assert rel(mm.split(r["mean"])[g], s["mean"]) < 1e-6
        assert abs(r["mlik"][g] - s["mlik"]) < 1e-6 * abs(s["mlik"])
