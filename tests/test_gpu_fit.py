"""GPU INLA fits: the plain reference control flow (Nelder-Mead, FD Hessian,
CCD, one theta-point per evaluation) against the oracle's restatement, and
the batched BFGS + adjoint path against the plain one."""
import numpy as np
import pytest

import oracle as O
from inla_b200 import models
from inla_b200.laplace import LaplaceModel

pytestmark = pytest.mark.gpu

THETA0 = np.array([3.0, -2.5, 2.0])


@pytest.fixture(scope="module")
def problem():
    p = models.make_spde_problem(nx=20, n_obs=300, seed=11)
    lm = LaplaceModel(p.model, a=p.a, family="gaussian", y=p.y, max_batch=25)
    return p, lm


def oracle_f(p):
    return lambda th: O.spde_neg_log_posterior(np.asarray(th), p.model, p.a, p.y)


def test_plain_fit_follows_reference_nelder_mead(problem):
    p, lm = problem
    r = lm.fit(THETA0, mode_search="nm", batched=False)
    mode_ref = O.nelder_mead(list(THETA0), 0.1, 200, 1e-6, oracle_f(p))
    np.testing.assert_allclose(r["mode"], mode_ref, atol=1e-6)
    h = max(1e-4, max(0.05 * abs(t) for t in mode_ref))
    H_ref = O.fd_hessian(mode_ref, oracle_f(p), h)
    np.testing.assert_allclose(r["hessian"], H_ref, rtol=1e-5, atol=1e-6)


def test_integration_parity_at_fixed_nodes(problem):
    """Weights, posterior means and marginal variances at the same mode/Hessian: 1e-8 relative."""
    p, lm = problem
    r = lm.fit(THETA0, mode_search="nm", batched=True)

    def node(theta):
        c = O.spde_coefs(theta[1], theta[2])
        lr = O.laplace(p.model.matrix(c), p.a, "gaussian", p.y, p1=np.exp(theta[0]), want_var=True)
        lp = O.loggamma_log_dens(theta[0], 1.0, 5e-5) + O.pc_spde_log_dens(theta[1], theta[2], 1.0, 0.05, 1.0, 0.01)
        return lr["x"], lr["var"], lr["mlik"] + lp

    ref = O.integrate(r["mode"], r["hessian"], node, f0=1.0, a=p.a)
    # node sets agree as sets (eigenvector sign conventions may permute them)
    got = sorted(map(tuple, np.round(r["node_theta"], 9)))
    exp = sorted(map(tuple, np.round(ref["thetas"], 9)))
    np.testing.assert_allclose(got, exp, atol=1e-8)
    rel = lambda a, b: np.max(np.abs(a - b)) / np.max(np.abs(b))
    assert rel(r["mean"], ref["mean"]) < 1e-8
    assert rel(r["var"], ref["var"]) < 1e-8
    assert abs(r["mlik"] - ref["mlik"]) < 1e-8 * abs(ref["mlik"])
    # linear predictor eta = A x (inference.rs:1451-1466): its mixture mean is A times the latent one
    assert rel(r["pred_mean"], ref["pred_mean"]) < 1e-8
    assert rel(r["pred_var"], ref["pred_var"]) < 1e-8
    assert rel(r["pred_mean"], p.a @ r["mean"]) < 1e-12


def test_model_selection_parity(problem):
    """DIC, WAIC, CPO / PIT and the Gaussian-approximation mlik of a fit (inference.rs:1470-1514)
    against the oracle's restatement on the oracle's node results at the fit's nodes."""
    p, lm = problem
    r = lm.fit(THETA0, mode_search="nm", batched=True)
    ms = lm.model_selection()
    ce, cv, lps = [], [], []
    for theta in r["node_theta"]:
        c = O.spde_coefs(theta[1], theta[2])
        lr = O.laplace(p.model.matrix(c), p.a, "gaussian", p.y, p1=np.exp(theta[0]), want_var=True)
        ce.append(O.matvec_csc(p.a, lr["x"]))
        cv.append(O.predictor_variances_diag(p.a, lr["var"]))
        lps.append(lr["mlik"] + O.loggamma_log_dens(theta[0], 1.0, 5e-5)
                   + O.pc_spde_log_dens(theta[1], theta[2], 1.0, 0.05, 1.0, 0.01))
    k0 = int(np.argmin(np.linalg.norm(r["node_theta"] - r["mode"], axis=1)))
    n = len(p.y)
    q1, q2 = np.full(n, np.exp(r["mode"][0])), np.ones(n)
    w = r["node_weight"]
    dic = O.compute_dic("gaussian", p.y, q1, q2, ce, w, k0)
    waic = O.compute_waic("gaussian", p.y, q1, q2, ce, w)
    close = lambda a, b: abs(a - b) <= 1e-8 * max(1.0, abs(b))
    assert close(ms["dic"], dic["dic"]) and close(ms["mean_deviance"], dic["mean_deviance"])
    assert close(ms["waic"], waic["waic"]) and close(ms["lppd"], waic["lppd"])
    assert close(ms["mlik_gaussian"], O.mlik_gaussian(lps[k0], -np.asarray(r["hessian"]), 3))
    cpo, pit, nf = O.compute_cpo_pit("gaussian", p.y, q1, q2, ce, cv, w)
    both = np.array([c is not None for c in cpo]) & ~np.isnan(ms["cpo"])
    assert abs(ms["cpo_failures"] - nf) <= 1 and both.sum() >= n - nf - 1
    np.testing.assert_allclose(ms["cpo"][both], [c for c, b in zip(cpo, both) if b], rtol=1e-7)
    np.testing.assert_allclose(ms["pit"][both], [q for q, b in zip(pit, both) if b], rtol=1e-7, atol=1e-12)


def test_fit_marginals_match_oracle(problem):
    """Latent, predictor and hyperparameter marginals of a fit (marginals.rs:83-162) against the
    oracle's restatement on the oracle's node results at the fit's nodes."""
    p, lm = problem
    r = lm.fit(THETA0, mode_search="nm", batched=True)
    w = list(r["node_weight"])
    nodes = []
    for theta in r["node_theta"]:
        c = O.spde_coefs(theta[1], theta[2])
        lr = O.laplace(p.model.matrix(c), p.a, "gaussian", p.y, p1=np.exp(theta[0]), want_var=True)
        nodes.append((lr["x"], lr["var"], O.matvec_csc(p.a, lr["x"]), O.predictor_variances_diag(p.a, lr["var"])))
    for kind, idx, pos in [("latent", 0, 0), ("latent", p.model.n - 1, 0), ("predictor", 7, 2)]:
        x, y = lm.marginal(kind, idx)
        xo, yo = O.gaussian_mixture_marginal([nd[pos][idx] for nd in nodes], [nd[pos + 1][idx] for nd in nodes], w)
        np.testing.assert_allclose(x, xo, rtol=1e-7, atol=1e-9 * np.max(np.abs(xo)))
        np.testing.assert_allclose(y, yo, rtol=1e-6, atol=1e-9 * np.max(yo))
    for j in range(3):
        x, y = lm.marginal("hyperpar", j)
        xo, yo = O.hyperpar_marginal_from_nodes(list(r["node_theta"][:, j]), w)
        np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(y, yo, rtol=1e-9, atol=1e-12 * np.max(yo))


def test_fit_posterior_precision(problem):
    """Posterior precision at the mode (inference.rs:1027-1058, 1565-1570): Q(theta*) + A^T W A at
    the latent mode of the node nearest the mode, with the observations as given to the model,
    against the host assembly on the oracle's mode at that node."""
    from inla_b200.laplace import posterior_precision

    p, lm = problem
    r = lm.fit(THETA0, mode_search="nm", batched=True)
    qp = lm.posterior_precision()
    k0 = int(np.argmin(np.linalg.norm(r["node_theta"] - r["mode"], axis=1)))
    th = r["node_theta"][k0]
    x = O.laplace(p.model.matrix(O.spde_coefs(th[1], th[2])), p.a, "gaussian", p.y, p1=np.exp(th[0]))["x"]
    c, _ = models.spde_coefs(r["mode"][1], r["mode"][2])
    ref = posterior_precision(p.model, c, x, a=p.a, family="gaussian", y=p.y)
    d = (qp - ref).toarray()
    assert np.max(np.abs(d)) <= 1e-8 * np.max(np.abs(ref.toarray()))


def test_lincomb_summaries_on_the_gpu_solver(problem):
    """lincomb_summaries (posterior.rs:55-92) with the posterior precision factorized on the GPU
    solver: sd against a dense inverse."""
    from inla_b200.laplace import lincomb_summaries

    p, lm = problem
    r = lm.fit(THETA0, mode_search="nm", batched=True)
    q = lm.posterior_precision()
    res = lincomb_summaries(r["mean"], q, [("x0", [(0, 1.0)]), ("pair", [(5, 1.0), (17, -0.5)])])
    cov = np.linalg.inv(q.toarray())
    a = np.zeros(q.shape[0])
    a[5], a[17] = 1.0, -0.5
    assert abs(res[0]["sd"] - np.sqrt(cov[0, 0])) <= 1e-9 * np.sqrt(cov[0, 0])
    assert abs(res[1]["sd"] - np.sqrt(a @ cov @ a)) <= 1e-9 * np.sqrt(a @ cov @ a)
    assert res[1]["mean"] == pytest.approx(a @ r["mean"], rel=1e-14, abs=1e-14)


@pytest.mark.parametrize("search", ["bfgs", "newton"])
def test_batched_adjoint_fit_matches_plain(problem, search):
    p, lm = problem
    plain = lm.fit(THETA0, mode_search="nm", batched=False)
    fast = lm.fit(THETA0, mode_search=search, batched=True, tol=1e-5)
    f = oracle_f(p)
    # BFGS on exact gradients reaches the optimum at least as well as NM
    assert f(fast["mode"]) <= f(plain["mode"]) + 1e-6
    np.testing.assert_allclose(fast["mode"], plain["mode"], atol=5e-2)
    assert np.max(np.abs(fast["mean"] - plain["mean"])) < 1e-2 * np.max(np.abs(plain["mean"]))
    assert np.max(np.abs(fast["var"] - plain["var"]) / plain["var"]) < 5e-2
    assert fast["n_batches"] < plain["n_batches"]


def test_fit_with_gradient_hessian(problem):
    p, lm = problem
    a = lm.fit(THETA0, mode_search="bfgs", batched=True, tol=1e-5, hessian="fd")
    b = lm.fit(THETA0, mode_search="bfgs", batched=True, tol=1e-5, hessian="grad")
    np.testing.assert_allclose(a["hessian"], b["hessian"], rtol=0.1, atol=0.5)


def test_fit_cancellation_stops_and_leaves_the_handle_usable(problem):
    """check_cancel (inference.rs:1116-1130, hyper_opt.rs:21-24): polled before every
    evaluation; a cancel stops the fit with the Cancelled status."""
    from inla_b200 import _lib

    p, lm = problem
    polls = []

    def cancel():
        polls.append(1)
        return len(polls) > 3

    with pytest.raises(_lib.InlaError) as e:
        lm.fit(THETA0, mode_search="nm", batched=False, cancel=cancel)
    assert e.value.code == _lib.INLA_ERR_CANCELLED
    assert len(polls) == 4  # three evaluations ran, the fourth poll cancelled
    with pytest.raises(_lib.InlaError) as e:
        lm.fit(THETA0, mode_search="newton", batched=True, cancel=lambda: True)
    assert e.value.code == _lib.INLA_ERR_CANCELLED
    r = lm.fit(THETA0, mode_search="newton", batched=True, tol=1e-5, cancel=lambda: False)
    plain = lm.fit(THETA0, mode_search="nm", batched=False)
    np.testing.assert_allclose(r["mode"], plain["mode"], atol=5e-2)


def test_fit_without_hyperparameters_is_one_laplace_node(problem):
    """m = 0 (inference.rs:1135-1239): one Laplace evaluation with variances, weight 1, the
    Laplace mlik without a prior term, no integration nodes."""
    p, lm = problem
    th = np.array([4.0, -3.0, 2.5])
    c = O.spde_coefs(th[1], th[2])
    r = lm.fit(np.zeros(0), theta_map=lambda t: (c, np.zeros((0, 3)), np.exp(th[0]), np.zeros(0)),
               priors=lambda t: (0.0, np.zeros(0)), batched=True)
    ref = O.laplace(p.model.matrix(c), p.a, "gaussian", p.y, p1=np.exp(th[0]), want_var=True)
    assert abs(r["mlik"] - ref["mlik"]) <= 1e-10 * abs(ref["logdet_post"])
    assert np.max(np.abs(r["mean"] - ref["x"])) <= 1e-8 * np.max(np.abs(ref["x"]))
    assert np.max(np.abs(r["var"] - ref["var"]) / ref["var"]) <= 1e-8
    assert r["node_theta"].shape[0] == 0 and r["n_evals"] == 1 and r["mode"].shape == (0,)
    np.testing.assert_allclose(r["pred_mean"], O.matvec_csc(p.a, ref["x"]), rtol=1e-8, atol=1e-10)
    np.testing.assert_allclose(r["pred_var"], O.predictor_variances_diag(p.a, ref["var"]), rtol=1e-8)
    ms = lm.model_selection()
    assert ms["mlik_gaussian"] == pytest.approx(r["mlik"], rel=1e-15)
    n = len(p.y)
    q1 = np.full(n, np.exp(th[0]))
    dic = O.compute_dic("gaussian", p.y, q1, np.ones(n), [O.matvec_csc(p.a, ref["x"])], [1.0], 0)
    assert abs(ms["dic"] - dic["dic"]) <= 1e-8 * max(1.0, abs(dic["dic"]))
