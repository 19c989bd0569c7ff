"""Parity at the benchmarked size and at the largest configuration.

SPDE 200 x 200 (n = 40 000 latent nodes, 20 000 Gaussian observations), the workload the
benchmark times: the batched + adjoint fit of the benchmark runs, and at three of its CCD
nodes the batched Laplace evaluation (prior and posterior log-determinants, the mode x* and
the marginal variances diag(Q_post^-1)) is compared with the CPU oracle's restatement of
find_latent_mode_a_with_solver (inference.rs:776-975) and of the Takahashi recurrence
(sparse_ldlt.rs:376-432) at the same theta: log-determinants 1e-10 relative, x* 1e-8 relative
to its largest entry, and every marginal variance 1e-8 relative to itself (element-wise).

SPDE 600 x 600 (n = 360 000, 100 000 negative-binomial counts): one theta-point; the prior and
posterior log-determinants against the oracle's factorization of the same matrices (1e-10
relative) and a sample of 24 marginal variances against (Q_post^-1)_ii from oracle solves
(1e-8 relative each). The oracle gets the library's nested-dissection permutation here (an
input like any other; its minimum-degree order takes minutes at this size); results do not
depend on the permutation beyond rounding.
"""
import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle as O
from inla_b200 import GpuSolver, _lib, models
from inla_b200.laplace import LaplaceModel

pytestmark = pytest.mark.gpu

RT_LD = 1e-10
RT_X = 1e-8
RT_VAR = 1e-8


def elementwise_rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)) / np.abs(np.asarray(b))))


def test_spde200_ccd_nodes_match_oracle():
    p = models.make_spde_problem(nx=200, n_obs=20_000)
    lm = LaplaceModel(p.model, a=p.a, family="gaussian", y=p.y, max_batch=25)
    r = lm.fit([0.0, 0.0, 0.0], mode_search="newton", batched=True, tol=1e-4)
    nodes = r["node_theta"][[0, 5, 12]]
    coefs = np.stack([models.spde_coefs(t[1], t[2])[0] for t in nodes])
    scale = np.exp(nodes[:, 0])
    out = lm.eval(coefs, scale, variances=True)
    assert np.all(out["status"] == 0)
    perm = O.reference_perm(p.model.pattern)

    def oracle_node(b):
        q = p.model.matrix(coefs[b])
        return O.laplace(q, p.a, "gaussian", p.y, p1=scale[b], want_var=True, perm=perm)

    with ThreadPoolExecutor(max_workers=len(nodes)) as ex:
        refs = list(ex.map(oracle_node, range(len(nodes))))
    worst = {"ld_prior": 0.0, "ld_post": 0.0, "x": 0.0, "var": 0.0}
    for b, ref in enumerate(refs):
        worst["ld_prior"] = max(worst["ld_prior"],
                                abs(out["logdet_prior"][b] - ref["logdet_prior"]) / abs(ref["logdet_prior"]))
        worst["ld_post"] = max(worst["ld_post"], abs(out["logdet_post"][b] - ref["logdet_post"]) / abs(ref["logdet_post"]))
        worst["x"] = max(worst["x"], np.max(np.abs(out["x"][b] - ref["x"])) / np.max(np.abs(ref["x"])))
        worst["var"] = max(worst["var"], elementwise_rel(out["var"][b], ref["var"]))
        assert abs(out["mlik"][b] - ref["mlik"]) <= RT_LD * abs(ref["logdet_post"])
    print(f"spde200 worst relative errors at 3 CCD nodes: {worst}")
    assert worst["ld_prior"] <= RT_LD and worst["ld_post"] <= RT_LD
    assert worst["x"] <= RT_X
    assert worst["var"] <= RT_VAR


def test_spde600_nbinomial_logdet_and_variance_sample():
    p = models.make_spde_problem(nx=600, n_obs=100_000, seed=models.SEED_BASE + 5, family="nbinomial")
    theta = (-3.0, 2.5)
    c, _ = models.spde_coefs(*theta)
    lm = LaplaceModel(p.model, a=p.a, family="nbinomial", y=p.y, p1=5.0, p2=1.0, max_batch=1)
    out = lm.eval(c[None, :], variances=True)
    assert out["status"][0] == 0
    s = GpuSolver(_lib.ORDER_ND)
    s.analyze(p.model.pattern)
    perm = s.perm()
    s.close()
    q = p.model.matrix(c)
    # the posterior precision at the library's mode: Q + A^T W(x*) A with the NB weights
    x = out["x"][0]
    eta = p.a @ x
    w = np.array([-O.eval_lik("nbinomial", e, yy, 5.0, 1.0)[2] for e, yy in zip(eta, p.y)])
    import scipy.sparse as sp

    qpost = (q + p.a.T @ sp.diags(w) @ p.a).tocsc()
    qpost.sort_indices()
    with ThreadPoolExecutor(max_workers=2) as ex:
        fp, fq = ex.map(lambda m: O.Factor(m, perm=perm), [q.tocsc(), qpost])
    ld_prior_ref = fp.logdet()
    ld_post_ref = fq.logdet()
    print(f"spde600: logdet prior {out['logdet_prior'][0]:.15g} vs {ld_prior_ref:.15g}, "
          f"post {out['logdet_post'][0]:.15g} vs {ld_post_ref:.15g}")
    # an unconstrained intrinsic-free SPDE prior: the 1e-12 jitter is below rounding here
    assert abs(out["logdet_prior"][0] - ld_prior_ref) <= RT_LD * abs(ld_prior_ref)
    assert abs(out["logdet_post"][0] - ld_post_ref) <= RT_LD * abs(ld_post_ref)
    rng = np.random.default_rng(5)
    idx = rng.choice(q.shape[0], size=24, replace=False)
    worst = 0.0
    for i in idx:
        e = np.zeros(q.shape[0])
        e[i] = 1.0
        vi = fq.solve(e)[i]
        worst = max(worst, abs(out["var"][0][i] - vi) / vi)
    print(f"spde600 worst relative variance error over 24 nodes: {worst:.3e}")
    assert worst <= RT_VAR
