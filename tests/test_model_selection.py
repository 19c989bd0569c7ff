"""Model-selection criteria (host code of the library, no GPU): the reference's own known-answer
tests (crates/inla_stats/src/model_selection.rs:529-800) through the C ABI, and DIC / WAIC /
CPO / PIT against the oracle's restatement for every family."""
import math

import numpy as np
import pytest

import oracle as O
from inla_b200 import InlaError
from inla_b200.laplace import cpo_failure, mlik_gaussian, model_selection, observation_cdf


# --- model_selection.rs:539-567: Gaussian approximation of the marginal likelihood -----------

def test_gaussian_mlik_trivial_1d():
    expect = -3.0 + 0.5 * math.log(2.0 * math.pi) - 0.5 * math.log(4.0)
    assert abs(mlik_gaussian(-3.0, [[4.0]]) - expect) < 1e-12
    assert abs(O.mlik_gaussian(-3.0, [4.0], 1) - expect) < 1e-12


def test_gaussian_mlik_2d():
    expect = -5.0 + math.log(2.0 * math.pi) - 0.5 * math.log(16.0)
    assert abs(mlik_gaussian(-5.0, [[2.0, 0.0], [0.0, 8.0]]) - expect) < 1e-12


def test_gaussian_mlik_zero_hyperparams():
    assert abs(mlik_gaussian(-2.0, []) + 2.0) < 1e-12


def test_gaussian_mlik_matches_oracle_and_rejects_indefinite():
    rng = np.random.default_rng(3)
    b = rng.normal(size=(4, 4))
    h = b @ b.T + 4 * np.eye(4)
    assert mlik_gaussian(1.5, h) == O.mlik_gaussian(1.5, h, 4)
    with pytest.raises(InlaError):
        mlik_gaussian(0.0, [[1.0, 2.0], [2.0, 1.0]])


# --- model_selection.rs:570-623: DIC and WAIC sanity ------------------------------------------

Y2 = [1.0, 2.0]
MODES2 = [[1.0, 2.0], [1.1, 1.9]]
W2 = [0.6, 0.4]


def test_dic_sanity_gaussian():
    r = model_selection("gaussian", Y2, W2, 0, MODES2, np.full((2, 2), 0.1), p1=2.0, criteria=["dic"])
    assert np.isfinite(r["mean_deviance"]) and r["dic_p_eff"] >= 0.0
    assert abs(r["dic"] - (r["mean_deviance"] + r["dic_p_eff"])) < 1e-12
    assert np.isnan(r["waic"]) and r["cpo_failures"] is None


def test_waic_sanity_gaussian():
    r = model_selection("gaussian", Y2, W2, 0, MODES2, np.full((2, 2), 0.1), p1=2.0, criteria=["waic"])
    assert np.isfinite(r["waic"]) and np.isfinite(r["lppd"]) and r["waic_p_eff"] >= 0.0
    assert abs(r["waic"] + 2.0 * (r["lppd"] - r["waic_p_eff"])) < 1e-12
    assert np.isnan(r["dic"])


# --- model_selection.rs:628-672: the CPO failure heuristic ------------------------------------

def test_cpo_failure_detection_reference_cases():
    assert not cpo_failure("gaussian", 1.0, 1.0, 0.2, p1=2.0)          # stable: tau_loo = 3
    assert cpo_failure("gaussian", 1.0, 1.0, 0.6, p1=2.0)              # tau_loo < 0
    assert cpo_failure("gaussian", 0.0, 10.0, 0.1, p1=5.0)             # monotonic
    assert cpo_failure("poisson", 1.0, 0.0, 0.05, p1=10.0)             # border difference < 3
    for args in [("gaussian", 1.0, 1.0, 0.2, 2.0), ("gaussian", 1.0, 1.0, 0.6, 2.0),
                 ("gaussian", 0.0, 10.0, 0.1, 5.0), ("poisson", 1.0, 0.0, 0.05, 10.0)]:
        fam, y, mu, var, p1 = args
        assert cpo_failure(fam, y, mu, var, p1=p1) == O.cpo_failure(fam, y, p1, 1.0, mu, var)


def test_pit_cdf_none_for_negative_binomial():
    """model_selection.rs:675-725: families without a CDF give None."""
    assert observation_cdf("nbinomial", 1.0, 2.0, 0.0, 0.1) is None
    assert O.observation_cdf("nbinomial", 1.0, 2.0, 0.0, 0.1) is None


def test_cpo_pit_gaussian_well_specified():
    """model_selection.rs:727-766: 3 observations, 5 nodes; CPO > 0 and PIT in (0, 1)."""
    n, K = 3, 5
    y = [1.0 + 0.1 * i for i in range(n)]
    ce = [[1.0 + 0.1 * i + (k - 2.0) * 0.5 for i in range(n)] for k in range(K)]
    cv = [[0.5] * n for _ in range(K)]
    w = [0.1, 0.2, 0.4, 0.2, 0.1]
    r = model_selection("gaussian", y, w, 2, ce, cv, p1=2.0, criteria=["cpo"])
    for c, p in zip(r["cpo"], r["pit"]):
        assert np.isnan(c) or c > 0.0
        assert np.isnan(p) or 0.0 < p < 1.0
    cpo, pit, nf = O.compute_cpo_pit("gaussian", y, [2.0] * n, [1.0] * n, ce, cv, w)
    assert r["cpo_failures"] == nf
    np.testing.assert_allclose(r["cpo"], [np.nan if c is None else c for c in cpo], rtol=1e-13)
    np.testing.assert_allclose(r["pit"], [np.nan if p is None else p for p in pit], rtol=1e-13)


# --- model_selection.rs:768-792: the CDF helpers ------------------------------------------------

def test_cdf_helpers_reference_values():
    # normal: Gaussian observation with precision 1 and no latent variance, z = y - eta
    assert abs(observation_cdf("gaussian", 0.0, 1.0, 0.0, 0.0) - 0.5) < 1e-6
    assert observation_cdf("gaussian", 3.0, 1.0, 0.0, 0.0) > 0.998
    assert observation_cdf("gaussian", -3.0, 1.0, 0.0, 0.0) < 0.002
    # Poisson(1): exposure 1 at eta = 0
    assert abs(observation_cdf("poisson", 0.0, 1.0, 0.0, 0.0) - math.exp(-1.0)) < 1e-10
    assert observation_cdf("poisson", 10.0, 1.0, 0.0, 0.0) > 0.9999
    # Binomial(10, 0.5): eta = 0
    assert abs(observation_cdf("binomial", 10.0, 10.0, 0.0, 0.0) - 1.0) < 1e-10
    assert abs(observation_cdf("binomial", 4.0, 10.0, 0.0, 0.0) - 0.376953125) < 1e-8
    assert abs(O.binomial_cdf(10, 0.5, 4) - 0.376953125) < 1e-8
    assert abs(O.poisson_cdf(1.0, 0) - math.exp(-1.0)) < 1e-10


# --- every family against the oracle -------------------------------------------------------------

def _family_case(family, seed, nobs=60, K=7):
    rng = np.random.default_rng(seed)
    base = rng.normal(0.3, 0.8, nobs)
    p1 = p2 = None
    if family == "gaussian":
        y = base + rng.normal(0, 0.5, nobs)
        p1 = rng.uniform(1.0, 6.0, nobs)
    elif family == "poisson":
        p1 = rng.uniform(0.5, 3.0, nobs)
        y = rng.poisson(p1 * np.exp(base)).astype(float)
    elif family == "binomial":
        p1 = rng.integers(1, 20, nobs).astype(float)
        y = rng.binomial(p1.astype(int), 1 / (1 + np.exp(-base))).astype(float)
    else:
        p1 = np.full(nobs, 5.0)
        p2 = rng.uniform(0.5, 2.0, nobs)
        y = rng.poisson(p2 * np.exp(base)).astype(float)
    ce = base[None, :] + rng.normal(0, 0.15, (K, nobs))
    cv = rng.uniform(0.01, 0.4, (K, nobs))
    w = rng.uniform(0.2, 1.0, K)
    w[0] = -0.3 * w[1:].sum() / (K - 1)
    return y, p1, p2, w / w.sum(), ce, cv


@pytest.mark.parametrize("family", ["gaussian", "poisson", "binomial", "nbinomial"])
def test_criteria_match_oracle(family):
    y, p1, p2, w, ce, cv = _family_case(family, {"gaussian": 1, "poisson": 2, "binomial": 3, "nbinomial": 4}[family])
    r = model_selection(family, y, w, 0, ce, cv, p1=p1, p2=p2)
    q1 = p1 if p1 is not None else np.ones(len(y))
    q2 = p2 if p2 is not None else np.ones(len(y))
    dic = O.compute_dic(family, y, q1, q2, ce, w, 0)
    waic = O.compute_waic(family, y, q1, q2, ce, w)
    for key, ref in [("dic", dic["dic"]), ("mean_deviance", dic["mean_deviance"]), ("dic_p_eff", dic["p_eff"]),
                     ("waic", waic["waic"]), ("lppd", waic["lppd"]), ("waic_p_eff", waic["p_eff"])]:
        assert abs(r[key] - ref) <= 1e-12 * max(1.0, abs(ref)), key
    cpo, pit, nf = O.compute_cpo_pit(family, y, q1, q2, ce, cv, w)
    assert r["cpo_failures"] == nf
    assert nf < len(y)
    np.testing.assert_allclose(r["cpo"], [np.nan if c is None else c for c in cpo], rtol=1e-12)
    np.testing.assert_allclose(r["pit"], [np.nan if p is None else p for p in pit], rtol=1e-12)
    if family == "nbinomial":
        assert np.all(np.isnan(r["pit"]))


def test_single_node_fails_every_cpo_and_errors_propagate():
    """K = 1: every CPO fails (model_selection.rs:270-273); a likelihood that cannot be
    evaluated (negative Poisson count) is the reference's DIC error."""
    r = model_selection("gaussian", Y2, [1.0], 0, [MODES2[0]], [[0.1, 0.1]], p1=2.0)
    assert r["cpo_failures"] == 2 and np.all(np.isnan(r["cpo"]))
    with pytest.raises(InlaError, match="DIC"):
        model_selection("poisson", [-1.0, 2.0], W2, 0, MODES2, np.full((2, 2), 0.1))
    with pytest.raises(InlaError):
        model_selection("gaussian", Y2, W2, 2, MODES2, np.full((2, 2), 0.1), p1=2.0)   # mode index out of range


def test_compute_flags_skip_criteria():
    """inference.rs compute_flags_skip_dic_waic_cpo: criteria not asked for stay NaN / None."""
    r = model_selection("gaussian", Y2, W2, 0, MODES2, np.full((2, 2), 0.1), p1=2.0, criteria=[])
    assert np.isnan(r["dic"]) and np.isnan(r["waic"]) and r["cpo_failures"] is None
    assert np.all(np.isnan(r["cpo"])) and np.all(np.isnan(r["pit"]))
