"""Linear-predictor moments of the integration mixture (host code of the library, no GPU):
``inla_predictor_moments`` against the oracle's restatement of matvec_csc /
predictor_variances_diag (design.rs:52-70, 198-210) and the mixture (inference.rs:1436-1466)."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from inla_b200 import InlaError
from inla_b200.laplace import predictor_moments


def _case(seed, nobs, n, K, zero_frac=0.1):
    rng = np.random.default_rng(seed)
    a = sp.random(nobs, n, density=min(1.0, 3.0 / n), random_state=rng, format="csr")
    a.data = rng.uniform(0.0, 1.0, a.nnz)
    cm = rng.normal(size=(K, n))
    cm[rng.random((K, n)) < zero_frac] = 0.0   # matvec_csc skips x_j == 0
    cv = rng.uniform(0.01, 2.0, size=(K, n))
    w = rng.uniform(0.1, 1.0, K)
    w[0] = -0.68                                # CCD centre weight for m = 3, f0 = 1
    return a, w / w.sum(), cm, cv


@pytest.mark.parametrize("seed,nobs,n,K", [(0, 50, 40, 3), (1, 400, 900, 15), (2, 2000, 1500, 25)])
def test_predictor_moments_match_oracle_bitwise(seed, nobs, n, K):
    a, w, cm, cv = _case(seed, nobs, n, K)
    pm, pv = predictor_moments(a, w, cm, cv)
    om, ov = O.predictor_moments(a, w, cm, cv)
    np.testing.assert_array_equal(pm, om)
    np.testing.assert_array_equal(pv, ov)


def test_identity_projector_mixes_the_latent_moments():
    """No A: eta = x* and its variance is the latent variance (projection.rs:132-143)."""
    _, w, cm, cv = _case(3, 10, 64, 5)
    pm, pv = predictor_moments(None, w, cm, cv)
    om, ov = O.mixture_moments(w, cm, cv)
    np.testing.assert_array_equal(pm, om)
    np.testing.assert_array_equal(pv, ov)
    pm1, pv1 = predictor_moments(None, [1.0], [[1.0, 2.0, 3.0, 4.0]], [[0.1, 0.2, 0.3, 0.4]])
    np.testing.assert_array_equal(pm1, [1.0, 2.0, 3.0, 4.0])
    np.testing.assert_array_equal(pv1, [0.1, 0.2, 0.3, 0.4])


def test_single_node_is_the_projection():
    """One node of weight 1: mean = A x, var = (A o A) var, with A x dense-checked."""
    a, _, cm, cv = _case(4, 300, 200, 1, zero_frac=0.0)
    pm, pv = predictor_moments(a, [1.0], cm, cv)
    np.testing.assert_allclose(pm, a @ cm[0], rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(pv, a.multiply(a) @ cv[0], rtol=1e-14, atol=1e-15)


def test_empty_rows_and_no_observations():
    a = sp.csr_matrix((5, 4))
    pm, pv = predictor_moments(a, [0.5, 0.5], np.ones((2, 4)), np.ones((2, 4)))
    np.testing.assert_array_equal(pm, 0.0)
    np.testing.assert_array_equal(pv, 0.0)
    pm, pv = predictor_moments(sp.csr_matrix((0, 4)), [1.0], np.ones((1, 4)), np.ones((1, 4)))
    assert pm.shape == (0,) and pv.shape == (0,)


def test_invalid_arguments_raise():
    with pytest.raises(ValueError):
        predictor_moments(sp.eye(3, 4), [1.0], np.ones((1, 3)), np.ones((1, 3)))
    with pytest.raises(InlaError):
        predictor_moments(None, np.ones(0), np.ones((0, 3)), np.ones((0, 3)))   # K = 0


def test_oracle_integrate_carries_the_predictor():
    """The oracle's node aggregation with a projector: the predictor mixture mean is A times the
    latent mixture mean, and its variance is the library's on the same node results."""
    rng = np.random.default_rng(5)
    a = sp.random(30, 20, density=0.15, random_state=rng, format="csr")
    base = rng.normal(size=20)
    nodes = []

    def node(theta):
        x = base * (1.0 + 0.1 * theta.sum())
        v = np.full(20, 0.5 + 0.05 * theta[0] ** 2)
        nodes.append((x, v))
        return x, v, -0.5 * float(theta @ theta)

    r = O.integrate(np.zeros(2), -np.eye(2), node, f0=1.0, a=a)
    np.testing.assert_allclose(r["pred_mean"], a @ r["mean"], rtol=1e-12, atol=1e-14)
    cm = np.stack([nodes[i][0] for i in range(len(r["weights"]))])
    cv = np.stack([nodes[i][1] for i in range(len(r["weights"]))])
    pm, pv = predictor_moments(a, r["weights"], cm, cv)
    np.testing.assert_array_equal(pm, r["pred_mean"])
    np.testing.assert_array_equal(pv, r["pred_var"])
