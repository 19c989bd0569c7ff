"""One-dimensional marginals (host code of the library, no GPU): the reference's tests of
crates/inla_stats/src/marginals.rs:236-271 and bitwise parity with the oracle's restatement."""
import math

import numpy as np
import pytest

import oracle as O
from inla_b200 import InlaError
from inla_b200.laplace import hyperpar_marginal, marginal_quantiles, mixture_marginal


def test_standard_normal_quantiles():
    """marginals.rs:237-255: a normalised N(0, 1) grid of 401 points on [-5, 5]."""
    x = -5.0 + 10.0 * np.arange(401) / 400.0
    y = np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)
    q025, q50, q975 = marginal_quantiles(x, y)
    assert abs(q50) < 0.05 and abs(q025 + 1.96) < 0.08 and abs(q975 - 1.96) < 0.08


def test_mixture_matches_closed_form_moments():
    """marginals.rs:257-270: equal mixture of N(0, 1) and N(2, 1) on 201 points over 5 sd."""
    x, y = mixture_marginal([0.0, 2.0], [1.0, 1.0], [0.5, 0.5], 201, 5.0)
    dx = np.diff(x)
    assert abs(np.sum(0.5 * (y[:-1] + y[1:]) * dx) - 1.0) < 1e-3
    ex = np.sum(0.5 * (x[:-1] * y[:-1] + x[1:] * y[1:]) * dx)
    assert abs(ex - 1.0) < 0.05


def test_marginals_match_oracle_bitwise():
    rng = np.random.default_rng(21)
    K = 15
    w = rng.uniform(0.1, 1.0, K)
    w[0] = -0.68 * w[1:].sum() / (K - 1)
    w = w / w.sum()
    means, vars_ = rng.normal(size=K), rng.uniform(0.05, 0.5, K)
    x, y = mixture_marginal(means, vars_, w)
    xo, yo = O.gaussian_mixture_marginal(list(means), list(vars_), list(w))
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_array_equal(y, yo)
    theta = rng.normal(size=K)
    x, y = hyperpar_marginal(theta, w, n_points=101, n_sd=3.0)
    xo, yo = O.hyperpar_marginal_from_nodes(list(theta), list(w), 101, 3.0)
    np.testing.assert_array_equal(x, xo)
    np.testing.assert_array_equal(y, yo)
    probs = [0.01, 0.025, 0.25, 0.5, 0.75, 0.975, 0.99]
    np.testing.assert_array_equal(marginal_quantiles(x, y, probs), O.marginal_quantiles(list(x), list(y), probs))


def test_degenerate_mixture_uses_the_variance_floor_and_errors():
    x, y = hyperpar_marginal([0.3, 0.3, 0.3], [0.2, 0.5, 0.3], n_points=11)
    assert abs(x[-1] - x[0] - 2 * 4.0 * 1e-4) < 1e-15       # sd = sqrt(1e-8)
    with pytest.raises(InlaError, match="n_points"):
        mixture_marginal([0.0], [1.0], [1.0], n_points=4)
    with pytest.raises(InlaError, match="probability"):
        marginal_quantiles([0.0, 1.0], [1.0, 1.0], [1.0])
