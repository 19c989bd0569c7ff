"""The three panel forms of the level launches (split, fused, look-ahead: the trailing update's
first tile factors the next 64 x 64 diagonal block) give the same log-determinants, solutions
and selected inverses bit for bit, on the SPDE posterior precision (fronts with many 64-column
blocks, including a last block narrower than 64) and on a lattice whose levels mix front sizes;
the look-ahead factorization also matches the oracle."""
import math

import numpy as np
import pytest

import oracle as O
from fixtures import grid_laplacian
from inla_b200 import BatchSolver, _lib, models

pytestmark = pytest.mark.gpu

FORMS = {"split": 0, "fused": 1, "lookahead": 2}


def make(q, B, form, ordering=_lib.ORDER_ND):
    lib = _lib.lib()
    _lib.check(lib.inla_set_persistent_schedule(0))
    _lib.check(lib.inla_set_panel_form(form))
    try:
        return BatchSolver(q, max_batch=B, ordering=ordering)
    finally:
        _lib.check(lib.inla_set_panel_form(-1))
        _lib.check(lib.inla_set_persistent_schedule(1))


def spde_post(nx):
    p = models.make_spde_problem(nx=nx, n_obs=nx * nx // 2)
    c, _ = models.spde_coefs(math.log(0.02), math.log(14.14))
    q = (p.model.matrix(c) + 100.0 * (p.a.T @ p.a)).tocsc()
    q.sort_indices()
    return q


def run_forms(q, vals, rhs):
    out = {}
    for name, form in FORMS.items():
        bs = make(q, vals.shape[0], form)
        ld, st = bs.factorize(vals)
        assert np.all(st == 0), name
        out[name] = (ld, bs.solve(rhs), bs.diag_inv())
        bs.factorize(vals)  # replay of the captured sequence
        np.testing.assert_array_equal(bs.solve(rhs), out[name][1])
        bs.close()
    for name in ("fused", "lookahead"):
        for a, b in zip(out["split"], out[name]):
            np.testing.assert_array_equal(a, b, err_msg=name)
    return out


@pytest.mark.parametrize("nx,B", [(60, 2), (120, 3), (200, 2)])
def test_panel_forms_bitwise_spde(nx, B):
    q = spde_post(nx)
    rng = np.random.default_rng(7 * nx)
    diag = np.array([q.indices[p] == c for c in range(q.shape[0]) for p in range(q.indptr[c], q.indptr[c + 1])])
    vals = np.tile(q.data, (B, 1))
    vals[:, diag] += rng.uniform(0.0, 1.0, size=(B, diag.sum()))
    rhs = rng.standard_normal((B, q.shape[0]))
    out = run_forms(q, vals, rhs)
    if nx <= 60:
        qk = q.copy()
        qk.data = vals[1]
        f = O.Factor(qk, perm=O.reference_perm(qk))
        assert abs(out["lookahead"][0][1] - f.logdet()) <= 1e-10 * abs(f.logdet())
        np.testing.assert_allclose(out["lookahead"][2][1], f.diag_inv(), rtol=1e-9)


def test_panel_forms_bitwise_mixed_fronts():
    q = grid_laplacian(70, 50, ridge=0.3)
    B = 4
    vals = np.stack([q.data * (1.0 + 0.1 * k) for k in range(B)])
    rhs = np.random.default_rng(3).standard_normal((B, q.shape[0]))
    run_forms(q, vals, rhs)
