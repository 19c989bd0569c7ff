"""The persistent factorization schedule (one launch per batched factorization, a task queue
in elimination-tree order) against the level-by-level launches: the same log-determinants,
solutions and selected inverses bit for bit, on the SPDE posterior precision (large fronts
with several 64-column blocks) and on batches that mix fronts of every size class. The
bounded dependency waits are exercised by a launch whose completion counts can never be
reached: it must end with the timeout code, and the handle must factorize correctly after."""
import math

import numpy as np
import pytest

import oracle as O
from fixtures import grid_laplacian
from inla_b200 import BatchSolver, _lib, models

pytestmark = pytest.mark.gpu


def make(q, B, persistent, ordering=_lib.ORDER_ND):
    _lib.check(_lib.lib().inla_set_persistent_schedule(2 if persistent else 0))
    try:
        bs = BatchSolver(q, max_batch=B, ordering=ordering)
    finally:
        _lib.check(_lib.lib().inla_set_persistent_schedule(1))
    import ctypes as C

    flag = C.c_int(-1)
    _lib.check(_lib.lib().inla_batch_schedule(bs._h, C.byref(flag)))
    assert flag.value == (1 if persistent else 0)
    return bs


def spde_post(nx):
    p = models.make_spde_problem(nx=nx, n_obs=nx * nx // 2)
    c, _ = models.spde_coefs(math.log(0.02), math.log(14.14))
    q = (p.model.matrix(c) + 100.0 * (p.a.T @ p.a)).tocsc()
    q.sort_indices()
    return q


@pytest.mark.parametrize("nx,B", [(60, 1), (100, 3), (200, 4)])
def test_persistent_equals_level_launches_bitwise(nx, B):
    q = spde_post(nx)
    rng = np.random.default_rng(nx)
    diag = np.array([q.indices[p] == c for c in range(q.shape[0]) for p in range(q.indptr[c], q.indptr[c + 1])])
    vals = np.tile(q.data, (B, 1))
    vals[:, diag] += rng.uniform(0.0, 1.0, size=(B, diag.sum()))
    rhs = rng.standard_normal((B, q.shape[0]))
    out = {}
    for persistent in (True, False):
        bs = make(q, B, persistent)
        ld, st = bs.factorize(vals)
        assert np.all(st == 0)
        out[persistent] = (ld, bs.solve(rhs), bs.diag_inv())
        bs.factorize(vals)  # a second factorization replays the captured launch sequence
        np.testing.assert_array_equal(bs.solve(rhs), out[persistent][1])
        bs.close()
    for a, b in zip(out[True], out[False]):
        np.testing.assert_array_equal(a, b)
    if nx <= 100:
        qk = q.copy()
        qk.data = vals[0]
        f = O.Factor(qk, perm=O.reference_perm(qk))
        assert abs(out[True][0][0] - f.logdet()) <= 1e-10 * abs(f.logdet())


def test_mixed_front_sizes_persistent_equals_levels():
    q = grid_laplacian(70, 50, ridge=0.3)
    B = 5
    vals = np.stack([q.data * (1.0 + 0.1 * k) for k in range(B)])
    res = []
    for persistent in (True, False):
        bs = make(q, B, persistent)
        ld, st = bs.factorize(vals)
        res.append((ld, bs.diag_inv()))
        bs.close()
    np.testing.assert_array_equal(res[0][0], res[1][0])
    np.testing.assert_array_equal(res[0][1], res[1][1])


def test_wait_limit_ends_the_launch_and_the_handle_recovers():
    import ctypes as C

    q = spde_post(60)
    bs = make(q, 2, True)
    code = C.c_int(0)
    _lib.check(_lib.lib().inla_batch_wait_limit_selftest(bs._h, 50.0, C.byref(code)))
    assert code.value == 1  # a dependency wait ran out and the launch ended
    ld, st = bs.factorize(np.tile(q.data, (2, 1)))
    assert np.all(st == 0)
    f = O.Factor(q, perm=O.reference_perm(q))
    assert abs(ld[0] - f.logdet()) <= 1e-10 * abs(f.logdet())
    bs.close()
