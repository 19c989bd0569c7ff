"""The allocation-free dense LDL^T entry point, through the C ABI.

``inla_dense_ldlt_solve_noalloc`` is for callers that own all device memory
and cannot let the library call cudaMalloc (pool allocators, plugins handed
fixed buffers, code running while other work is captured): they pass device
buffers for the matrix, right-hand side and results, and the factor is kept
in a fixed static device scratch (n <= 1024). Its results must match the
allocating entry points (``inla_solver_factorize`` / ``solve`` /
``log_abs_det``) on the same matrix within the tolerances the other GPU tests
use (log-det 1e-10 relative, solution 1e-8 relative plus a 1e-14 backward
error), on two calls in a row, since consecutive calls share the scratch.
The log-determinant is also checked against numpy's LAPACK ``slogdet``, which
shares no code with this library.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from inla_b200 import GpuSolver, _lib

pytestmark = pytest.mark.gpu


def spd(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    return a @ a.T / n + np.eye(n)


def enqueue(q, b, stream):
    """Queue one call on ``stream`` without synchronizing; returns the device buffers."""
    import torch

    n = q.shape[0]
    bufs = {
        "q": torch.tensor(np.asfortranarray(q).ravel(order="F"), dtype=torch.float64, device="cuda"),
        "b": None if b is None else torch.tensor(b, dtype=torch.float64, device="cuda"),
        "x": None if b is None else torch.zeros(n, dtype=torch.float64, device="cuda"),
        "ld": torch.zeros(1, dtype=torch.float64, device="cuda"),
        "st": torch.full((1,), -1, dtype=torch.int32, device="cuda"),
    }
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    torch.cuda.synchronize()  # the inputs above are written before the library's stream reads them
    rc = _lib.lib().inla_dense_ldlt_solve_noalloc(n, ptr(bufs["q"]), ptr(bufs["b"]), ptr(bufs["x"]),
                                                   ptr(bufs["ld"]), ptr(bufs["st"]), C.c_void_p(stream))
    _lib.check(rc)
    return bufs


def results(bufs):
    import torch

    torch.cuda.synchronize()
    x = None if bufs["x"] is None else bufs["x"].cpu().numpy()
    return x, float(bufs["ld"].item()), int(bufs["st"].item())


def call_noalloc(q, b):
    import torch

    return results(enqueue(q, b, torch.cuda.current_stream().cuda_stream))


def backward_error(q, x, b):
    r = q @ x - b
    return np.max(np.abs(r)) / (np.max(np.abs(q).sum(axis=1)) * np.max(np.abs(x)) + np.max(np.abs(b)))


def test_noalloc_matches_allocating_entry_point_twice():
    for n, seed in ((300, 11), (1024, 12)):  # two calls in a row share the scratch
        q = spd(n, seed)
        b = np.sin(np.arange(n) * 0.3) + 0.5
        ref = GpuSolver()
        ref.factorize(sp.csc_matrix(q))
        ld_ref, x_ref = ref.log_abs_det(), ref.solve(b)
        x, ld, status = call_noalloc(q, b)
        assert status == 0
        assert abs(ld - ld_ref) <= 1e-10 * abs(ld_ref)
        sign, ld_np = np.linalg.slogdet(q)
        assert sign > 0 and abs(ld - ld_np) <= 1e-10 * abs(ld_np)
        assert np.max(np.abs(x - x_ref)) <= 1e-8 * np.max(np.abs(x_ref))
        assert backward_error(q, x, b) < 1e-14


def test_noalloc_calls_queued_back_to_back_on_one_stream():
    """Calls on one stream run in order: the second overwrites the scratch only after the first
    has read it, so both results are right although nothing synchronizes between them."""
    import torch

    stream = torch.cuda.current_stream().cuda_stream
    qa, qb = spd(700, 21), spd(257, 22)
    ba, bb = np.linspace(-1.0, 1.0, 700), np.cos(np.arange(257.0))
    first = enqueue(qa, ba, stream)
    second = enqueue(qb, bb, stream)
    xa, lda, sa = results(first)
    xb, ldb, sb = results(second)
    assert sa == 0 and sb == 0
    assert abs(lda - np.linalg.slogdet(qa)[1]) <= 1e-10 * abs(lda)
    assert abs(ldb - np.linalg.slogdet(qb)[1]) <= 1e-10 * abs(ldb)
    assert backward_error(qa, xa, ba) < 1e-14 and backward_error(qb, xb, bb) < 1e-14


def test_noalloc_reports_a_singular_matrix():
    """A zero last row and column leaves a zero pivot: the status word is nonzero (|D| < 1e-14,
    sparse_ldlt.rs:104-149)."""
    n = 64
    q = spd(n, 31)
    q[-1, :] = 0.0
    q[:, -1] = 0.0
    _, _, status = call_noalloc(q, None)
    assert status != 0
    # the scratch holds the singular factor now; the next call starts from its own input
    q2 = spd(n, 32)
    x, ld, status = call_noalloc(q2, np.ones(n))
    assert status == 0 and abs(ld - np.linalg.slogdet(q2)[1]) <= 1e-10 * abs(ld)


def test_noalloc_rejects_sizes_beyond_the_limit():
    rc = _lib.lib().inla_dense_ldlt_solve_noalloc(1025, C.c_void_p(1), None, None, C.c_void_p(1), C.c_void_p(1),
                                                   None)
    assert rc == _lib.INLA_ERR_DIM_MISMATCH
    assert b"no-allocation limit" in _lib.lib().inla_last_error()
