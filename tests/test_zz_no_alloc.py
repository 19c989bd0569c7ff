"""The allocation-free dense LDL^T entry point, through the C ABI.

``inla_dense_ldlt_solve_noalloc`` is for callers that own all device memory
and cannot let the library call cudaMalloc: they pass device buffers for the
matrix, right-hand side and results, and the factor is kept in a fixed static
device scratch (n <= 1024). Its results must match the allocating entry
points (``inla_solver_factorize`` / ``solve`` / ``log_abs_det``) on the same
matrix within the tolerances the other GPU tests use (log-det 1e-10
relative, solution 1e-8 relative plus a 1e-14 backward error), on two calls
in a row, since consecutive calls share the scratch.

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


def call_noalloc(q, b):
    import torch

    n = q.shape[0]
    dq = torch.tensor(np.asfortranarray(q).ravel(order="F"), dtype=torch.float64, device="cuda")
    db = torch.tensor(b, dtype=torch.float64, device="cuda")
    dx = torch.zeros(n, dtype=torch.float64, device="cuda")
    dld = torch.zeros(1, dtype=torch.float64, device="cuda")
    dst = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib().inla_dense_ldlt_solve_noalloc(n, C.c_void_p(dq.data_ptr()), C.c_void_p(db.data_ptr()),
                                                   C.c_void_p(dx.data_ptr()), C.c_void_p(dld.data_ptr()),
                                                   C.c_void_p(dst.data_ptr()), C.c_void_p(stream))
    _lib.check(rc)
    torch.cuda.synchronize()
    return dx.cpu().numpy(), float(dld.item()), int(dst.item())


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
        assert np.max(np.abs(x - x_ref)) <= 1e-8 * np.max(np.abs(x_ref))
        r = q @ x - b
        assert np.max(np.abs(r)) / (np.max(np.abs(q).sum(axis=1)) * np.max(np.abs(x)) + np.max(np.abs(b))) < 1e-14


def test_noalloc_rejects_sizes_beyond_the_limit():
    rc = _lib.lib().inla_dense_ldlt_solve_noalloc(1025, C.c_void_p(1), None, None, C.c_void_p(1), C.c_void_p(1),
                                                   None)
    assert rc == _lib.INLA_ERR_DIM_MISMATCH
    assert b"no-allocation limit" in _lib.lib().inla_last_error()
