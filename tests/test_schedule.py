"""Host check of the persistent factorization schedule (no GPU): for the patterns the engines
run (SPDE meshes under nested dissection and AMD, the Besag (x) AR1 group model, a dense
block, grids with fronts of every size class, a block-diagonal many-model pattern), walking
the task queue in order finds every task's dependencies complete when the task is reached and
every front complete at the end -- the property that lets the GPU's smallest unfinished task
always run -- and every table index in range."""
import ctypes as C
import math

import numpy as np
import pytest
import scipy.sparse as sp

from fixtures import grid_laplacian, random_spd
from inla_b200 import GpuSolver, _lib, models


def check(q, ordering):
    s = GpuSolver(ordering)
    s.analyze(q)
    info = np.zeros(3, dtype=np.int64)
    rc = _lib.lib().inla_solver_check_schedule(s._h, _lib.lptr(info))
    assert rc == _lib.INLA_OK, _lib.lib().inla_last_error()
    return info


def spde_post(nx):
    p = models.make_spde_problem(nx=nx, n_obs=nx * nx // 2)
    c, _ = models.spde_coefs(math.log(0.02), math.log(14.14))
    return (p.model.matrix(c) + 100.0 * (p.a.T @ p.a)).tocsc()


@pytest.mark.parametrize("ordering", [_lib.ORDER_ND, _lib.ORDER_AMD])
@pytest.mark.parametrize("nx", [30, 100, 200])
def test_spde_schedules(nx, ordering):
    info = check(spde_post(nx), ordering)
    assert info[0] > 0 and info[2] == 1 and info[1] <= 227 * 1024


def test_group_model_schedule():
    p = models.make_group_problem(nr=20, nc=20, T=10)
    info = check(p.model.pattern, _lib.ORDER_ND)
    assert info[2] == 1


@pytest.mark.parametrize("q", [grid_laplacian(70, 50, ridge=0.3), random_spd(400, 0.02, 3),
                               sp.csc_matrix(np.ones((150, 150)) + 150 * np.eye(150))],
                         ids=["grid", "random", "dense"])
def test_other_schedules(q):
    check(sp.csc_matrix(q), _lib.ORDER_ND)


def test_block_diagonal_schedule():
    blocks = [grid_laplacian(8 + i, 7, ridge=0.5) for i in range(12)]
    check(sp.block_diag(blocks).tocsc(), _lib.ORDER_ND)


def test_schedule_setters_reject_out_of_range_values():
    """The process-wide schedule choices (no device needed): persistent-schedule mode 0..2 and
    panel form -1..2 are accepted, anything else is INLA_ERR_INVALID and leaves the setting as it was."""
    lib = _lib.lib()
    for bad in (-1, 3):
        assert lib.inla_set_persistent_schedule(bad) == _lib.INLA_ERR_INVALID
    for bad in (-2, 3, 100):
        assert lib.inla_set_panel_form(bad) == _lib.INLA_ERR_INVALID
        assert "panel form" in lib.inla_last_error().decode()
    for ok in (0, 1, 2, -1):
        assert lib.inla_set_panel_form(ok) == _lib.INLA_OK
    assert lib.inla_set_persistent_schedule(1) == _lib.INLA_OK
