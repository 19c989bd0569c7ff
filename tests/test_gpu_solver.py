"""GPU parity of the supernodal LDL^T / solve / log-det / Takahashi path
against the committed golden vectors and the CPU oracle, through the C ABI.

Tolerances (FP64): log-det 1e-10 relative, solves 1e-12 relative to |x|_inf,
selected-inverse entries 1e-8 relative.
"""
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from fixtures import KNOWN_ANSWER, ar1_q, grid_laplacian, random_spd
from inla_b200 import BatchSolver, GpuSolver, _lib, models

pytestmark = pytest.mark.gpu

GOLDEN = np.load(Path(__file__).parent / "golden" / "golden.npz")
LOGDET_RTOL = 1e-10
SOLVE_RTOL = 1e-12
SIGMA_RTOL = 1e-8


def golden_matrix(name):
    n = len(GOLDEN[f"{name}/indptr"]) - 1
    return sp.csc_matrix((GOLDEN[f"{name}/data"], GOLDEN[f"{name}/indices"], GOLDEN[f"{name}/indptr"]), shape=(n, n))


def rel(a, b):
    return np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300)


def backward_error(q, x, b):
    """|Qx - b|_inf / (|Q|_inf |x|_inf + |b|_inf): FP64 solves reach ~1e-16 regardless of conditioning."""
    r = q @ x - b
    qn = np.max(np.asarray(abs(q).sum(axis=1)).ravel())
    return np.max(np.abs(r)) / (qn * np.max(np.abs(x)) + np.max(np.abs(b)))


@pytest.mark.parametrize("name", sorted({k.split("/")[0] for k in GOLDEN.files}))
@pytest.mark.parametrize("ordering", [_lib.ORDER_AMD, _lib.ORDER_REFERENCE, _lib.ORDER_NATURAL, _lib.ORDER_ND])
def test_golden_known_answers(name, ordering):
    q = golden_matrix(name)
    s = GpuSolver(ordering)
    s.factorize(q)
    ld = GOLDEN[f"{name}/logdet"][0]
    assert abs(s.log_abs_det() - ld) <= LOGDET_RTOL * max(1.0, abs(ld))
    b = np.arange(1, q.shape[0] + 1, dtype=float)
    assert rel(s.solve(b), GOLDEN[f"{name}/solve"]) < 1e-11
    tol = KNOWN_ANSWER[name][1] if name in KNOWN_ANSWER else 1e-10
    assert np.max(np.abs(s.diag_inv() - GOLDEN[f"{name}/diag_inv"])) < tol


def dense_spd(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.standard_normal((n, n))
    m = a @ a.T / n + np.eye(n)
    return sp.csc_matrix(m)


CASES = {
    "ar1_500": lambda: ar1_q(500, 0.9, 3.0),
    "grid_40x40": lambda: grid_laplacian(40, 40, ridge=0.2),
    "grid_90x70": lambda: grid_laplacian(90, 70, ridge=0.05),
    "random_400": lambda: random_spd(400, 0.02, 3),
    "dense_300": lambda: dense_spd(300, 5),
    "dense_130": lambda: dense_spd(130, 6),
    "spde_40": lambda: models.make_spde_problem(nx=40, n_obs=800).model.matrix([1.0, 2.0, 0.5]),
    "spde_70_post": lambda: _spde_post(70),
}


def _spde_post(nx):
    p = models.make_spde_problem(nx=nx, n_obs=nx * nx // 2)
    c, _ = models.spde_coefs(-1.0, 1.5)
    q = p.model.matrix(c)
    return (q + 50.0 * (p.a.T @ p.a)).tocsc()


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("ordering", [_lib.ORDER_AMD, _lib.ORDER_REFERENCE, _lib.ORDER_ND])
def test_factor_solve_selinv_vs_oracle(name, ordering):
    q = sp.csc_matrix(CASES[name]())
    q.sort_indices()
    n = q.shape[0]
    f = O.Factor(q, perm=O.default_perm(q))
    s = GpuSolver(ordering)
    s.factorize(q)
    ld = f.logdet()
    assert abs(s.log_abs_det() - ld) <= LOGDET_RTOL * abs(ld)
    b = np.sin(np.arange(n) * 0.37) + 0.1
    x_ref = f.solve(b)
    x = s.solve(b)
    assert backward_error(q, x, b) < 1e-14
    assert rel(x, x_ref) < SIGMA_RTOL
    d_ref = f.diag_inv()
    assert rel(s.diag_inv(), d_ref) < SIGMA_RTOL
    sig_ref = f.sigma_on_pattern(q)
    sig = s.selinv_pattern()
    assert rel(sig, sig_ref) < SIGMA_RTOL


def test_numeric_refactor_reuses_symbolic():
    """scratch.rs:90-103: identical pattern => numeric-only; new values give new results."""
    q = grid_laplacian(30, 30, ridge=0.5)
    s = GpuSolver()
    s.factorize(q)
    p1 = s.perm().copy()
    ld1 = s.log_abs_det()
    q2 = q.copy()
    q2.data = q2.data * 2.0
    s.factorize(q2)
    np.testing.assert_array_equal(s.perm(), p1)
    assert abs(s.log_abs_det() - (ld1 + q.shape[0] * np.log(2.0))) < 1e-9 * abs(ld1)


def test_batch_matches_single():
    q = grid_laplacian(50, 40, ridge=0.3)
    B = 5
    rng = np.random.default_rng(0)
    vals = np.stack([q.data * (1.0 + 0.5 * k) + 0.0 for k in range(B)])
    # perturb diagonal per problem so problems differ beyond scaling
    diag = np.array([q.indices[p] == c for c in range(q.shape[0]) for p in range(q.indptr[c], q.indptr[c + 1])])
    vals[:, diag] += rng.uniform(0.0, 1.0, size=(B, diag.sum()))
    bs = BatchSolver(q, max_batch=8)
    ld, st = bs.factorize(vals)
    assert np.all(st == 0)
    rhs = rng.standard_normal((B, q.shape[0]))
    xs = bs.solve(rhs)
    dg = bs.diag_inv()
    for k in range(B):
        qk = q.copy()
        qk.data = vals[k]
        f = O.Factor(qk, perm=O.default_perm(qk))
        assert abs(ld[k] - f.logdet()) <= LOGDET_RTOL * abs(f.logdet())
        assert backward_error(qk, xs[k], rhs[k]) < 1e-14
        assert rel(xs[k], f.solve(rhs[k])) < SIGMA_RTOL
        assert rel(dg[k], f.diag_inv()) < SIGMA_RTOL


def test_batch_throughput_path_matches_oracle():
    """A batch large enough that the level kernels switch to their throughput
    layout (one diagonal-block factorization per front and problem, rows formed
    by a separate launch) still matches the oracle problem by problem."""
    import math

    p = models.make_spde_problem(nx=100, n_obs=5000)
    c, _ = models.spde_coefs(math.log(0.02), math.log(14.14))
    q = (p.model.matrix(c) + 100.0 * (p.a.T @ p.a)).tocsc()
    q.sort_indices()
    B = 12
    scale = 1.0 + 0.25 * np.arange(B)
    vals = np.stack([q.data * sc for sc in scale])
    bs = BatchSolver(q, max_batch=B, ordering=_lib.ORDER_ND)
    ld, st = bs.factorize(vals)
    assert np.all(st == 0)
    rng = np.random.default_rng(3)
    rhs = rng.standard_normal((B, q.shape[0]))
    xs = bs.solve(rhs)
    dg = bs.diag_inv()
    f = O.Factor(q, perm=O.default_perm(q))
    ld0, d0 = f.logdet(), f.diag_inv()
    n = q.shape[0]
    for k in (0, B // 2, B - 1):
        # Q_k = scale_k Q: log|Q_k| = log|Q| + n log(scale_k), diag(Q_k^-1) = diag(Q^-1) / scale_k
        ref = ld0 + n * np.log(scale[k])
        assert abs(ld[k] - ref) <= LOGDET_RTOL * abs(ref)
        qk = q * scale[k]
        assert backward_error(qk, xs[k], rhs[k]) < 1e-14
        assert rel(dg[k], d0 / scale[k]) < SIGMA_RTOL


def test_singular_matrix_reports_singular():
    """Zero pivot => SolverError::Singular (sparse_ldlt.rs:117-120)."""
    q = sp.csc_matrix(np.array([[1.0, 1.0, 0.0], [1.0, 1.0, 0.0], [0.0, 0.0, 2.0]]))
    s = GpuSolver(_lib.ORDER_NATURAL)
    with pytest.raises(_lib.InlaError) as e:
        s.factorize(q)
    assert e.value.code == _lib.INLA_ERR_SINGULAR
    with pytest.raises(_lib.InlaError) as e:
        s.solve(np.ones(3))
    assert e.value.code == _lib.INLA_ERR_NOT_FACTORED


def test_nonfinite_values_report_singular():
    q = grid_laplacian(8, 8)
    # a lower-triangle entry (entries with row < col are never read, as in the reference)
    col = 5
    p = q.indptr[col] + int(np.searchsorted(q.indices[q.indptr[col]:q.indptr[col + 1]], col))
    q.data[p] = np.nan
    s = GpuSolver()
    with pytest.raises(_lib.InlaError) as e:
        s.factorize(q)
    assert e.value.code == _lib.INLA_ERR_SINGULAR


def test_deterministic_bitwise():
    q = _spde_post(50)
    a, b = GpuSolver(), GpuSolver()
    a.factorize(q)
    b.factorize(q)
    assert a.log_abs_det() == b.log_abs_det()
    r = np.cos(np.arange(q.shape[0]))
    np.testing.assert_array_equal(a.solve(r), b.solve(r))
    np.testing.assert_array_equal(a.diag_inv(), b.diag_inv())


def test_small_handle_built_later_does_not_break_a_large_one():
    """Two engines in one process: a large-front engine, then a small one, then a first
    factorization and solve of the large engine at a batch size it has not launched yet
    (a new captured launch sequence). The sweep kernels' shared-memory limit must still
    admit the large engine's fronts."""
    import math

    p = models.make_spde_problem(nx=60, n_obs=1800)
    c, _ = models.spde_coefs(math.log(0.05), math.log(10.0))
    q = (p.model.matrix(c) + 40.0 * (p.a.T @ p.a)).tocsc()
    q.sort_indices()
    big = BatchSolver(q, max_batch=3, ordering=_lib.ORDER_ND)
    ld1, st1 = big.factorize(q.data)
    assert st1[0] == 0
    small = GpuSolver()
    small.factorize(ar1_q(40, 0.5, 1.0))
    assert small.info()["max_m"] < 40
    vals = np.stack([q.data, 2.0 * q.data])
    ld2, st2 = big.factorize(vals)  # batch size 2: first capture of this sequence
    assert np.all(st2 == 0)
    rhs = np.stack([np.sin(np.arange(q.shape[0]) * 0.1), np.cos(np.arange(q.shape[0]) * 0.2)])
    xs = big.solve(rhs)
    f = O.Factor(q, perm=O.default_perm(q))
    ref = f.logdet()
    assert abs(ld2[0] - ref) <= LOGDET_RTOL * abs(ref)
    assert abs(ld2[1] - (ref + q.shape[0] * math.log(2.0))) <= LOGDET_RTOL * abs(ref)
    assert backward_error(q, xs[0], rhs[0]) < 1e-14
    assert backward_error(2.0 * q, xs[1], rhs[1]) < 1e-14
    assert rel(xs[0], f.solve(rhs[0])) < SIGMA_RTOL
