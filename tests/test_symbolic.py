"""Host-side (no GPU) checks of the product library: C-ABI exports, the
ordering choice restated bit-exact, and the symbolic analysis (etree, column
counts, supernodes) against the CPU oracle."""
import re
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from fixtures import (ar1_q, grid_laplacian, mixture_major_fgn_like, mixture_major_path_cliques, random_spd,
                      tridiagonal8)
from inla_b200 import GpuSolver, _lib, choose_symmetric_order, models

ROOT = Path(__file__).resolve().parent.parent


def header_symbols():
    text = (ROOT / "include" / "inla_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const char\*|int64_t|int|void|double)\s+(inla_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    declared = header_symbols()
    assert len(declared) >= 20
    bound = {name for name, _, _ in _lib.SIGNATURES}
    for name in declared:
        assert hasattr(L, name), f"{name} declared in include/inla_b200.h but not exported"
        assert name in bound, f"{name} has no ctypes signature"


def test_no_gpu_calls_fail_loudly():
    """Without a device the compute entry points return INLA_ERR_CUDA; nothing falls back to the CPU."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("device present")
    s = GpuSolver()
    q = tridiagonal8()
    with pytest.raises(_lib.InlaError) as e:
        s.factorize(q)
    assert e.value.code in (_lib.INLA_ERR_CUDA, _lib.INLA_ERR_OOM)


def spde_small():
    return models.make_spde_problem(nx=24, n_obs=300).model.pattern


MATRICES = {
    "tridiagonal8": tridiagonal8,
    "ar1_200": lambda: ar1_q(200, 0.5, 1.0),
    "grid_30x20": lambda: grid_laplacian(30, 20),
    "grid_60x60": lambda: grid_laplacian(60, 60),
    "fgn_like": lambda: mixture_major_fgn_like(64, 5),
    "path_cliques": lambda: mixture_major_path_cliques(64, 5),
    "random_300": lambda: random_spd(300, 0.01, 7),
    "spde_24": spde_small,
}


@pytest.mark.parametrize("name", list(MATRICES))
def test_choose_symmetric_order_bit_exact(name):
    """ordering.rs:149-162 restated in the product == the oracle's restatement."""
    q = MATRICES[name]()
    k_prod, fwd_prod = choose_symmetric_order(q)
    k_orc, fwd_orc = O.choose_order(q)
    assert k_prod == k_orc
    if fwd_orc is not None:
        np.testing.assert_array_equal(fwd_prod, fwd_orc)


@pytest.mark.parametrize("name", list(MATRICES))
@pytest.mark.parametrize("ordering", [_lib.ORDER_AMD, _lib.ORDER_REFERENCE, _lib.ORDER_NATURAL, _lib.ORDER_ND])
def test_symbolic_structure(name, ordering):
    q = MATRICES[name]()
    n = q.shape[0]
    s = GpuSolver(ordering)
    s.analyze(q)
    perm = s.perm()
    assert sorted(perm.tolist()) == list(range(n))
    parent = s.etree()
    # etree is postordered: parent > child
    assert np.all((parent == -1) | (parent > np.arange(n)))
    # column counts equal the oracle's factor under the same permutation
    cc = s.colcounts()
    f = O.Factor(q, perm=perm)
    assert int(cc.sum()) == f.nnz()
    info = s.info()
    assert info["nnz_l"] == f.nnz()
    assert info["nnz_l_stored"] >= info["nnz_l"]
    first = s.supernodes()
    assert first[0] == 0 and first[-1] == n and np.all(np.diff(first) > 0)


def test_amd_reduces_fill_on_meshes():
    """AMD fill on a 2-D mesh stays within 1.2x of the banded (RCM) ordering or better."""
    q = models.make_spde_problem(nx=40, n_obs=500).model.pattern
    a = GpuSolver(_lib.ORDER_AMD)
    a.analyze(q)
    r = GpuSolver(_lib.ORDER_RCM)
    r.analyze(q)
    assert a.info()["nnz_l"] <= 1.2 * r.info()["nnz_l"]
    # AMD gives a shallow tree (level parallelism) where RCM gives a chain
    assert a.info()["nlevels"] * 3 < r.info()["nlevels"]


def _longest_pivot_path(s):
    """Pivot columns on the longest root-to-leaf path of the supernodal tree."""
    first, et = s.supernodes(), s.etree()
    ns = len(first) - 1
    col2sn = np.repeat(np.arange(ns), np.diff(first))
    k = np.diff(first)
    path = k.astype(np.int64).copy()
    for t in range(ns):  # postordered: children before parents
        pc = et[first[t + 1] - 1]
        if pc >= 0:
            p = col2sn[pc]
            path[p] = max(path[p], path[t] + k[p])
    return int(path.max())


def test_nested_dissection_shortens_the_elimination_tree():
    """On a 2-D mesh, nested dissection gives fewer levels and a shorter pivot
    chain than AMD at comparable fill (the GPU engine's default ordering)."""
    p = models.make_spde_problem(nx=60, n_obs=1800)
    q = (p.model.pattern + p.a.T @ p.a).tocsc()
    a = GpuSolver(_lib.ORDER_AMD)
    a.analyze(q)
    d = GpuSolver(_lib.ORDER_ND)
    d.analyze(q)
    assert sorted(d.perm().tolist()) == list(range(q.shape[0]))
    assert d.info()["nlevels"] < a.info()["nlevels"]
    assert _longest_pivot_path(d) < _longest_pivot_path(a)
    assert d.info()["nnz_l"] <= 1.25 * a.info()["nnz_l"]


def test_custom_permutation_is_used():
    q = grid_laplacian(10, 10)
    p = np.random.default_rng(1).permutation(100)
    s = GpuSolver()
    s.set_perm(p)
    s.analyze(q)
    f = O.Factor(q, perm=s.perm())
    assert s.info()["nnz_l"] == f.nnz()
    # the postordering keeps the fill of the given permutation
    assert s.info()["nnz_l"] == O.Factor(q, perm=p).nnz()


def test_invalid_inputs_are_rejected():
    s = GpuSolver()
    bad = sp.csc_matrix(np.ones((3, 4)))
    with pytest.raises(_lib.InlaError) as e:
        s.analyze(bad)
    assert e.value.code == _lib.INLA_ERR_DIM_MISMATCH
    with pytest.raises(_lib.InlaError) as e:
        s.solve(np.ones(3))
    assert e.value.code == _lib.INLA_ERR_NOT_FACTORED
    s2 = GpuSolver()
    with pytest.raises(_lib.InlaError):
        s2.set_perm(np.array([0, 0, 1]))
        s2.analyze(tridiagonal8()[:3, :3])
