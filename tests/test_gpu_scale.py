"""scale_model_csc (design.rs:150-195) by the bordered selected inverse on the GPU, against the
dense eigendecomposition it replaces (``models.scale_model``, the reference's method) and, at a
size the dense method cannot reach, against the oracle's LDL^T of the same bordered matrix."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from inla_b200 import models
from inla_b200.solver import scale_model

pytestmark = pytest.mark.gpu


def lattice(nr, nc):
    """Rook-adjacency Besag structure matrix of an nr x nc lattice (column-major nodes)."""
    idx = lambda i, j: j * nr + i
    rows, cols = [], []
    for j in range(nc):
        for i in range(nr):
            if i + 1 < nr:
                rows.append(idx(i, j)); cols.append(idx(i + 1, j))
            if j + 1 < nc:
                rows.append(idx(i, j)); cols.append(idx(i, j + 1))
    n = nr * nc
    a = sp.coo_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    a = (a + a.T).tocsr()
    return (sp.diags(np.asarray(a.sum(1)).ravel()) - a).tocsc()


def dense_ginv_diag(r):
    lam, v = np.linalg.eigh(r.toarray())
    tol = np.sqrt(np.finfo(float).eps) * max(abs(max(lam.max(), 0.0)), 1.0)
    keep = lam > tol
    return (v[:, keep] ** 2) @ (1.0 / lam[keep])


def test_besag_lattice_matches_dense_eigendecomposition():
    r = lattice(30, 30)
    qs, fac, d = scale_model(r)
    _, fac_ref = models.scale_model(r)
    assert abs(fac - fac_ref) < 1e-10 * fac_ref
    np.testing.assert_allclose(d, dense_ginv_diag(r), rtol=1e-10)
    np.testing.assert_allclose(qs.toarray(), fac * r.toarray(), rtol=0, atol=0)


def test_disconnected_graph_with_isolated_node_and_proper_block():
    """Two intrinsic components, an isolated node (zero row: ginv diagonal 0, left out of the
    mean) and a proper block (no null vector)."""
    blocks = [lattice(6, 5), lattice(4, 4), sp.csc_matrix((1, 1)), (lattice(3, 3) + sp.identity(9)).tocsc()]
    r = sp.block_diag(blocks, format="csc")
    qs, fac, d = scale_model(r)
    _, fac_ref = models.scale_model(r)
    assert abs(fac - fac_ref) < 1e-10 * fac_ref
    np.testing.assert_allclose(d, dense_ginv_diag(r), rtol=1e-10, atol=1e-14)
    assert d[30 + 16] == 0.0


def test_rw2_with_given_null_basis():
    n = 60
    dd = sp.diags([1.0, -2.0, 1.0], [0, 1, 2], shape=(n - 2, n)).tocsc()
    r = (dd.T @ dd).tocsc()
    t = np.arange(n) - (n - 1) / 2.0
    u = np.vstack([np.ones(n) / np.sqrt(n), t / np.linalg.norm(t)])
    _, fac, d = scale_model(r, null_basis=u)
    _, fac_ref = models.scale_model(r)
    assert abs(fac - fac_ref) < 1e-8 * fac_ref
    np.testing.assert_allclose(d, dense_ginv_diag(r), rtol=1e-8)


def test_proper_precision_needs_no_border():
    n = 200
    rho = 0.8
    main = np.r_[1.0, np.full(n - 2, 1 + rho * rho), 1.0]
    q = sp.diags([main, np.full(n - 1, -rho), np.full(n - 1, -rho)], [0, 1, -1], format="csc")
    _, fac, d = scale_model(q)
    ref = np.diag(np.linalg.inv(q.toarray()))
    np.testing.assert_allclose(d, ref, rtol=1e-12)
    assert abs(fac - np.exp(np.mean(np.log(ref)))) < 1e-12 * fac


def test_large_lattice_against_oracle_bordered_factor():
    """100 x 100 lattice (10 000 nodes, a dense eigendecomposition of minutes): the oracle's
    LDL^T of the same bordered matrix gives diag(Q^+)."""
    r = lattice(100, 100)
    n = r.shape[0]
    _, fac, d = scale_model(r)
    u = np.full((1, n), 1.0 / np.sqrt(n))
    m = sp.bmat([[r, sp.csc_matrix(u.T)], [sp.csc_matrix(u), sp.csc_matrix(np.zeros((1, 1)))]], format="lil")
    m[n, n] = 0.0
    m = m.tocsc()
    perm = list(O.default_perm(r))
    last = perm[-1]
    full = np.array([p for p in perm if p != last] + [n, last])
    ref = O.Factor(m, perm=full).diag_inv()[:n]
    np.testing.assert_allclose(d, ref, rtol=1e-10)
    assert abs(fac - np.exp(np.mean(np.log(ref)))) < 1e-10 * fac


def test_identity_scale_is_one():
    """design.rs:234-243: Q = I gives ginv = I and a factor of 1."""
    qs, fac, d = scale_model(sp.identity(4, format="csc"))
    assert abs(fac - 1.0) < 1e-8 and np.all(np.abs(qs.diagonal() - 1.0) < 1e-8)
