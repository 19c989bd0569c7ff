"""Mesh tools of the library (host code, no GPU): the reference's own fmesher tests
(crates/inla_fmesher/src/fmesher.rs:945-1163), bitwise parity with the oracle's restatement of
the FEM assembly and the projector walk, and agreement with the numpy input generators."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from inla_b200 import InlaError, models
from inla_b200.mesh import FEM_BLOCKS, Mesh

SQUARE_V = [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]]
SQUARE_T = [[0, 1, 2], [1, 3, 2]]


def test_builds_topology_for_two_triangles():
    """fmesher.rs:945-960."""
    nb = Mesh(SQUARE_V, SQUARE_T).neighbors
    assert nb[0][0] == 1 and nb[1][1] == 0


def test_locates_point_in_triangle_edge_and_vertex():
    """fmesher.rs:1065-1095."""
    m = Mesh(SQUARE_V, SQUARE_T)
    t, b = m.locate([[0.1, 0.1], [0.5, 0.5], [0.0, 0.0], [2.0, 2.0]])
    assert t[0] >= 0 and np.all(np.abs(b[0]) > 1e-15)              # strictly inside
    assert t[1] >= 0 and np.sum(np.abs(b[1]) <= 1e-15) >= 1         # on the shared edge
    assert t[2] == 0 and np.argmax(b[2]) == 0 and abs(b[2][0] - 1.0) < 1e-15   # vertex 0
    assert t[3] == -1                                                # outside


def test_assembles_fem_blocks_for_square_mesh():
    """fmesher.rs:1122-1163: areas, lumped mass, identity vs anisotropic vs barrier stiffness."""
    m = Mesh(SQUARE_V, SQUARE_T)
    f = m.fem()
    assert f["areas"].tolist() == [0.5, 0.5]
    assert f["c0"].diagonal().tolist() == [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]
    assert f["g1"].nnz > 0 and f["b1"].nnz > 0
    ident = m.fem(diffusion=[1.0, 0.0, 1.0])
    assert (f["g1"] != ident["g1"]).nnz == 0
    aniso = m.fem(diffusion=[2.0, 0.0, 0.5])
    assert f["g1"][0, 0] != aniso["g1"][0, 0]
    barrier = m.fem(triangle_scale=[0.1 ** 2, 1.0])
    assert (f["g1"] != barrier["g1"]).nnz > 0
    assert (f["c0"] != barrier["c0"]).nnz == 0


def test_invalid_meshes_raise_the_reference_errors():
    with pytest.raises(InlaError, match="three vertices"):
        Mesh([[0, 0], [1, 0]], [])
    with pytest.raises(InlaError, match="out of range"):
        Mesh(SQUARE_V, [[0, 1, 7]])
    with pytest.raises(InlaError, match="duplicate"):
        Mesh(SQUARE_V, [[0, 1, 1]])
    with pytest.raises(InlaError, match="near-zero area"):
        Mesh([[0, 0], [1, 0], [2, 0]], [[0, 1, 2]])
    with pytest.raises(InlaError, match="non-manifold"):
        Mesh(SQUARE_V, [[0, 1, 2], [0, 1, 3]])
    with pytest.raises(InlaError, match="SPD"):
        Mesh(SQUARE_V, SQUARE_T).fem(diffusion=[1.0, 2.0, 1.0])
    with pytest.raises(InlaError, match="outside the mesh"):
        Mesh(SQUARE_V, SQUARE_T).projector([[0.2, 0.2], [1.5, 0.5]])


def _jittered(nx, seed):
    rng = np.random.default_rng(seed)
    return models.grid_mesh(nx, rng)


@pytest.mark.parametrize("scale,diff", [(None, None), ("barrier", (2.0, 0.3, 0.7))])
def test_fem_blocks_match_oracle_bitwise(scale, diff):
    v, t = _jittered(12, 5)
    ts = None
    if scale == "barrier":
        ts = np.ones(len(t))
        ts[::7] = 0.25 ** 2
    f = Mesh(v, t).fem(triangle_scale=ts, diffusion=diff)
    ref = O.fem_blocks(v, t, ts, diff if diff is not None else (1.0, 0.0, 1.0))
    assert f["areas"].tolist() == ref["areas"]
    for name in FEM_BLOCKS:
        got = f[name].tocoo()
        d = {(int(r), int(c)): x for r, c, x in zip(got.row, got.col, got.data)}
        assert d == ref[name], name


def test_fem_matches_input_generator():
    """The generator's numpy assembly (scipy sums duplicates in its own order)."""
    v, t = _jittered(40, 7)
    f = Mesh(v, t).fem()
    c0, g = models.fem_matrices(v, t)
    np.testing.assert_allclose(f["c0"].diagonal(), c0, rtol=1e-15)
    assert abs(f["g1"] - g).max() <= 1e-14 * abs(g).max()


def test_projector_matches_oracle_walk_and_generator():
    nx = 25
    v, t = _jittered(nx, 9)
    rng = np.random.default_rng(10)
    pts = rng.uniform(0.0, 1.0, size=(400, 2))
    a = Mesh(v, t).projector(pts)
    ref = sp.coo_matrix(([w for _, _, w in O.projector_triplets(v, t, pts)],
                         ([r for r, _, _ in O.projector_triplets(v, t, pts)],
                          [c for _, c, _ in O.projector_triplets(v, t, pts)])), shape=a.shape).tocsr()
    ref.sort_indices()
    assert (a != ref).nnz == 0
    g = models.grid_projector(v, t, nx, pts)
    assert (a != g).nnz == 0
    np.testing.assert_allclose(np.asarray(a.sum(1)).ravel(), 1.0, atol=1e-14)


def test_projector_at_full_mesh_size():
    """The 200 x 200 mesh (79 202 triangles) with 20 000 points: rows sum to one and the
    interpolant of a linear function is exact."""
    v, t = _jittered(200, 11)
    rng = np.random.default_rng(12)
    pts = rng.uniform(0.0, 1.0, size=(20_000, 2))
    a = Mesh(v, t).projector(pts)
    np.testing.assert_allclose(np.asarray(a.sum(1)).ravel(), 1.0, atol=1e-13)
    lin = 0.3 + 1.7 * v[:, 0] - 0.9 * v[:, 1]
    np.testing.assert_allclose(a @ lin, 0.3 + 1.7 * pts[:, 0] - 0.9 * pts[:, 1], atol=1e-12)


# --- SPDE precision components (crates/inla_stats/src/spde.rs) -----------------------------------

from inla_b200.mesh import spde_components  # noqa: E402


def test_projector_interpolates_at_vertices():
    """spde.rs:149-161: a point at vertex 0 of a single triangle."""
    a = Mesh([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]], [[0, 1, 2]]).projector([[0.0, 0.0]])
    assert a.shape == (1, 3)
    assert abs(a[0, 0] - 1.0) < 1e-12 and abs(a[0, 1]) < 1e-12


def _q_from_components(pattern, comp, kappa, tau):
    c = tau * tau * np.array([kappa ** 4, 2 * kappa ** 2, 1.0])
    return sp.csc_matrix((c @ comp, pattern.indices, pattern.indptr), shape=pattern.shape)


def test_spde_precision_square_mesh():
    """spde.rs:163-189: kappa = 1, tau = 2 on the 2-triangle square: positive diagonal; the
    components give the oracle's restatement of spde_precision_csc."""
    v = [[0.0, 1.0], [1.0, 1.0], [0.0, 0.0], [1.0, 0.0]]
    f = Mesh(v, [[0, 2, 1], [1, 2, 3]]).fem()
    pattern, comp = spde_components(f["c0"].diagonal(), f["g1"])
    q = _q_from_components(pattern, comp, 1.0, 2.0)
    assert q.shape == (4, 4) and q.nnz > 0 and np.all(q.diagonal() > 0)
    ref, _ = O.spde_precision(f["c0"].diagonal(), f["g1"], 1.0, 2.0)
    dense = np.zeros((4, 4))
    for (i, j), x in ref.items():
        dense[i, j] = x
    np.testing.assert_allclose(q.toarray(), dense, rtol=1e-14, atol=1e-14)


def test_spde_components_match_oracle_and_generator():
    v, t = _jittered(15, 13)
    f = Mesh(v, t).fem()
    c0, g = f["c0"].diagonal(), f["g1"]
    pattern, comp = spde_components(c0, g)
    _, gcg = O.spde_precision(c0, g, 1.0, 1.0)
    got = sp.csc_matrix((comp[2], pattern.indices, pattern.indptr), shape=pattern.shape).tocoo()
    d = {(int(r), int(c)): x for r, c, x in zip(got.row, got.col, got.data)}
    assert {k: x for k, x in d.items() if k in gcg} == gcg          # bit for bit, same sum order
    assert all(x == 0.0 for k, x in d.items() if k not in gcg)     # diagonal-only fill
    lm = models.build_latent(len(c0), models.spde_components(c0, g), "spde")
    assert (lm.pattern != pattern).nnz == 0
    np.testing.assert_allclose(comp, lm.comp_values, rtol=1e-13, atol=1e-13 * np.abs(comp).max())


def test_spde_components_reject_zero_mass():
    g = sp.identity(3, format="csc")
    with pytest.raises(InlaError, match="Zero entry in mass matrix"):
        spde_components([1.0, 0.0, 1.0], g)


# --- 1-D meshes (crates/inla_fmesher/src/mesh1d.rs:143-190) ---------------------------------------

from inla_b200.mesh import Mesh1D  # noqa: E402


def test_mesh1d_unit_interval_two_knots():
    f = Mesh1D([0.0, 1.0]).fem()
    assert f["c0"][0, 0] == 0.5 and f["c0"][1, 1] == 0.5
    assert abs(f["g1"][0, 0] - 1.0) < 1e-14 and abs(f["g1"][0, 1] + 1.0) < 1e-14
    assert f["b1"].nnz == 0


def test_mesh1d_projector_at_knots_and_midpoint():
    a = Mesh1D([0.0, 2.0, 5.0]).projector([0.0, 2.0, 3.5, 5.0, -1.0, 9.0]).toarray()
    assert abs(a[0, 0] - 1) < 1e-12 and abs(a[1, 1] - 1) < 1e-12
    assert abs(a[2, 1] - 0.5) < 1e-12 and abs(a[2, 2] - 0.5) < 1e-12
    assert abs(a[3, 2] - 1) < 1e-12 and abs(a[4, 0] - 1) < 1e-12 and abs(a[5, 2] - 1) < 1e-12


def test_mesh1d_rejects_unsorted():
    with pytest.raises(InlaError):
        Mesh1D([1.0, 0.0]).fem()
    with pytest.raises(InlaError):
        Mesh1D([0.0, 0.0]).projector([0.5])


def test_mesh1d_spde_precision_positive_diagonal():
    """spde.rs:205-213: the 1-D blocks feed the same SPDE components."""
    f = Mesh1D([0.0, 1.0, 2.0, 3.0]).fem()
    pattern, comp = spde_components(f["c0"].diagonal(), f["g1"])
    q = _q_from_components(pattern, comp, 1.0, 2.0)
    assert q.shape == (4, 4) and np.all(q.diagonal() > 0)
    rng = np.random.default_rng(14)
    knots = np.cumsum(rng.uniform(0.1, 1.0, 40))
    f = Mesh1D(knots).fem()
    h = np.diff(knots)
    np.testing.assert_array_equal(f["c0"].diagonal(), np.r_[h / 2, 0.0] + np.r_[0.0, h / 2])


def test_barrier_spde_reduces_covariance_across_strip():
    """structured.rs barrier_spde_reduces_covariance_across_strip: on a 7 x 2 vertex lattice,
    triangles whose centroid has 0.35 <= x < 0.65 become barrier triangles (range fraction 0.1,
    stiffness scale 0.01); the covariance between the two ends of the strip drops below half."""
    nxv, nyv = 7, 2
    v = np.array([[i / (nxv - 1), j / (nxv - 1)] for j in range(nyv) for i in range(nxv)])
    t = []
    for j in range(nyv - 1):
        for i in range(nxv - 1):
            a, b, c, d = j * nxv + i, j * nxv + i + 1, (j + 1) * nxv + i, (j + 1) * nxv + i + 1
            t += [[a, b, d], [a, d, c]]
    t = np.array(t)
    cx = v[t].mean(axis=1)[:, 0]
    barrier = (cx >= 0.35) & (cx < 0.65)
    assert barrier.any()
    m = Mesh(v, t)
    covs = []
    for scale in (None, np.where(barrier, 0.1 ** 2, 1.0)):
        f = m.fem(triangle_scale=scale)
        pattern, comp = spde_components(f["c0"].diagonal(), f["g1"])
        q = _q_from_components(pattern, comp, 1.0, 1.0).toarray()
        covs.append(abs(np.linalg.inv(q)[0, nxv - 1]))
    assert covs[1] < 0.5 * covs[0], covs


# --- device forms: what needs no GPU (patterns, plan validation, loud failure without a device) ---

from inla_b200.mesh import SpdePlan  # noqa: E402


@pytest.mark.parametrize("nx,seed", [(2, 1), (3, 0), (12, 5), (40, 7)])
def test_device_fem_patterns_equal_the_host_blocks(nx, seed):
    """The device forms' patterns come from the topology alone and equal the host assembly's
    (nx = 3: the square plus a vertex no triangle uses, whose columns stay empty)."""
    if nx == 2:
        m = Mesh(SQUARE_V, SQUARE_T)
    elif nx == 3:
        m = Mesh(SQUARE_V + [[2.0, 2.0]], SQUARE_T)
    else:
        v, t = _jittered(nx, seed)
        m = Mesh(v, t)
    f = m.fem(triangle_scale=None)
    for name in FEM_BLOCKS:
        cp, ri = m.fem_pattern(name)
        assert np.array_equal(cp, f[name].indptr) and np.array_equal(ri, f[name].indices), name


def test_spde_plan_pattern_equals_the_host_components():
    v, t = _jittered(20, 3)
    f = Mesh(v, t).fem()
    pat, _ = spde_components(f["c0"].diagonal(), f["g1"])
    plan = SpdePlan(len(v), f["g1"].indptr, f["g1"].indices)
    assert np.array_equal(plan.colptr, pat.indptr) and np.array_equal(plan.rowidx, pat.indices)


def test_spde_plan_rejects_unsorted_or_out_of_range_rows():
    with pytest.raises(InlaError, match="strictly ascending"):
        SpdePlan(2, [0, 2, 3], [1, 0, 1])
    with pytest.raises(InlaError, match="out of range"):
        SpdePlan(2, [0, 1, 2], [0, 5])
    with pytest.raises(InlaError, match="non-empty"):
        SpdePlan(0, [0], [])


def test_device_mesh_calls_fail_loudly_without_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("device present")
    from inla_b200 import _lib

    m = Mesh(SQUARE_V, SQUARE_T)
    rc = _lib.lib().inla_mesh_fem_dev(m._h, None, None, None, None, None, None, None, None)
    assert rc == _lib.INLA_ERR_CUDA
