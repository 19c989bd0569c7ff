"""Device forms of the mesh tools through the C ABI: FEM blocks, SPDE components and the
observation projector on the GPU against the library's host forms, bit for bit (the host forms
equal the oracle's restatement of fmesher.rs / spde.rs bit for bit in tests/test_mesh.py).
Sizes: the 200 x 200 mesh of the SPDE benchmark and the 600 x 600 mesh (360 000 nodes,
100 000 points) of the largest configuration."""
import numpy as np
import pytest

from inla_b200 import InlaError, models
from inla_b200.mesh import FEM_BLOCKS, Mesh, SpdePlan, spde_components

pytestmark = pytest.mark.gpu

SQUARE_V = [[0.0, 0.0], [1.0, 0.0], [0.0, 1.0], [1.0, 1.0]]
SQUARE_T = [[0, 1, 2], [1, 3, 2]]


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.int64)


def same_bits(dev, host):
    return np.array_equal(bits(dev.cpu().numpy()), bits(host))


def jittered(nx, seed):
    return models.grid_mesh(nx, np.random.default_rng(seed))


def check_fem(m, ts=None, diff=None):
    import torch

    host = m.fem(triangle_scale=ts, diffusion=diff)
    d_ts = None if ts is None else torch.tensor(np.asarray(ts, dtype=np.float64), device="cuda")  # float64, not
    dev = m.fem_device(triangle_scale=d_ts, diffusion=diff)                                         # torch's float32
    assert same_bits(dev["areas"], host["areas"])
    for name in FEM_BLOCKS:
        assert same_bits(dev[name], host[name].data), name
    return host, dev


@pytest.mark.parametrize("case", ["square", "default", "barrier_aniso"])
def test_fem_device_equals_host_bitwise(case):
    if case == "square":
        check_fem(Mesh(SQUARE_V, SQUARE_T))
        check_fem(Mesh(SQUARE_V, SQUARE_T), ts=[0.1 ** 2, 1.0], diff=[2.0, 0.0, 0.5])
        return
    v, t = jittered(200, 11)
    m = Mesh(v, t)
    if case == "default":
        check_fem(m)
    else:
        ts = np.ones(len(t))
        ts[::7] = 0.25 ** 2
        check_fem(m, ts=ts, diff=[1.5, -0.2, 0.8])
        check_fem(m)  # a second call on the same mesh reuses its device data


def test_fem_device_rejects_a_non_spd_tensor():
    with pytest.raises(InlaError, match="SPD"):
        Mesh(SQUARE_V, SQUARE_T).fem_device(diffusion=[1.0, 2.0, 1.0])


def test_spde_components_device_chain_equals_host():
    """mesh -> FEM -> components entirely on the device, against the host chain."""
    import torch

    v, t = jittered(200, 11)
    m = Mesh(v, t)
    host, dev = check_fem(m)
    c0 = host["c0"].diagonal()
    pat, comp = spde_components(c0, host["g1"])
    cp, ri = m.fem_pattern("g1")
    plan = SpdePlan(len(v), cp, ri)
    assert np.array_equal(plan.colptr, pat.indptr) and np.array_equal(plan.rowidx, pat.indices)
    assert dev["c0"].numel() == len(v)  # every vertex in a triangle: the c0 block is the dense diagonal
    got = plan.components(dev["c0"], dev["g1"])
    assert same_bits(got, comp)
    got2 = plan.components(dev["c0"], dev["g1"])  # the plan's scratch is reused
    assert torch.equal(got, got2)
    bad = dev["c0"].clone()
    bad[17] = 0.0
    with pytest.raises(InlaError, match="Zero entry"):
        plan.components(bad, dev["g1"])


def check_projector(m, pts):
    import torch

    a = m.projector(pts)
    rp, ci, v = m.projector_device(torch.tensor(pts, device="cuda"))
    assert np.array_equal(rp.cpu().numpy(), a.indptr)
    assert np.array_equal(ci.cpu().numpy(), a.indices)
    assert same_bits(v, a.data)


def test_projector_device_equals_host_with_edge_and_vertex_points():
    v, t = jittered(200, 11)
    m = Mesh(v, t)
    rng = np.random.default_rng(12)
    pts = rng.uniform(0.0, 1.0, size=(20_000, 2))
    tt = t[rng.integers(0, len(t), 500)]
    extra = np.concatenate([v[rng.integers(0, len(v), 500)],            # on vertices
                            0.5 * (v[tt[:, 0]] + v[tt[:, 1]]),          # on edges
                            [[0.0, 0.0], [1.0, 1.0], [0.5, 0.0], [0.0, 0.37]]])
    pts = np.concatenate([pts, extra])
    rng.shuffle(pts)
    check_projector(m, pts)
    check_projector(m, pts[:1])
    check_projector(Mesh(SQUARE_V, SQUARE_T), np.array([[0.1, 0.1], [0.5, 0.5], [0.0, 0.0], [0.9, 0.2]]))


def test_projector_device_reports_the_host_error_and_empty_input():
    import torch

    v, t = jittered(60, 3)
    m = Mesh(v, t)
    pts = np.random.default_rng(4).uniform(0.0, 1.0, size=(300, 2))
    pts = np.concatenate([pts[:100], [[1.5, 0.5]], pts[100:], [[-2.0, 0.0]]])
    with pytest.raises(InlaError) as host_err:
        m.projector(pts)
    with pytest.raises(InlaError) as dev_err:
        m.projector_device(torch.tensor(pts, device="cuda"))
    assert str(dev_err.value) == str(host_err.value) and "outside the mesh" in str(dev_err.value)
    rp, ci, vals = m.projector_device(torch.zeros((0, 2), dtype=torch.float64, device="cuda"))
    assert rp.cpu().tolist() == [0] and ci.numel() == 0 and vals.numel() == 0


def test_mesh_tools_device_at_the_largest_configuration():
    """600 x 600 mesh (717 602 triangles), 100 000 points: FEM, SPDE components and projector."""
    v, t = jittered(600, 13)
    m = Mesh(v, t)
    host, dev = check_fem(m)
    pat, comp = spde_components(host["c0"].diagonal(), host["g1"])
    cp, ri = m.fem_pattern("g1")
    assert same_bits(SpdePlan(len(v), cp, ri).components(dev["c0"], dev["g1"]), comp)
    pts = np.random.default_rng(14).uniform(0.0, 1.0, size=(100_000, 2))
    check_projector(m, pts)
