"""2-D triangle meshes for SPDE models over the C ABI: topology, P1 finite-element blocks and
the barycentric observation projector (crates/inla_fmesher/src/fmesher.rs), on the host and,
with results equal bit for bit, on the device (``fem_device``, ``projector_device``,
``SpdePlan``; torch tensors on the current CUDA device)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from ._lib import as_f64, as_i64, check, dptr, lib, lptr

FEM_BLOCKS = ("c0", "c1", "g1", "b1")


class Mesh:
    """``build_mesh2d`` (fmesher.rs:119-158): ``vertices`` [nv][2], ``triangles`` [ntri][3]."""

    def __init__(self, vertices, triangles):
        self.vertices = as_f64(np.asarray(vertices, dtype=float).reshape(-1, 2))
        self.triangles = as_i64(np.asarray(triangles).reshape(-1, 3))
        self.nv, self.ntri = len(self.vertices), len(self.triangles)
        h = C.c_void_p()
        check(lib().inla_mesh_create(self.nv, dptr(self.vertices), self.ntri, lptr(self.triangles), C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().inla_mesh_free(h)
            self._h = None

    @property
    def neighbors(self):
        nb = np.zeros((self.ntri, 3), dtype=np.int64)
        check(lib().inla_mesh_neighbors(self._h, lptr(nb)))
        return nb

    def fem(self, triangle_scale=None, diffusion=None):
        """``assemble_fem_blocks_diffusion`` (fmesher.rs:515-626): dict of CSC blocks
        ``c0``, ``c1``, ``g1``, ``b1`` and the triangle ``areas``."""
        sc = None if triangle_scale is None else as_f64(np.broadcast_to(triangle_scale, (self.ntri,)))
        df = None if diffusion is None else as_f64(diffusion)
        areas = np.zeros(self.ntri)
        check(lib().inla_mesh_fem(self._h, None if sc is None else dptr(sc), None if df is None else dptr(df),
                                  dptr(areas)))
        out = {"areas": areas}
        for which, name in enumerate(FEM_BLOCKS):
            nnz = C.c_int64()
            check(lib().inla_mesh_fem_block(self._h, which, C.byref(nnz), None, None, None))
            cp = np.zeros(self.nv + 1, dtype=np.int64)
            ri = np.zeros(nnz.value, dtype=np.int64)
            v = np.zeros(nnz.value)
            check(lib().inla_mesh_fem_block(self._h, which, None, lptr(cp), lptr(ri), dptr(v)))
            out[name] = sp.csc_matrix((v, ri, cp), shape=(self.nv, self.nv))
        return out

    def fem_pattern(self, which):
        """CSC pattern ``(colptr, rowidx)`` of FEM block ``which`` (a name of ``FEM_BLOCKS`` or its
        index), from the topology alone; equal to ``fem()[name]``'s."""
        w = FEM_BLOCKS.index(which) if isinstance(which, str) else int(which)
        nnz = C.c_int64()
        check(lib().inla_mesh_fem_pattern(self._h, w, C.byref(nnz), None, None))
        cp = np.zeros(self.nv + 1, dtype=np.int64)
        ri = np.zeros(nnz.value, dtype=np.int64)
        check(lib().inla_mesh_fem_pattern(self._h, w, None, lptr(cp), lptr(ri)))
        return cp, ri

    def fem_device(self, triangle_scale=None, diffusion=None):
        """The blocks of ``fem`` computed on the current CUDA device: dict of float64 tensors of
        the values on ``fem_pattern``'s patterns, plus ``areas``; ``triangle_scale`` a device
        tensor [ntri] or None (converted to float64: a float32 tensor keeps its float32 rounding,
        so pass float64 values to match ``fem`` bit for bit)."""
        import torch

        dev = torch.device("cuda", torch.cuda.current_device())
        out = {"areas": torch.empty(self.ntri, dtype=torch.float64, device=dev)}
        for name in FEM_BLOCKS:
            out[name] = torch.empty(len(self.fem_pattern(name)[1]), dtype=torch.float64, device=dev)
        sc = None
        if triangle_scale is not None:
            sc = torch.as_tensor(triangle_scale, dtype=torch.float64, device=dev).expand(self.ntri).contiguous()
        df = None if diffusion is None else as_f64(diffusion)
        stream = torch.cuda.current_stream(dev).cuda_stream
        vp = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        check(lib().inla_mesh_fem_dev(self._h, vp(sc), None if df is None else dptr(df), vp(out["areas"]),
                                      *(vp(out[n]) for n in FEM_BLOCKS), C.c_void_p(stream)))
        torch.cuda.current_stream(dev).synchronize()
        return out

    def projector_device(self, points):
        """``projector`` on the current CUDA device: ``points`` a tensor [npts][2]; returns
        ``(rowptr, colidx, vals)`` device tensors of the CSR matrix."""
        import torch

        dev = torch.device("cuda", torch.cuda.current_device())
        p = torch.as_tensor(points, dtype=torch.float64, device=dev).reshape(-1, 2).contiguous()
        n = p.shape[0]
        rp = torch.empty(n + 1, dtype=torch.int64, device=dev)
        ci = torch.empty(max(3 * n, 1), dtype=torch.int64, device=dev)
        v = torch.empty(max(3 * n, 1), dtype=torch.float64, device=dev)
        nnz = C.c_int64()
        stream = torch.cuda.current_stream(dev).cuda_stream
        check(lib().inla_mesh_projector_dev(self._h, n, C.c_void_p(p.data_ptr()), C.c_void_p(rp.data_ptr()),
                                            C.c_void_p(ci.data_ptr()), C.c_void_p(v.data_ptr()), C.byref(nnz),
                                            C.c_void_p(stream)))
        return rp, ci[:nnz.value], v[:nnz.value]

    def locate(self, points):
        """Triangle of each point (-1 outside) and its barycentric weights (fmesher.rs:161-263)."""
        p = as_f64(np.asarray(points, dtype=float).reshape(-1, 2))
        t = np.zeros(len(p), dtype=np.int64)
        b = np.zeros((len(p), 3))
        check(lib().inla_mesh_locate(self._h, len(p), dptr(p), lptr(t), dptr(b)))
        return t, b

    def projector(self, points):
        """``observation_projector_triplets`` (fmesher.rs:168-219) as a CSR matrix."""
        p = as_f64(np.asarray(points, dtype=float).reshape(-1, 2))
        n = len(p)
        rp = np.zeros(n + 1, dtype=np.int64)
        ci = np.zeros(3 * n, dtype=np.int64)
        v = np.zeros(3 * n)
        check(lib().inla_mesh_projector(self._h, n, dptr(p), lptr(rp), lptr(ci), dptr(v)))
        nnz = int(rp[-1])
        return sp.csr_matrix((v[:nnz], ci[:nnz], rp), shape=(n, self.nv))


class Mesh1D:
    """``build_mesh1d`` (mesh1d.rs:15-34): knots strictly increasing."""

    def __init__(self, loc):
        self.loc = as_f64(np.ravel(loc))
        self.n = len(self.loc)

    def fem(self):
        """``assemble_fem_blocks`` (mesh1d.rs:42-79): CSC blocks ``c0``, ``c1``, ``g1``, ``b1``."""
        out = {}
        for which, name in enumerate(FEM_BLOCKS):
            nnz = C.c_int64()
            check(lib().inla_mesh1d_fem(self.n, dptr(self.loc), which, C.byref(nnz), None, None, None))
            cp = np.zeros(self.n + 1, dtype=np.int64)
            ri = np.zeros(nnz.value, dtype=np.int64)
            v = np.zeros(nnz.value)
            check(lib().inla_mesh1d_fem(self.n, dptr(self.loc), which, None, lptr(cp), lptr(ri), dptr(v)))
            out[name] = sp.csc_matrix((v, ri, cp), shape=(self.n, self.n))
        return out

    def projector(self, s):
        """``observation_projector_triplets`` (mesh1d.rs:85-110) as a CSR matrix."""
        s = as_f64(np.ravel(s))
        rp = np.zeros(len(s) + 1, dtype=np.int64)
        ci = np.zeros(2 * len(s), dtype=np.int64)
        v = np.zeros(2 * len(s))
        check(lib().inla_mesh1d_projector(self.n, dptr(self.loc), len(s), dptr(s), lptr(rp), lptr(ci), dptr(v)))
        nnz = int(rp[-1])
        return sp.csr_matrix((v[:nnz], ci[:nnz], rp), shape=(len(s), self.n))


def spde_components(c0, g):
    """``spde_precision_csc`` (spde.rs:70-140) as components on one pattern through
    ``inla_spde_components``: ``(pattern, comp_values [3][nnz])`` for C0, G1 and
    G1 C0^-1 G1, the coefficients being tau^2 (kappa^4, 2 kappa^2, 1)."""
    c0 = as_f64(c0)
    g = sp.csc_matrix(g)
    n = len(c0)
    cp, ri, v = as_i64(g.indptr), as_i64(g.indices), as_f64(g.data)
    nnz = C.c_int64()
    check(lib().inla_spde_components(n, dptr(c0), lptr(cp), lptr(ri), dptr(v), C.byref(nnz), None, None, None))
    pcp = np.zeros(n + 1, dtype=np.int64)
    pri = np.zeros(nnz.value, dtype=np.int64)
    comp = np.zeros((3, nnz.value))
    check(lib().inla_spde_components(n, dptr(c0), lptr(cp), lptr(ri), dptr(v), None, lptr(pcp), lptr(pri),
                                     dptr(comp)))
    pattern = sp.csc_matrix((np.ones(nnz.value), pri, pcp), shape=(n, n))
    return pattern, comp


class SpdePlan:
    """The SPDE components of ``spde_components`` on the device for a fixed G1 pattern
    (``colptr``, ``rowidx``, rows strictly ascending in each column)."""

    def __init__(self, n, colptr, rowidx):
        self.n = int(n)
        self._cp, self._ri = as_i64(colptr), as_i64(rowidx)
        h = C.c_void_p()
        check(lib().inla_spde_plan_create(self.n, lptr(self._cp), lptr(self._ri), C.byref(h)))
        self._h = h
        nnz = C.c_int64()
        check(lib().inla_spde_plan_pattern(h, C.byref(nnz), None, None))
        self.colptr = np.zeros(self.n + 1, dtype=np.int64)
        self.rowidx = np.zeros(nnz.value, dtype=np.int64)
        check(lib().inla_spde_plan_pattern(h, None, lptr(self.colptr), lptr(self.rowidx)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().inla_spde_plan_free(h)
            self._h = None

    @property
    def pattern(self):
        return sp.csc_matrix((np.ones(len(self.rowidx)), self.rowidx, self.colptr), shape=(self.n, self.n))

    def components(self, c0, g_vals):
        """Device tensors ``c0`` [n] and ``g_vals`` (on the G1 pattern) -> ``comp`` [3][nnz]
        on the device; raises ``InlaError`` for a near-zero ``c0`` entry as the host form does."""
        import torch

        from ._lib import INLA_ERR_INVALID, InlaError

        dev = c0.device
        comp = torch.empty((3, len(self.rowidx)), dtype=torch.float64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        check(lib().inla_spde_components_dev(self._h, C.c_void_p(c0.data_ptr()), C.c_void_p(g_vals.data_ptr()),
                                             C.c_void_p(comp.data_ptr()), C.c_void_p(status.data_ptr()),
                                             C.c_void_p(stream)))
        if int(status.item()) != 0:
            raise InlaError(INLA_ERR_INVALID, "Zero entry in mass matrix c0 diagonal")
        return comp

