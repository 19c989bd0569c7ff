"""Host mirror of rust-inla's ``InlaSolver`` seam over the C ABI.

``GpuSolver`` follows ``trait InlaSolver`` (crates/inla_math/src/solver.rs:29-44)
method by method: ``factorize(q)`` (symbolic analysis on a new pattern,
numeric-only refactorization on an identical one, scratch.rs:90-103),
``solve(rhs)``, ``diag_inv()`` (Takahashi selected inverse) and
``log_abs_det()``. Errors surface as :class:`InlaError` with the status code
of the matching ``SolverError`` variant.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import InlaError, as_f64, as_i64, check, dptr, iptr, lib, lptr


def _csc_arrays(q):
    q = sp.csc_matrix(q)
    if q.shape[0] != q.shape[1]:
        raise InlaError(_lib.INLA_ERR_DIM_MISMATCH, f"matrix must be square, got {q.shape}")
    return q.shape[0], as_i64(q.indptr), as_i64(q.indices), as_f64(q.data)


def choose_symmetric_order(q):
    """Restated ``choose_symmetric_order`` (ordering.rs:149-162) -> (branch, fwd or None)."""
    n, cp, ri, _ = _csc_arrays(q)
    fwd = np.zeros(n, dtype=np.int64)
    kind = lib().inla_choose_symmetric_order(n, lptr(cp), lptr(ri), lptr(fwd))
    if kind < 0:
        check(-kind)
    return kind, (fwd if kind in (_lib.ORDER_RCM, _lib.ORDER_TIME_MAJOR) else None)


def scale_model(q, null_basis=None, ordering=None):
    """``scale_model_csc`` (design.rs:150-195) by a sparse selected inverse on the GPU instead of
    a dense eigendecomposition: ``(fac * Q, fac, diag(Q^+))``. ``null_basis`` (k x n) spans the
    null space of ``Q``; None derives one constant row per intrinsic connected component."""
    q = sp.csc_matrix(q)
    n, cp, ri, v = _csc_arrays(q)
    if null_basis is None:
        k, ub = -1, None
    else:
        ub = as_f64(np.atleast_2d(null_basis))
        if ub.shape[1] != n:
            raise InlaError(_lib.INLA_ERR_DIM_MISMATCH, "null_basis must have n columns")
        k = ub.shape[0]
    fac = C.c_double()
    scaled = np.zeros(len(v))
    d = np.zeros(n)
    check(lib().inla_scale_model(n, lptr(cp), lptr(ri), dptr(v), k, None if ub is None or k == 0 else dptr(ub),
                                 _lib.ORDER_ND if ordering is None else int(ordering), C.byref(fac), dptr(scaled),
                                 dptr(d)))
    return sp.csc_matrix((scaled, q.indices.copy(), q.indptr.copy()), shape=q.shape), fac.value, d


class GpuSolver:
    """One factor per solver (FaerCpuSolver equivalent, solver.rs:48-99)."""

    def __init__(self, ordering: int = _lib.ORDER_AMD):
        h = C.c_void_p()
        check(lib().inla_solver_new(int(ordering), C.byref(h)))
        self._h = h
        self.n = None
        self.nnz = None

    def close(self):
        if getattr(self, "_h", None):
            lib().inla_solver_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_perm(self, perm) -> None:
        p = as_i64(perm)
        check(lib().inla_solver_set_perm(self._h, len(p), lptr(p)))

    def analyze(self, q) -> None:
        """Host-only symbolic analysis (no GPU needed)."""
        n, cp, ri, _ = _csc_arrays(q)
        check(lib().inla_solver_analyze(self._h, n, lptr(cp), lptr(ri)))
        self.n = n
        self.nnz = len(ri)

    def colcounts(self) -> np.ndarray:
        c = np.empty(self.n, dtype=np.int64)
        check(lib().inla_solver_colcounts(self._h, lptr(c)))
        return c

    def factorize(self, q) -> None:
        n, cp, ri, v = _csc_arrays(q)
        check(lib().inla_solver_factorize(self._h, n, lptr(cp), lptr(ri), dptr(v)))
        self.n = n
        self.nnz = len(v)

    def solve(self, rhs) -> np.ndarray:
        if self.n is None:
            raise InlaError(_lib.INLA_ERR_NOT_FACTORED, "Factorization not computed yet")
        b = as_f64(rhs)
        if b.shape != (self.n,):
            raise InlaError(_lib.INLA_ERR_DIM_MISMATCH, f"rhs length {b.shape} != {self.n}")
        x = np.empty(self.n)
        check(lib().inla_solver_solve(self._h, dptr(b), dptr(x)))
        return x

    def diag_inv(self) -> np.ndarray:
        if self.n is None:
            raise InlaError(_lib.INLA_ERR_NOT_FACTORED, "Factorization not computed yet")
        d = np.empty(self.n)
        check(lib().inla_solver_diag_inv(self._h, dptr(d)))
        return d

    def log_abs_det(self) -> float:
        out = C.c_double()
        check(lib().inla_solver_log_abs_det(self._h, C.byref(out)))
        return out.value

    def selinv_pattern(self) -> np.ndarray:
        s = np.empty(self.nnz)
        check(lib().inla_solver_selinv_pattern(self._h, dptr(s)))
        return s

    def info(self) -> dict:
        a = np.zeros(8, dtype=np.int64)
        check(lib().inla_solver_info(self._h, lptr(a)))
        keys = ["n", "nnz_l", "nnz_l_stored", "nsuper", "nlevels", "max_m", "ordering", "front_total"]
        return dict(zip(keys, map(int, a)))

    def perm(self) -> np.ndarray:
        p = np.empty(self.n, dtype=np.int64)
        check(lib().inla_solver_perm(self._h, lptr(p)))
        return p

    def etree(self) -> np.ndarray:
        p = np.empty(self.n, dtype=np.int64)
        check(lib().inla_solver_etree(self._h, lptr(p)))
        return p

    def supernodes(self) -> np.ndarray:
        cnt = C.c_int64()
        check(lib().inla_solver_supernodes(self._h, None, C.byref(cnt)))
        first = np.empty(cnt.value + 1, dtype=np.int64)
        check(lib().inla_solver_supernodes(self._h, lptr(first), None))
        return first


class BatchSolver:
    """B problems that share one sparsity pattern (one symbolic analysis)."""

    def __init__(self, pattern, max_batch: int, ordering: int = _lib.ORDER_ND):
        n, cp, ri, _ = _csc_arrays(pattern)
        h = C.c_void_p()
        check(lib().inla_batch_create(n, lptr(cp), lptr(ri), int(ordering), int(max_batch), C.byref(h)))
        self._h = h
        self.n = n
        self.nnz = len(ri)
        self.max_batch = max_batch
        self.B = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().inla_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def factorize(self, values):
        v = as_f64(values)
        if v.ndim == 1:
            v = v[None, :]
        B = v.shape[0]
        if v.shape[1] != self.nnz:
            raise InlaError(_lib.INLA_ERR_DIM_MISMATCH, "values must be [B][nnz]")
        ld = np.empty(B)
        st = np.empty(B, dtype=np.int32)
        code = lib().inla_batch_factorize(self._h, B, dptr(v), dptr(ld), iptr(st))
        self.B = B
        if code not in (_lib.INLA_OK, _lib.INLA_ERR_SINGULAR):
            check(code)
        return ld, st

    def solve(self, rhs):
        b = as_f64(rhs).reshape(self.B, self.n)
        x = np.empty_like(b)
        check(lib().inla_batch_solve(self._h, self.B, dptr(b), dptr(x)))
        return x

    def diag_inv(self):
        d = np.empty((self.B, self.n))
        check(lib().inla_batch_diag_inv(self._h, self.B, dptr(d)))
        return d

    def selinv_pattern(self):
        s = np.empty((self.B, self.nnz))
        check(lib().inla_batch_selinv_pattern(self._h, self.B, dptr(s)))
        return s
