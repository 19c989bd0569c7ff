"""ctypes binding of ``lib/libinla_b200.so`` (the C ABI in ``include/inla_b200.h``).

There is no CPU fallback: importing the package raises when the shared library
is missing, and every call raises :class:`InlaError` on a non-zero status.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .build import LIB

INLA_OK = 0
INLA_ERR_SINGULAR = 1
INLA_ERR_NOT_PD = 2
INLA_ERR_DIM_MISMATCH = 3
INLA_ERR_OOM = 4
INLA_ERR_NONCONVERGED = 5
INLA_ERR_CANCELLED = 6
INLA_ERR_INVALID = 7
INLA_ERR_NOT_FACTORED = 8
INLA_ERR_CUDA = 9
INLA_ERR_INTERNAL = 10

ORDER_REFERENCE = 0
ORDER_AMD = 1
ORDER_RCM = 2
ORDER_NATURAL = 3
ORDER_CUSTOM = 4
ORDER_TIME_MAJOR = 5
ORDER_ND = 6
LAP_NO_PRIOR_SHARING = 8

_ERROR_NAMES = {
    INLA_ERR_SINGULAR: "Singular",
    INLA_ERR_NOT_PD: "NotPositiveDefinite",
    INLA_ERR_DIM_MISMATCH: "DimensionMismatch",
    INLA_ERR_OOM: "OutOfMemory",
    INLA_ERR_NONCONVERGED: "NonConverged",
    INLA_ERR_CANCELLED: "Cancelled",
    INLA_ERR_INVALID: "Invalid",
    INLA_ERR_NOT_FACTORED: "NotFactored",
    INLA_ERR_CUDA: "CudaError",
    INLA_ERR_INTERNAL: "Internal",
}


class InlaError(RuntimeError):
    """Non-zero status from the C ABI (``code`` is the INLA_ERR_* value)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None

P = C.c_void_p
I64 = C.c_int64
DP = C.POINTER(C.c_double)
LP = C.POINTER(C.c_int64)
IP = C.POINTER(C.c_int)

# (name, restype, argtypes) of every exported symbol in include/inla_b200.h
SIGNATURES = [
    ("inla_last_error", C.c_char_p, []),
    ("inla_kernel_launches", I64, []),
    ("inla_release_cached_memory", C.c_int, []),
    ("inla_choose_symmetric_order", C.c_int, [I64, LP, LP, LP]),
    ("inla_solver_new", C.c_int, [C.c_int, C.POINTER(P)]),
    ("inla_solver_free", None, [P]),
    ("inla_solver_set_perm", C.c_int, [P, I64, LP]),
    ("inla_solver_analyze", C.c_int, [P, I64, LP, LP]),
    ("inla_solver_factorize", C.c_int, [P, I64, LP, LP, DP]),
    ("inla_solver_solve", C.c_int, [P, DP, DP]),
    ("inla_solver_diag_inv", C.c_int, [P, DP]),
    ("inla_solver_log_abs_det", C.c_int, [P, DP]),
    ("inla_solver_selinv_pattern", C.c_int, [P, DP]),
    ("inla_solver_info", C.c_int, [P, LP]),
    ("inla_solver_perm", C.c_int, [P, LP]),
    ("inla_solver_etree", C.c_int, [P, LP]),
    ("inla_solver_supernodes", C.c_int, [P, LP, LP]),
    ("inla_solver_colcounts", C.c_int, [P, LP]),
    ("inla_batch_create", C.c_int, [I64, LP, LP, C.c_int, C.c_int, C.POINTER(P)]),
    ("inla_batch_free", None, [P]),
    ("inla_batch_factorize", C.c_int, [P, C.c_int, DP, DP, IP]),
    ("inla_batch_solve", C.c_int, [P, C.c_int, DP, DP]),
    ("inla_batch_diag_inv", C.c_int, [P, C.c_int, DP]),
    ("inla_batch_selinv_pattern", C.c_int, [P, C.c_int, DP]),
    ("inla_batch_factorize_dev", C.c_int, [P, C.c_int, P, P, P, P]),
    ("inla_batch_schedule", C.c_int, [P, IP]),
    ("inla_solver_check_schedule", C.c_int, [P, LP]),
    ("inla_set_persistent_schedule", C.c_int, [C.c_int]),
    ("inla_set_panel_form", C.c_int, [C.c_int]),
    ("inla_batch_wait_limit_selftest", C.c_int, [P, C.c_double, IP]),
    ("inla_batch_solve_dev", C.c_int, [P, C.c_int, P, P]),
    ("inla_batch_diag_inv_dev", C.c_int, [P, C.c_int, P, P]),
    ("inla_batch_selinv_pattern_dev", C.c_int, [P, C.c_int, P, P]),
    ("inla_laplace_create", C.c_int, [I64, LP, LP, C.c_int, DP, I64, LP, LP, DP, C.c_int, DP, DP, DP, C.c_int,
                                      C.c_int, C.POINTER(P)]),
    ("inla_laplace_free", None, [P]),
    ("inla_laplace_set_constraints", C.c_int, [P, C.c_int, DP, DP, C.c_int]),
    ("inla_multi_create", C.c_int, [C.c_int, LP, LP, LP, LP, C.c_int, DP, LP, LP, DP, C.c_int, DP, DP, DP,
                                    C.c_int, C.c_int, C.POINTER(P)]),
    ("inla_multi_free", None, [P]),
    ("inla_multi_eval", C.c_int, [P, C.c_int, DP, DP, C.c_int, DP, DP, DP, DP]),
    ("inla_multi_fit", C.c_int, [P, C.c_int, DP, P, P, P, P, DP, DP, DP, DP, DP, IP, IP, DP]),
    ("inla_multi_fit_predictor", C.c_int, [P, DP, DP]),
    ("inla_multi_fit_model_selection", C.c_int, [P, C.c_int, C.c_int, DP, DP, DP]),
    ("inla_multi_theta_map_ar1_iid", C.c_int, [C.c_int, DP, C.c_int, DP, DP, DP, DP, P]),
    ("inla_multi_log_prior_set", C.c_double, [C.c_int, DP, C.c_int, DP, P]),
    ("inla_laplace_eval", C.c_int, [P, C.c_int, DP, DP, C.c_int, DP, DP, DP, DP]),
    ("inla_prior_log_density", C.c_double, [P, C.c_int, DP, C.c_int, DP]),
    ("inla_log_prior_set", C.c_double, [DP, C.c_int, DP, P]),
    ("inla_fit", C.c_int, [P, C.c_int, DP, P, P, P, P, DP, DP, DP, DP, DP, DP, DP]),
    ("inla_fit_predictor", C.c_int, [P, DP, DP]),
    ("inla_fit_phase_seconds", C.c_int, [P, DP]),
    ("inla_scale_model", C.c_int, [I64, LP, LP, DP, C.c_int, DP, C.c_int, DP, DP, DP]),
    ("inla_mesh_create", C.c_int, [I64, DP, I64, LP, C.POINTER(P)]),
    ("inla_mesh_free", None, [P]),
    ("inla_mesh_neighbors", C.c_int, [P, LP]),
    ("inla_mesh_fem", C.c_int, [P, DP, DP, DP]),
    ("inla_mesh_fem_block", C.c_int, [P, C.c_int, LP, LP, LP, DP]),
    ("inla_mesh_locate", C.c_int, [P, I64, DP, LP, DP]),
    ("inla_mesh_projector", C.c_int, [P, I64, DP, LP, LP, DP]),
    ("inla_spde_components", C.c_int, [I64, DP, LP, LP, DP, LP, LP, LP, DP]),
    ("inla_mesh_fem_pattern", C.c_int, [P, C.c_int, LP, LP, LP]),
    ("inla_mesh_fem_dev", C.c_int, [P, P, DP, P, P, P, P, P, P]),
    ("inla_mesh_projector_dev", C.c_int, [P, I64, P, P, P, P, LP, P]),
    ("inla_spde_plan_create", C.c_int, [I64, LP, LP, C.POINTER(P)]),
    ("inla_spde_plan_free", None, [P]),
    ("inla_spde_plan_pattern", C.c_int, [P, LP, LP, LP]),
    ("inla_spde_components_dev", C.c_int, [P, P, P, P, P, P]),
    ("inla_mesh1d_fem", C.c_int, [I64, DP, C.c_int, LP, LP, LP, DP]),
    ("inla_mesh1d_projector", C.c_int, [I64, DP, I64, DP, LP, LP, DP]),
    ("inla_predictor_moments", C.c_int, [I64, I64, LP, LP, DP, C.c_int, DP, DP, DP, DP, DP]),
    ("inla_fit_model_selection", C.c_int, [P, C.c_int, DP, DP, DP]),
    ("inla_model_selection", C.c_int, [C.c_int, I64, DP, DP, DP, C.c_int, DP, C.c_int, DP, DP, C.c_int, DP, DP,
                                       DP]),
    ("inla_predictor_moments_dev", C.c_int, [I64, I64, P, P, P, C.c_int, P, P, P, P, P, P, P, P]),
    ("inla_model_selection_dev", C.c_int, [C.c_int, I64, P, P, P, C.c_int, DP, C.c_int, P, P, C.c_int, DP, DP, DP,
                                           P]),
    ("inla_mlik_gaussian", C.c_int, [C.c_double, C.c_int, DP, DP]),
    ("inla_fit_marginal", C.c_int, [P, C.c_int, I64, C.c_int, C.c_double, DP, DP]),
    ("inla_fit_posterior_precision", C.c_int, [P, LP, LP, LP, DP]),
    ("inla_posterior_precision", C.c_int, [I64, LP, LP, C.c_int, DP, DP, I64, LP, LP, DP, C.c_int, DP, DP, DP, DP,
                                           C.c_int, DP, LP, LP, LP, DP]),
    ("inla_mixture_marginal", C.c_int, [C.c_int, DP, DP, DP, C.c_int, C.c_double, DP, DP]),
    ("inla_hyperpar_marginal", C.c_int, [C.c_int, DP, DP, C.c_int, C.c_double, DP, DP]),
    ("inla_marginal_quantiles", C.c_int, [C.c_int, DP, DP, C.c_int, DP, DP]),
    ("inla_observation_cdf", C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, DP]),
    ("inla_cpo_failure", C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]),
    ("inla_theta_map_spde", C.c_int, [DP, C.c_int, DP, DP, DP, DP, P]),
    ("inla_dense_ldlt_solve_noalloc", C.c_int, [C.c_int, P, P, P, P, P, P]),
]


def lib():
    """Load the shared library (raises when it has not been built)."""
    global _lib
    if _lib is None:
        path = Path(LIB)
        if not path.exists():
            raise ImportError(f"libinla_b200.so is not built ({path}); run inla_b200.build.build()")
        L = C.CDLL(str(path))
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int):
    if code != INLA_OK:
        raise InlaError(code, lib().inla_last_error().decode())


def dptr(a: np.ndarray):
    return a.ctypes.data_as(DP)


def lptr(a: np.ndarray):
    return a.ctypes.data_as(LP)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(IP)


def as_i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


def as_f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)
