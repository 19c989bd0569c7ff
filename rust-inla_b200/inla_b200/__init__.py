"""B200-native INLA inner hot path (CUDA sm_100a, FP64) behind rust-inla's solver seam.

The compute path is ``lib/libinla_b200.so`` (C ABI in ``include/inla_b200.h``);
this package is its host-side mirror: the ``InlaSolver`` seam
(:mod:`inla_b200.solver`), the Laplace / INLA drivers and the seeded input
generators (:mod:`inla_b200.models`).
"""
from ._lib import InlaError, lib  # noqa: F401  (raises ImportError when the library is missing)
from .solver import BatchSolver, GpuSolver, choose_symmetric_order  # noqa: F401

lib()
