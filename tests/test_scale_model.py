"""Host-side behaviour of inla_scale_model that needs no GPU: the reference's singleton rule
and the argument checks made before any device work."""
import numpy as np
import pytest
import scipy.sparse as sp

from inla_b200 import InlaError
from inla_b200.solver import scale_model


def test_singleton_becomes_one():
    """design.rs:160-163: a 1 x 1 Q is replaced by [1]."""
    qs, fac, d = scale_model(sp.csc_matrix([[4.0]]))
    assert qs.toarray().tolist() == [[1.0]] and fac == 0.25 and d[0] == 0.25


def test_basis_outside_the_null_space_is_rejected():
    r = sp.csc_matrix(np.array([[1.0, -1.0, 0.0], [-1.0, 2.0, -1.0], [0.0, -1.0, 1.0]]))
    with pytest.raises(InlaError, match="null space"):
        scale_model(r, null_basis=[[1.0, 0.0, 0.0]])


def test_rows_with_the_same_single_support_are_rejected():
    r = sp.csc_matrix(np.array([[1.0, -1.0], [-1.0, 1.0]]))
    u = np.full((1, 2), 1 / np.sqrt(2))
    with pytest.raises(InlaError):
        scale_model(r, null_basis=np.vstack([u, u, u]))
    with pytest.raises(InlaError):
        scale_model(sp.csc_matrix((3, 3)))   # no nonzero


def test_dense_generator_identity_scale_is_one():
    """design.rs:234-243 on the generator's dense restatement (models.scale_model)."""
    from inla_b200 import models

    qs, fac = models.scale_model(sp.identity(4, format="csc"))
    assert abs(fac - 1.0) < 1e-8 and np.all(np.abs(qs.diagonal() - 1.0) < 1e-8)
