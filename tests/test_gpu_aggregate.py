"""Post-node aggregation on the device (inference.rs:1370-1384, 1436-1514; design.rs:52-70,
198-210; model_selection.rs:101-325) through the C ABI's device forms, against the library's
host forms and the oracle's restatement: the per-node predictor and the mixture moments are
bit-identical to the host code; DIC, WAIC, CPO and PIT agree with the host code and the
oracle to 1e-12 relative (the device sums over observations use a fixed reduction tree)."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from inla_b200 import _lib
from inla_b200.laplace import model_selection, predictor_moments

pytestmark = pytest.mark.gpu


def dev(a, dtype=None):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=dtype or torch.float64, device="cuda")


def ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def test_predictor_moments_device_equal_host():
    import torch

    rng = np.random.default_rng(1)
    K, n, nobs = 15, 3000, 2200
    a = sp.random(nobs, n, density=3.0 / n, random_state=2, format="csr")
    a.data = rng.uniform(0.1, 1.0, a.nnz)
    a.sort_indices()
    cm = rng.standard_normal((K, n))
    cm[:, ::17] = 0.0  # zero entries are skipped in the sum, as matvec_csc does
    cv = rng.uniform(0.01, 2.0, (K, n))
    w = rng.uniform(0.1, 1.0, K)
    w /= w.sum()
    pm_h, pv_h = predictor_moments(a, w, cm, cv)
    z = lambda *shape: torch.zeros(*shape, dtype=torch.float64, device="cuda")
    d_eta, d_etav, d_pm, d_pv = z(K, nobs), z(K, nobs), z(nobs), z(nobs)
    rp, ci, av = dev(a.indptr, torch.int64), dev(a.indices, torch.int32), dev(a.data)
    dw, dcm, dcv = dev(w), dev(cm), dev(cv)
    torch.cuda.synchronize()
    _lib.check(_lib.lib().inla_predictor_moments_dev(nobs, n, ptr(rp), ptr(ci), ptr(av), K, ptr(dw), ptr(dcm),
                                                      ptr(dcv), ptr(d_eta), ptr(d_etav), ptr(d_pm), ptr(d_pv), None))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(d_pm.cpu().numpy(), pm_h)
    np.testing.assert_array_equal(d_pv.cpu().numpy(), pv_h)
    ref = O.predictor_moments(a, list(w), list(cm), list(cv))
    np.testing.assert_allclose(d_pm.cpu().numpy(), ref[0], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(d_pv.cpu().numpy(), ref[1], rtol=1e-12)
    np.testing.assert_allclose(d_eta.cpu().numpy()[3], O.matvec_csc(a, cm[3]), rtol=1e-14, atol=1e-15)


def family_data(family, nobs, K, rng):
    eta0 = rng.normal(0.3, 0.4, nobs)
    if family == "gaussian":
        y, p1, p2 = eta0 + rng.normal(0, 0.3, nobs), np.full(nobs, 8.0), None
    elif family == "poisson":
        y, p1, p2 = rng.poisson(np.exp(eta0)).astype(float), np.full(nobs, 1.5), None
    elif family == "binomial":
        p1 = np.full(nobs, 10.0)
        y, p2 = rng.binomial(10, 1 / (1 + np.exp(-eta0))).astype(float), None
    else:
        y, p1, p2 = rng.negative_binomial(5, 5 / (5 + np.exp(eta0))).astype(float), np.full(nobs, 5.0), np.ones(nobs)
    ce = eta0[None, :] + rng.normal(0, 0.05, (K, nobs))
    cv = rng.uniform(0.002, 0.05, (K, nobs))
    w = rng.uniform(0.2, 1.0, K)
    return y, p1, p2, ce, cv, w / w.sum()


@pytest.mark.parametrize("family", ["gaussian", "poisson", "binomial", "nbinomial"])
def test_model_selection_device_matches_host_and_oracle(family):
    import torch

    rng = np.random.default_rng(7)
    K, nobs, k0 = 9, 3000, 4
    y, p1, p2, ce, cv, w = family_data(family, nobs, K, rng)
    host = model_selection(family, y, w, k0, ce, cv, p1=p1, p2=p2)
    crit, cpo, pit = np.zeros(8), np.zeros(nobs), np.zeros(nobs)
    dy, dp1, dp2, dce, dcv = dev(y), dev(p1), None if p2 is None else dev(p2), dev(ce), dev(cv)
    torch.cuda.synchronize()
    fam = {"gaussian": 0, "poisson": 1, "binomial": 2, "nbinomial": 3}[family]
    _lib.check(_lib.lib().inla_model_selection_dev(fam, nobs, ptr(dy), ptr(dp1), ptr(dp2), K, _lib.dptr(w), k0,
                                                    ptr(dce), ptr(dcv), 7, _lib.dptr(crit), _lib.dptr(cpo),
                                                    _lib.dptr(pit), None))
    close = lambda a, b, scale=None: abs(a - b) <= 1e-12 * max(1.0, abs(b) if scale is None else scale)
    # the effective-parameter counts are differences of sums of order |mean deviance| and |lppd|;
    # the device and host sums of those agree to 1e-12 of their own size
    scales = {"dic_p_eff": abs(host["mean_deviance"]), "waic_p_eff": abs(host["lppd"])}
    for j, key in enumerate(["dic", "mean_deviance", "dic_p_eff", "waic", "lppd", "waic_p_eff"]):
        assert close(crit[j], host[key], scales.get(key)), (key, crit[j], host[key])
    assert int(crit[7]) == host["cpo_failures"]
    np.testing.assert_array_equal(np.isnan(cpo), np.isnan(host["cpo"]))
    np.testing.assert_array_equal(np.isnan(pit), np.isnan(host["pit"]))
    ok = ~np.isnan(cpo)
    np.testing.assert_allclose(cpo[ok], host["cpo"][ok], rtol=1e-12)
    okp = ~np.isnan(pit)
    np.testing.assert_allclose(pit[okp], host["pit"][okp], rtol=1e-12, atol=1e-15)
    q1 = p1 if p1 is not None else np.ones(nobs)
    q2 = p2 if p2 is not None else np.ones(nobs)
    dic = O.compute_dic(family, y, q1, q2, list(ce), list(w), k0)
    waic = O.compute_waic(family, y, q1, q2, list(ce), list(w))
    assert close(crit[0], dic["dic"]) and close(crit[3], waic["waic"]) and close(crit[4], waic["lppd"])
    ocpo, opit, nf = O.compute_cpo_pit(family, y, q1, q2, list(ce), list(cv), list(w))
    assert int(crit[7]) == nf
    got = [(c, o) for c, o in zip(cpo, ocpo) if o is not None]
    assert len(got) == int(ok.sum())
    np.testing.assert_allclose([c for c, _ in got], [o for _, o in got], rtol=1e-12)


def test_model_selection_device_reports_the_reference_error():
    """A likelihood that cannot be evaluated (a negative Poisson count) is the reference's DIC error."""
    import torch

    rng = np.random.default_rng(3)
    y, p1, p2, ce, cv, w = family_data("poisson", 100, 3, rng)
    y[37] = -1.0
    crit, cpo, pit = np.zeros(8), np.zeros(100), np.zeros(100)
    dy, dp1, dce, dcv = dev(y), dev(p1), dev(ce), dev(cv)
    torch.cuda.synchronize()
    rc = _lib.lib().inla_model_selection_dev(1, 100, ptr(dy), ptr(dp1), None, 3, _lib.dptr(w), 0, ptr(dce), ptr(dcv), 7,
                                             _lib.dptr(crit), _lib.dptr(cpo), _lib.dptr(pit), None)
    assert rc == _lib.INLA_ERR_INVALID
    assert b"DIC: likelihood evaluation failed at observation 37" in _lib.lib().inla_last_error()
