"""Per-model DIC / WAIC / CPO / PIT and Gaussian-approximation mlik of a many-model fit against
the same model's single-model fit (whose criteria are checked against the oracle in
test_gpu_fit.py). The two fits agree to ~1e-6 in their modes, so the criteria agree to that
order; differences of large deviances (effective parameters) get absolute bounds."""
import numpy as np
import pytest

from inla_b200 import models
from inla_b200.multi import MultiModel

pytestmark = pytest.mark.gpu


def test_multi_fit_criteria_match_single_model_fits():
    from inla_b200.laplace import LaplaceModel
    from inla_b200.multi import AR1_IID_PRIORS

    p = models.make_multi_problem(G=6, n_hi=1200, seed=9)
    mm = MultiModel(p.models, p.a, p.y, family="poisson", max_batch=4)
    r = mm.fit(np.zeros((mm.G, 3)))
    assert np.all(r["status"] == 0)

    def tmap(t):
        c, dc = models.ar1_iid_coefs(t)
        return c, dc, 1.0, np.zeros(3)

    for g in (0, mm.G - 1):
        lm = LaplaceModel(p.models[g], a=p.a[g], family="poisson", y=p.y[g], max_batch=25)
        lm.fit(np.zeros(3), theta_map=tmap, priors=AR1_IID_PRIORS, mode_search="newton", batched=True)
        s = lm.model_selection()
        t = mm.model_selection(g)
        for key in ("dic", "mean_deviance", "waic", "lppd"):
            assert abs(t[key] - s[key]) <= 1e-4 * max(1.0, abs(s[key])), key
        for key in ("dic_p_eff", "waic_p_eff"):
            assert abs(t[key] - s[key]) <= 1e-2, key
        assert abs(t["mlik_gaussian"] - s["mlik_gaussian"]) <= 1e-3
        assert abs(t["cpo_failures"] - s["cpo_failures"]) <= 2
        both = ~np.isnan(t["cpo"]) & ~np.isnan(s["cpo"])
        assert both.sum() >= len(t["cpo"]) - s["cpo_failures"] - 2
        np.testing.assert_allclose(t["cpo"][both], s["cpo"][both], rtol=1e-4)
