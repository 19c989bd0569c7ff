"""Config 5 at full size: SPDE on the 600 x 600 jittered mesh (360 000 latent nodes) with
100 000 negative-binomial counts (size 5); theta = [log tau, log kappa] (the reference's
negative-binomial model keeps the size fixed), CCD with 9 nodes. The batch is admitted by the
measured front size against the device's free memory. No oracle runs at this size (its
simplicial factorization would take hours); the negative-binomial Laplace is compared with the
oracle at small size in test_gpu_laplace.py. Checked here: a batch evaluation equals the
single ones, the fit is finite and recovers the generating hyperparameters."""
import numpy as np
import pytest

from inla_b200 import _lib, models
from inla_b200.laplace import PRIOR_PC_SPDE, LaplaceModel
from inla_b200.solver import GpuSolver

pytestmark = pytest.mark.gpu


def test_config5_spde600_nbinomial_fit():
    import torch

    p = models.make_spde_problem(nx=600, n_obs=100_000, seed=models.SEED_BASE + 5, family="nbinomial")
    s = GpuSolver(_lib.ORDER_ND)
    s.analyze(p.model.pattern)
    info = s.info()
    # two slots of fronts and two of selected inverses per batch member (prior + posterior);
    # blocks cached by the library for reuse count as free device memory here
    from inla_b200._lib import check, lib

    check(lib().inla_release_cached_memory())
    per_point = 4 * 8 * info["front_total"]
    free = torch.cuda.mem_get_info()[0]
    admit = int(0.7 * free // per_point)
    print(f"config5: nnz(L) {info['nnz_l']}, max front {info['max_m']}, {per_point / 1e9:.1f} GB per theta-point, "
          f"{admit} admitted")
    assert admit >= 5  # the mode-search batch (1 + 2m points)
    lm = LaplaceModel(p.model, a=p.a, family="nbinomial", y=p.y, p1=5.0, p2=1.0, max_batch=min(admit, 9))

    thetas = [(-3.0, 2.5), (-3.4, 2.7)]
    coefs = np.stack([models.spde_coefs(a, b)[0] for a, b in thetas])
    both = lm.eval(coefs, variances=True)
    one = lm.eval(coefs[1:], variances=True)
    assert np.all(both["status"] == 0) and one["status"][0] == 0
    assert abs(both["mlik"][1] - one["mlik"][0]) <= 1e-12 * abs(one["logdet_post"][0])
    assert np.max(np.abs(both["var"][1] - one["var"][0])) <= 1e-10 * np.max(np.abs(one["var"][0]))
    assert np.all(both["var"] > 0)

    def tmap(t):
        c, dc = models.spde_coefs(t[0], t[1])
        return c, dc, 1.0, np.zeros(2)

    res = lm.fit(np.zeros(2), theta_map=tmap, priors=[(PRIOR_PC_SPDE, 0, (1.0, 0.05, 1.0, 0.01))],
                 mode_search="newton", batched=True)
    print(f"config5 fit: {res['seconds']:.2f} s, {res['n_evals']} theta-evaluations in {res['n_batches']} batches, "
          f"mode {res['mode']}")
    assert np.isfinite(res["mlik"]) and np.all(np.isfinite(res["mean"])) and np.all(np.isfinite(res["var"]))
    truth = np.array([p.truth["log_tau"], p.truth["log_kappa"]])
    assert np.max(np.abs(res["mode"] - truth)) < 0.5, (res["mode"], truth)
