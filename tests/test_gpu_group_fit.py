"""The space x time group model at full size (Besag 50 x 50 (x) AR1 T = 40 + iid + intercept,
n = 200 001, binomial(10), one sum-to-zero row per time held bordered): the adjoint gradient
of log pi(theta | y) against central finite differences (step 1e-4) of the same engine's
mlik at 1e-5 relative, and a full INLA fit with CCD over the 4 hyperparameters (25 nodes;
structured.rs:884-963, inference.rs:1246-1468). The downscaled model is compared with the
oracle's own finite differences at the same tolerance."""
import numpy as np
import pytest

import oracle as O
from inla_b200 import models
from inla_b200.laplace import PRIOR_PC_COR1, PRIOR_PC_PREC, LaplaceModel

pytestmark = pytest.mark.gpu

GROUP_PRIORS = [(PRIOR_PC_PREC, 0, (1.0, 0.01)), (PRIOR_PC_PREC, 1, (1.0, 0.01)), (PRIOR_PC_COR1, 2, (0.5, 0.75)),
                (PRIOR_PC_PREC, 3, (1.0, 0.01))]


def adjoint(lm, t):
    c, dc = models.group_coefs(t)
    out = lm.eval(c[None], gradient=True)
    T = len(c)
    return dc @ (0.5 * out["trP"][0, :T] - 0.5 * out["trQ"][0, :T] - 0.5 * out["xMx"][0, :T]
                 + 0.5 * out["zMx"][0, :T])


def test_group_adjoint_vs_oracle_fd_small():
    p = models.make_group_problem(nr=6, nc=6, T=4)
    lm = LaplaceModel(p.model, a=p.a, family="binomial", y=p.y, p1=p.ntrials, max_batch=2)
    lm.set_constraints(*p.constraint, method="bordered")
    t = np.array([0.2, -0.1, 1.8, 1.2])
    g = adjoint(lm, t)

    def mlik(tt):
        q = p.model.matrix(models.group_coefs(tt)[0])
        return O.laplace(q, p.a, "binomial", p.y, p1=p.ntrials, constraints=p.constraint, tol=1e-10)["mlik"]

    h = 1e-4
    fd = np.array([(mlik(t + h * e) - mlik(t - h * e)) / (2 * h) for e in np.eye(4)])
    err = np.max(np.abs(g - fd)) / np.max(np.abs(fd))
    print(f"group 6x6x4 adjoint vs oracle FD: {err:.3e}")
    assert err <= 1e-5, (g, fd)


def test_group_full_size_adjoint_vs_fd_and_ccd25_fit():
    p = models.make_group_problem()
    lm = LaplaceModel(p.model, a=p.a, family="binomial", y=p.y, p1=p.ntrials, max_batch=9)
    lm.set_constraints(*p.constraint)  # auto -> bordered at this size
    t = np.array([0.1, -0.1, 2.0, 1.3])
    g = adjoint(lm, t)
    h = 1e-4
    pts = [t] + [t + s * h * e for e in np.eye(4) for s in (1.0, -1.0)]
    out = lm.eval(np.stack([models.group_coefs(x)[0] for x in pts]))
    assert np.all(out["status"] == 0)
    fd = np.array([(out["mlik"][1 + 2 * i] - out["mlik"][2 + 2 * i]) / (2 * h) for i in range(4)])
    err = np.max(np.abs(g - fd)) / np.max(np.abs(fd))
    print(f"group full-size adjoint vs central FD: {err:.3e} (gradient {g})")
    assert err <= 1e-5, (g, fd)

    def tmap(th):
        c, dc = models.group_coefs(th)
        return c, dc, 1.0, np.zeros(4)

    r = lm.fit(np.array([0.0, 0.0, 1.5, 1.0]), theta_map=tmap, priors=GROUP_PRIORS, mode_search="newton",
               batched=True)
    print(f"group CCD fit: {r['seconds']:.2f} s, {r['n_evals']} theta-evaluations in {r['n_batches']} batches, "
          f"mode {r['mode']}, phases {r['phase_s']}")
    assert r["node_theta"].shape == (25, 4)
    assert np.isfinite(r["mlik"]) and np.all(np.isfinite(r["mean"])) and np.all(r["var"] > 0)
    c, e = p.constraint
    assert np.max(np.abs(c @ r["mean"] - e)) < 1e-8
    # rho = 0.8 (logit-type 2.197) and tau_iid = 4 (log 1.386) are identified by the data
    rho = 2.0 / (1.0 + np.exp(-r["mode"][2])) - 1.0
    assert abs(rho - 0.8) < 0.1 and abs(r["mode"][3] - np.log(4.0)) < 0.5, r["mode"]
