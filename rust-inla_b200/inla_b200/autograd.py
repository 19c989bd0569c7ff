"""``torch.autograd.Function`` face of the adjoint gradient of log pi(theta | y).

``log_posterior(theta, model)`` returns ``mlik(theta) + log pi(theta)`` for one
theta-point (shape ``[m]``) or a batch (shape ``[B, m]``, evaluated in one
batched launch sequence); its backward pass uses the hand-written adjoint
(trace contractions of the Takahashi selected inverses of Q and Q_post plus
the Laplace-mode terms) instead of finite differences. The reference has no
gradient at all (it uses Nelder-Mead on values and an FD Hessian).
"""
from __future__ import annotations

import numpy as np
import torch

from .laplace import SPDE_DEFAULT_PRIORS, LaplaceModel, log_prior, prior_set


def spde_theta_map(theta):
    """theta = [log prec_eps, log tau, log kappa] -> (coef, dcoef[m][3], p1scale, dp1scale[m])."""
    t2 = np.exp(2.0 * theta[1])
    k2 = np.exp(2.0 * theta[2])
    c = np.array([t2 * k2 * k2, 2.0 * t2 * k2, t2])
    dc = np.zeros((3, 3))
    dc[1] = 2.0 * c
    dc[2] = [4.0 * c[0], 2.0 * c[1], 0.0]
    s = float(np.exp(theta[0]))
    return c, dc, s, np.array([s, 0.0, 0.0])


def _values_and_grads(model: LaplaceModel, thetas: np.ndarray, theta_map, priors):
    ps = prior_set(priors)
    maps = [theta_map(t) for t in thetas]
    coefs = np.stack([m[0] for m in maps])
    scale = np.array([m[2] for m in maps])
    out = model.eval(coefs, scale, gradient=True, mode=False)
    T = model.ncomp
    vals = np.empty(len(thetas))
    grads = np.empty_like(thetas)
    for b, (t, (c, dc, s, ds)) in enumerate(zip(thetas, maps)):
        lp, gp = log_prior(ps, t)
        if out["status"][b] != 0:
            vals[b] = -1e12
            grads[b] = 0.0
            continue
        g = dc @ (0.5 * out["trP"][b, :T] - 0.5 * out["trQ"][b, :T] - 0.5 * out["xMx"][b, :T]
                  + 0.5 * out["zMx"][b, :T])
        g = g + ds / s * (out["dll"][b] - 0.5 * out["trQ"][b, T])
        vals[b] = out["mlik"][b] + lp
        grads[b] = g + gp
    return vals, grads


class LogPosterior(torch.autograd.Function):
    """theta -> log pi(theta | y) (up to a constant), with the adjoint gradient in backward."""

    @staticmethod
    def forward(ctx, theta, model, theta_map, priors):
        th = theta.detach().to("cpu", torch.float64).numpy()
        single = th.ndim == 1
        th2 = th[None, :] if single else th
        vals, grads = _values_and_grads(model, th2, theta_map, priors)
        g = torch.as_tensor(grads, dtype=theta.dtype, device=theta.device)
        ctx.save_for_backward(g[0] if single else g)
        v = torch.as_tensor(vals, dtype=theta.dtype, device=theta.device)
        return v[0] if single else v

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        if g.ndim == 1:
            return grad_out * g, None, None, None
        return grad_out[:, None] * g, None, None, None


def log_posterior(theta: torch.Tensor, model: LaplaceModel, theta_map=spde_theta_map,
                  priors=SPDE_DEFAULT_PRIORS) -> torch.Tensor:
    return LogPosterior.apply(theta, model, theta_map, priors)
