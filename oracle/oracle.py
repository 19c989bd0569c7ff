"""CPU ORACLE — test infrastructure only.

Python face of ``liboracle.so`` (plain-C restatement of rust-inla's INLA inner
path, ``oracle/inla_oracle.c``) plus pure-Python restatements of the small
theta-level algorithms (Nelder-Mead, finite-difference Hessian, CCD / grid
designs, weight normalisation). Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline / ``--impl reference`` leg use this module; the
product library never calls it.

Parity status: pinned against the reference's own known-answer tests for the
path (see ``tests/test_oracle.py``) and dense numpy references; the reference
itself (Rust + faer 0.24) cannot be built here.
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_lib = None
DP = C.POINTER(C.c_double)
LP = C.POINTER(C.c_int64)


def build(force: bool = False) -> Path:
    src = [HERE / "inla_oracle.c", HERE / "inla_oracle.h"]
    if force or not LIB.exists() or any(p.stat().st_mtime > LIB.stat().st_mtime for p in src):
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        sig = {
            "orc_lower_bandwidth": (C.c_int64, [C.c_int64, LP, LP]),
            "orc_bandwidth_with_fwd": (C.c_int64, [C.c_int64, LP, LP, LP]),
            "orc_try_time_major": (C.c_int, [C.c_int64, LP, LP, LP]),
            "orc_rcm": (None, [C.c_int64, LP, LP, LP]),
            "orc_choose_order": (C.c_int, [C.c_int64, LP, LP, LP]),
            "orc_min_degree": (None, [C.c_int64, LP, LP, LP]),
            "orc_factor_create": (C.c_int, [C.c_int64, LP, LP, DP, LP, C.POINTER(C.c_void_p)]),
            "orc_factor_create_sn": (C.c_int, [C.c_int64, LP, LP, DP, LP, C.POINTER(C.c_void_p)]),
            "orc_set_supernodal": (None, [C.c_int]),
            "orc_set_threads": (None, [C.c_int]),
            "orc_factor_free": (None, [C.c_void_p]),
            "orc_factor_nnz": (C.c_int64, [C.c_void_p]),
            "orc_logdet": (C.c_double, [C.c_void_p]),
            "orc_solve": (None, [C.c_void_p, DP, DP]),
            "orc_takahashi_diag": (C.c_int, [C.c_void_p, DP]),
            "orc_takahashi_pattern": (C.c_int, [C.c_void_p, LP, LP, DP]),
            "orc_eval_lik": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, DP, DP, DP]),
            "orc_log_gamma": (C.c_double, [C.c_double]),
            "orc_project_constraints": (C.c_int, [C.c_int64, DP, C.c_int, DP, DP]),
            "orc_laplace": (C.c_int, [C.c_int64, LP, LP, DP, C.c_int64, LP, LP, DP, C.c_int, DP, DP, DP,
                                      C.c_int, DP, DP, C.c_int, C.c_double, LP, DP, DP, DP]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a, t=DP):
    return None if a is None else a.ctypes.data_as(t)


def _csc(q):
    q = sp.csc_matrix(q)
    q.sort_indices()
    return q.shape[0], _i64(q.indptr), _i64(q.indices), _f64(q.data)


# ---------------------------------------------------------------------------
# ordering.rs
# ---------------------------------------------------------------------------

def lower_bandwidth(q) -> int:
    n, cp, ri, _ = _csc(q)
    return int(lib().orc_lower_bandwidth(n, _p(cp, LP), _p(ri, LP)))


def choose_order(q):
    """(branch, fwd): 5 time-major, 2 RCM, 1 AMD (fwd None for AMD)."""
    n, cp, ri, _ = _csc(q)
    fwd = np.zeros(n, dtype=np.int64)
    k = int(lib().orc_choose_order(n, _p(cp, LP), _p(ri, LP), _p(fwd, LP)))
    return k, (fwd if k in (2, 5) else None)


def rcm(q):
    n, cp, ri, _ = _csc(q)
    fwd = np.zeros(n, dtype=np.int64)
    lib().orc_rcm(n, _p(cp, LP), _p(ri, LP), _p(fwd, LP))
    return fwd


def min_degree_perm(q):
    """perm[new] = old: a minimum-degree order standing in for faer's AMD (not bit-identical)."""
    n, cp, ri, _ = _csc(q)
    perm = np.zeros(n, dtype=np.int64)
    lib().orc_min_degree(n, _p(cp, LP), _p(ri, LP), _p(perm, LP))
    return perm


def reference_perm(q):
    """perm[new] = old following the reference's choice (ordering.rs:149-162): time-major or RCM
    where it picks them, a minimum-degree order where it picks AMD."""
    k, fwd = choose_order(q)
    if fwd is None:
        return min_degree_perm(q)
    perm = np.empty(q.shape[0], dtype=np.int64)
    perm[fwd] = np.arange(q.shape[0])
    return perm


def default_perm(q):
    """perm[new] = old from the reference choice (AMD branch -> natural order)."""
    k, fwd = choose_order(q)
    n = q.shape[0]
    if fwd is None:
        return np.arange(n, dtype=np.int64)
    perm = np.empty(n, dtype=np.int64)
    perm[fwd] = np.arange(n)
    return perm


# ---------------------------------------------------------------------------
# factor
# ---------------------------------------------------------------------------

class OracleError(RuntimeError):
    pass


class Factor:
    """Simplicial LDL^T of a full-symmetric CSC (only row >= col entries read); with
    ``supernodal`` the same factor by the supernodal form (the CPU baseline's)."""

    def __init__(self, q, perm=None, supernodal=False):
        n, cp, ri, v = _csc(q)
        self.n = n
        self._q = (cp, ri)
        h = C.c_void_p()
        pp = None if perm is None else _i64(perm)
        create = lib().orc_factor_create_sn if supernodal else lib().orc_factor_create
        rc = create(n, _p(cp, LP), _p(ri, LP), _p(v), _p(pp, LP), C.byref(h))
        self._h = h
        self.singular = rc != 0

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_factor_free(self._h)
            self._h = None

    def nnz(self) -> int:
        return int(lib().orc_factor_nnz(self._h))

    def logdet(self) -> float:
        return float(lib().orc_logdet(self._h))

    def solve(self, b) -> np.ndarray:
        b = _f64(b)
        x = np.empty(self.n)
        lib().orc_solve(self._h, _p(b), _p(x))
        return x

    def diag_inv(self) -> np.ndarray:
        d = np.empty(self.n)
        if lib().orc_takahashi_diag(self._h, _p(d)):
            raise OracleError("Takahashi failed")
        return d

    def sigma_on_pattern(self, q) -> np.ndarray:
        n, cp, ri, _ = _csc(q)
        out = np.empty(len(ri))
        if lib().orc_takahashi_pattern(self._h, _p(cp, LP), _p(ri, LP), _p(out)):
            raise OracleError("Takahashi failed")
        return out


def set_threads(t: int):
    """OpenMP threads inside one supernodal factorization (1: none). Set it above 1 only where
    evaluations run one at a time, and before threads use the oracle."""
    lib().orc_set_threads(int(t))


def set_supernodal(on: bool):
    """Factorize with the supernodal form inside ``laplace`` (the CPU baseline); off by default,
    the simplicial form being the one the parity tests pin. Set before threads use the oracle."""
    lib().orc_set_supernodal(1 if on else 0)


# ---------------------------------------------------------------------------
# likelihoods / Laplace
# ---------------------------------------------------------------------------

FAMILIES = {"gaussian": 0, "poisson": 1, "binomial": 2, "nbinomial": 3}


def eval_lik(family, eta, y, p1=1.0, p2=1.0):
    lp, g, h = C.c_double(), C.c_double(), C.c_double()
    rc = lib().orc_eval_lik(FAMILIES.get(family, family), float(eta), float(y), float(p1), float(p2),
                            C.byref(lp), C.byref(g), C.byref(h))
    if rc:
        raise OracleError("likelihood evaluation failed")
    return lp.value, g.value, h.value


def project_constraints(x, c, e):
    """constraints.rs:316-353 on a copy of ``x``."""
    x = _f64(x).copy()
    c = _f64(np.atleast_2d(c))
    e = _f64(np.broadcast_to(e, (c.shape[0],)))
    if lib().orc_project_constraints(len(x), _p(x), c.shape[0], _p(c), _p(e)):
        raise OracleError("project_constraints: singular A A^T")
    return x


def log_gamma(z: float) -> float:
    return float(lib().orc_log_gamma(float(z)))


def laplace(q, a, family, y, p1=None, p2=None, constraints=None, max_iter=200, tol=1e-5, perm=None,
            want_var=False):
    """find_latent_mode_a_with_solver (inference.rs:776-975) -> dict."""
    n, cp, ri, v = _csc(q)
    y = _f64(y)
    nobs = len(y)
    if a is not None:
        a = sp.csr_matrix(a)
        a.sort_indices()
        acp, aci, av = _i64(a.indptr), _i64(a.indices), _f64(a.data)
    else:
        acp = aci = av = None
    p1 = None if p1 is None else _f64(np.broadcast_to(p1, (nobs,)))
    p2 = None if p2 is None else _f64(np.broadcast_to(p2, (nobs,)))
    kc = 0
    ca = ce = None
    if constraints is not None:
        ca = _f64(np.atleast_2d(constraints[0]))
        ce = _f64(constraints[1])
        kc = ca.shape[0]
    x = np.zeros(n)
    out = np.zeros(4)
    var = np.zeros(n) if want_var else None
    pp = None if perm is None else _i64(perm)
    rc = lib().orc_laplace(n, _p(cp, LP), _p(ri, LP), _p(v), nobs, _p(acp, LP), _p(aci, LP), _p(av),
                           FAMILIES.get(family, family), _p(y), _p(p1), _p(p2), kc, _p(ca), _p(ce),
                           int(max_iter), float(tol), _p(pp, LP), _p(x), _p(out), _p(var))
    if rc:
        raise OracleError(f"laplace failed with code {rc}")
    return {"x": x, "mlik": out[0], "logdet_prior": out[1], "logdet_post": out[2], "iters": int(out[3]),
            "var": var}


# ---------------------------------------------------------------------------
# theta-level algorithms (pure Python restatements)
# ---------------------------------------------------------------------------

def nelder_mead(x0, step, max_iter, tol, f):
    """inla_math/src/hyper_opt.rs:15-183 (reflect 1, expand 2, contract 0.5, shrink 0.5)."""
    m = len(x0)
    verts = [list(map(float, x0))]
    fv = [f(verts[0])]
    for i in range(m):
        v = list(map(float, x0))
        v[i] += step
        verts.append(v)
        fv.append(f(v))
    for _ in range(max_iter):
        idx = sorted(range(m + 1), key=lambda k: fv[k])
        verts = [verts[k] for k in idx]
        fv = [fv[k] for k in idx]
        mean = sum(fv) / (m + 1)
        var = sum((v - mean) ** 2 for v in fv) / (m + 1)
        if math.sqrt(var) < tol:
            return verts[0]
        cen = [sum(verts[i][j] for i in range(m)) / m for j in range(m)]
        refl = [cen[j] + 1.0 * (cen[j] - verts[m][j]) for j in range(m)]
        fr = f(refl)
        if fv[0] <= fr < fv[m - 1]:
            verts[m], fv[m] = refl, fr
            continue
        if fr < fv[0]:
            exp_ = [cen[j] + 2.0 * (refl[j] - cen[j]) for j in range(m)]
            fe = f(exp_)
            if fe < fr:
                verts[m], fv[m] = exp_, fe
            else:
                verts[m], fv[m] = refl, fr
            continue
        contract = False
        if fr < fv[m]:
            con = [cen[j] + 0.5 * (refl[j] - cen[j]) for j in range(m)]
            fc = f(con)
            if fc < fr:
                verts[m], fv[m] = con, fc
                contract = True
        else:
            con = [cen[j] + 0.5 * (verts[m][j] - cen[j]) for j in range(m)]
            fc = f(con)
            if fc < fv[m]:
                verts[m], fv[m] = con, fc
                contract = True
        if contract:
            continue
        for i in range(1, m + 1):
            verts[i] = [verts[0][j] + 0.5 * (verts[i][j] - verts[0][j]) for j in range(m)]
            fv[i] = f(verts[i])
    return verts[0]


def fd_hessian(mode, f, h):
    """inla_math/src/hyper_opt.rs:197-259: Hessian of g = -f by central differences."""
    m = len(mode)
    H = np.zeros((m, m))

    def g(t):
        return -f(list(t))

    g0 = g(mode)
    for i in range(m):
        for j in range(m):
            if i == j:
                tp = list(mode); tp[i] += h
                tm = list(mode); tm[i] -= h
                H[i, i] = (g(tp) - 2.0 * g0 + g(tm)) / (h * h)
            elif i < j:
                pp = list(mode); pp[i] += h; pp[j] += h
                pm = list(mode); pm[i] += h; pm[j] -= h
                mp = list(mode); mp[i] -= h; mp[j] += h
                mm = list(mode); mm[i] -= h; mm[j] -= h
                v = (g(pp) - g(pm) - g(mp) + g(mm)) / (4.0 * h * h)
                H[i, j] = H[j, i] = v
    return H


def fd_gradient(theta, f, h=1e-4):
    """Central-difference gradient of f with the stencil fd_hessian uses."""
    m = len(theta)
    gr = np.zeros(m)
    for i in range(m):
        tp = list(theta); tp[i] += h
        tm = list(theta); tm[i] -= h
        gr[i] = (f(tp) - f(tm)) / (2.0 * h)
    return gr


def ccd_design(m, f0=1.0):
    """inla_math/src/integration.rs:1-62."""
    pts = [[0.0] * m]
    for i in range(m):
        p1 = [0.0] * m; p1[i] = f0
        p2 = [0.0] * m; p2[i] = -f0
        pts += [p1, p2]
    if 2 <= m <= 4:
        val = f0 / math.sqrt(m)
        for k in range(1 << m):
            pts.append([(1.0 if (k >> i) & 1 else -1.0) * val for i in range(m)])
    elif m == 5:
        val = f0 / math.sqrt(5.0)
        for k in range(16):
            p = [0.0] * 5
            sp_ = 1.0
            for i in range(4):
                s = 1.0 if (k >> i) & 1 else -1.0
                p[i] = s * val
                sp_ *= s
            p[4] = sp_ * val
            pts.append(p)
    elif m > 5:
        raise ValueError(f"CCD strategy for m={m} is not supported")
    ne = len(pts)
    if ne > 1:
        w = 1.0 / ((ne - 1) * (1.0 + math.exp(-0.5 * f0 * f0) * (f0 * f0 / m - 1.0)))
    else:
        w = 1.0
    ws = [w] * ne
    ws[0] = 1.0 - (ne - 1) * w
    return np.array(pts), np.array(ws)


def grid_design(m, step, threshold, evaluator):
    """inla_math/src/integration.rs:64-156: m = 1 walks +step, then -step, while the
    log-density drop from the centre stays <= threshold; m = 2 walks the axes, then keeps
    the grid points within the threshold; m > 2 falls back to CCD with f0 = 2.5. Weights 1."""
    if m == 0:
        raise ValueError("Grid requires at least 1 factor")
    if m > 2:
        return ccd_design(m, 2.5)
    g0 = evaluator([0.0] * m)
    pts = []
    if m == 1:
        pts.append([0.0])
        for sgn in (1.0, -1.0):
            k = 1
            while True:
                z = [sgn * k * step]
                if g0 - evaluator(z) > threshold:
                    break
                pts.append(z)
                k += 1
    else:
        ext = []
        for axis, sgn in ((0, 1.0), (0, -1.0), (1, 1.0), (1, -1.0)):
            k = 0
            while True:
                z = [0.0, 0.0]
                z[axis] = sgn * (k + 1) * step
                if g0 - evaluator(z) > threshold:
                    break
                k += 1
            ext.append(k)
        max_i, min_i, max_j, min_j = ext
        for i in range(-min_i, max_i + 1):
            for j in range(-min_j, max_j + 1):
                z = [i * step, j * step]
                if g0 - evaluator(z) <= threshold:
                    pts.append(z)
    return np.array(pts), np.ones(len(pts))


def matvec_csc(a, x):
    """design.rs:52-70: y = A x column by column, columns with x_j == 0 skipped."""
    a = sp.csc_matrix(a)
    y = [0.0] * a.shape[0]
    for j in range(a.shape[1]):
        xv = float(x[j])
        if xv == 0.0:
            continue
        for p in range(a.indptr[j], a.indptr[j + 1]):
            y[a.indices[p]] += float(a.data[p]) * xv
    return np.array(y)


def predictor_variances_diag(a, var_x):
    """design.rs:198-210: sum_j A_ij^2 var_j, column by column."""
    a = sp.csc_matrix(a)
    out = [0.0] * a.shape[0]
    for j in range(a.shape[1]):
        v = float(var_x[j])
        for p in range(a.indptr[j], a.indptr[j + 1]):
            val = float(a.data[p])
            out[a.indices[p]] += val * val * v
    return np.array(out)


def mixture_moments(weights, cond_mean, cond_var):
    """inference.rs:1436-1466: mean = sum_k w_k m_k, var = sum_k w_k (v_k + (m_k - mean)^2),
    k ascending per element."""
    K = len(weights)
    cm, cv = np.asarray(cond_mean, dtype=float), np.asarray(cond_var, dtype=float)
    mean = np.zeros(cm.shape[1])
    for k in range(K):
        mean = mean + weights[k] * cm[k]
    var = np.zeros(cm.shape[1])
    for k in range(K):
        d = cm[k] - mean
        var = var + weights[k] * (cv[k] + d * d)
    return mean, var


def predictor_moments(a, weights, cond_mean, cond_var):
    """inference.rs:1370-1384 (eta = A x*, eta-var = predictor_variances_diag per node; x* and
    its variances themselves when there is no A) and 1451-1466 (their mixture)."""
    if a is None:
        return mixture_moments(weights, cond_mean, cond_var)
    eta = [matvec_csc(a, m) for m in cond_mean]
    ev = [predictor_variances_diag(a, v) for v in cond_var]
    return mixture_moments(weights, eta, ev)


def integrate(mode, hessian, eval_node, f0=1.0, strategy="ccd", a=None):
    """run_inla_inference_a_cancellable node map + aggregation (inference.rs:1262-1466).

    ``eval_node(theta) -> (x_star, variances, log_post)``; ``strategy`` "ccd" (f0) or
    "grid" (step f0, threshold 4.0, evaluator = log_post at the mapped node). With the
    projector ``a`` the result also holds the predictor moments ("pred_mean", "pred_var").
    """
    m = len(mode)
    sigma = np.linalg.inv(-np.asarray(hessian))
    lam, V = np.linalg.eigh(sigma)
    to_theta = lambda zk: np.asarray(mode) + V @ (np.sqrt(np.abs(lam)) * np.asarray(zk, dtype=float))
    cache = {}

    def node(zk):
        key = tuple(float(v) for v in zk)
        if key not in cache:
            cache[key] = eval_node(to_theta(zk))
        return cache[key]

    if strategy == "grid":
        z, w = grid_design(m, f0, 4.0, lambda zk: node(zk)[2])
    else:
        z, w = ccd_design(m, f0)
    thetas = [to_theta(zk) for zk in z]
    res = [node(zk) for zk in z]
    lps = np.array([r[2] for r in res])
    mx = lps.max()
    dens = np.exp(lps - mx)
    sw = float(np.sum(w * dens))
    nw = w * dens / sw
    means = np.stack([r[0] for r in res])
    vars_ = np.stack([r[1] for r in res])
    mean = nw @ means
    var = nw @ (vars_ + (means - mean) ** 2)
    out = {"thetas": np.array(thetas), "weights": nw, "mean": mean, "var": var, "log_posts": lps,
           "mlik": mx + math.log(abs(sw))}
    if a is not None:
        out["pred_mean"], out["pred_var"] = predictor_moments(a, nw, means, vars_)
    return out


# ---------------------------------------------------------------------------
# model selection (crates/inla_stats/src/model_selection.rs)
# ---------------------------------------------------------------------------

CPO_DIFF = 3.0  # model_selection.rs:7


def mlik_gaussian(log_post_mode, neg_hessian, m):
    """model_selection.rs:25-73: in-place Cholesky of -H (row-major), None when not PD."""
    if m == 0:
        return log_post_mode
    a = [float(v) for v in np.ravel(neg_hessian)]
    log_det = 0.0
    for j in range(m):
        for k in range(j):
            ljk = a[j * m + k]
            a[j * m + j] -= ljk * ljk
        if a[j * m + j] <= 0.0:
            return None
        log_det += math.log(a[j * m + j])
        djj = math.sqrt(a[j * m + j])
        a[j * m + j] = djj
        for i in range(j + 1, m):
            for k in range(j):
                a[i * m + j] -= a[i * m + k] * a[j * m + k]
            a[i * m + j] /= djj
    return log_post_mode + 0.5 * m * math.log(2.0 * math.pi) - 0.5 * log_det


def _lik_or_none(family, eta, y, p1, p2):
    try:
        return eval_lik(family, eta, y, p1, p2)
    except OracleError:
        return None


def compute_dic(family, y, p1, p2, cond_eta, weights, mode_index):
    """model_selection.rs:82-150; None where the reference returns Err."""
    dev = []
    for eta in cond_eta:
        s = 0.0
        for i in range(len(y)):
            e = _lik_or_none(family, eta[i], y[i], p1[i], p2[i])
            if e is None:
                return None
            s += e[0]
        dev.append(-2.0 * s)
    mean_dev = 0.0
    for k in range(len(dev)):
        mean_dev += weights[k] * dev[k]
    p_eff = mean_dev - dev[mode_index]
    return {"dic": mean_dev + p_eff, "mean_deviance": mean_dev, "p_eff": p_eff}


def compute_waic(family, y, p1, p2, cond_eta, weights):
    """model_selection.rs:152-211; None where the reference returns Err."""
    lppd = p_waic = 0.0
    for i in range(len(y)):
        lls = []
        for eta in cond_eta:
            e = _lik_or_none(family, eta[i], y[i], p1[i], p2[i])
            if e is None:
                return None
            lls.append(e[0])
        mx = -math.inf
        for v in lls:
            mx = v if math.isnan(mx) else (mx if math.isnan(v) else max(mx, v))
        sw = ml = 0.0
        for k, v in enumerate(lls):
            sw += weights[k] * math.exp(v - mx)
            ml += weights[k] * v
        if not (math.isfinite(sw) and sw > 0.0):
            return None
        lppd += mx + math.log(sw)
        var = 0.0
        for k, v in enumerate(lls):
            d = v - ml
            var += weights[k] * d * d
        p_waic += var
    return {"waic": -2.0 * (lppd - p_waic), "lppd": lppd, "p_eff": p_waic}


def normal_cdf(x):
    """model_selection.rs:450-467 (Abramowitz & Stegun 7.1.26)."""
    a1, a2, a3, a4, a5, p = 0.254829592, -0.284496736, 1.421413741, -1.453152027, 1.061405429, 0.3275911
    sign = -1.0 if x < 0.0 else 1.0
    ax = abs(x)
    t = 1.0 / (1.0 + p * ax)
    y = 1.0 - (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t * math.exp(-ax * ax / 2.0)
    return 0.5 * (1.0 + sign * y)


def poisson_cdf(lam, k):
    """model_selection.rs:470-486."""
    if lam <= 0.0:
        return 1.0
    cdf, log_pmf = 0.0, -lam
    for j in range(k + 1):
        cdf += math.exp(log_pmf)
        if j < k:
            log_pmf += math.log(lam) - math.log(float(j + 1))
    return min(cdf, 1.0)


def binomial_cdf(n, p, k):
    """model_selection.rs:488-504 with the reference's Lanczos log-gamma."""
    if p <= 0.0:
        return 1.0
    if p >= 1.0:
        return 1.0 if k >= n else 0.0
    cdf = 0.0
    for j in range(k + 1):
        lc = log_gamma(n + 1.0) - log_gamma(j + 1.0) - log_gamma(float(n - j) + 1.0)
        cdf += math.exp(lc + j * math.log(p) + (n - j) * math.log(1.0 - p))
    return min(cdf, 1.0)


def _logistic(x):
    if x >= 0.0:
        z = math.exp(-x)
        return 1.0 / (1.0 + z)
    z = math.exp(x)
    return z / (1.0 + z)


def observation_cdf(family, y, p1, eta, variance):
    """model_selection.rs:398-448; None where the reference gives None."""
    family = FAMILIES.get(family, family)
    if family == 0:
        tv = 1.0 / p1 + variance
        if tv <= 0.0:
            return None
        return normal_cdf((y - eta) / math.sqrt(tv))
    if family == 1:
        lam = p1 * math.exp(eta)
        if lam < 0.0 or not math.isfinite(lam):
            return None
        yi = math.floor(y)
        return 0.0 if yi < 0 else poisson_cdf(lam, int(yi))
    if family == 2:
        prob = _logistic(eta)
        n = int(p1) if p1 > 0 else 0
        yi = math.floor(y)
        return 0.0 if yi < 0 else binomial_cdf(n, prob, min(int(yi), n))
    return None


def cpo_failure(family, y, p1, p2, mu, var):
    """check_cpo_failure_for_obs (model_selection.rs:327-396)."""
    if var <= 0.0 or not math.isfinite(var):
        return True
    e = _lik_or_none(family, mu, y, p1, p2)
    if e is None:
        return True
    g, c = e[1], -e[2]
    tau_loo = 1.0 / var - c
    if tau_loo <= 0.0 or not math.isfinite(tau_loo):
        return True
    var_loo = 1.0 / tau_loo
    std_loo = math.sqrt(var_loo)
    mu_loo = var_loo * (mu / var - c * mu + g)
    ld = []
    for step in (-3.0, -1.5, 0.0, 1.5, 3.0):
        x = mu_loo + step * std_loo
        prior = -0.5 * (x - mu) * (x - mu) / var
        e = _lik_or_none(family, x, y, p1, p2)
        if e is None:
            return True
        ld.append(prior + e[0])
    inc = all(not (ld[j] < ld[j - 1]) for j in range(1, 5))
    dec = all(not (ld[j] > ld[j - 1]) for j in range(1, 5))
    if inc or dec:
        return True
    mx = max(ld)
    return mx - ld[0] < CPO_DIFF or mx - ld[4] < CPO_DIFF


def compute_cpo_pit(family, y, p1, p2, cond_eta, cond_var, weights):
    """model_selection.rs:222-325: (cpo, pit, n_failures) with None entries."""
    n, K = len(y), len(weights)
    cpo, pit, nf = [None] * n, [None] * n, 0
    for i in range(n):
        if any(cpo_failure(family, y[i], p1[i], p2[i], cond_eta[k][i], cond_var[k][i]) for k in range(K)):
            nf += 1
            continue
        lls = []
        for k in range(K):
            e = _lik_or_none(family, cond_eta[k][i], y[i], p1[i], p2[i])
            if e is None:
                break
            lls.append(e[0])
        if len(lls) < K or len(lls) < 2:
            nf += 1
            continue
        max_neg = max(-v for v in lls)
        inv = 0.0
        for k in range(K):
            inv += weights[k] * math.exp(-lls[k] - max_neg)
        inv *= math.exp(max_neg)
        if not math.isfinite(inv) or inv <= 0.0:
            nf += 1
            continue
        cpo[i] = 1.0 / inv
        ps, ok = 0.0, True
        for k in range(K):
            f = observation_cdf(family, y[i], p1[i], cond_eta[k][i], cond_var[k][i])
            if f is None:
                ok = False
                break
            ps += weights[k] * f
        if ok and math.isfinite(ps):
            pit[i] = min(max(ps, 0.0), 1.0)
    return cpo, pit, nf


# ---------------------------------------------------------------------------
# hyperpriors (crates/inla_stats/src/priors.rs) and the SPDE theta map
# ---------------------------------------------------------------------------

def pc_prec_log_dens(theta, u, alpha):
    """priors.rs:532-548 with lambda = -ln(alpha)/u (priors.rs:78-86)."""
    lam = -math.log(alpha) / u
    return math.log(lam) - math.log(2.0) - lam * math.exp(-0.5 * theta) - 0.5 * theta


def pc_cor1_lambda(u, alpha):
    """priors.rs:611-660: scan, then 60 golden-section steps on the squared residual."""
    if not -1.0 < u < 1.0 or not math.sqrt((1.0 - u) / 2.0) < alpha < 1.0:
        raise ValueError("pc.cor1: invalid (u, alpha)")
    fun = lambda lam: ((1.0 - math.exp(-lam * math.sqrt(1.0 - u))) / (1.0 - math.exp(-lam * math.sqrt(2.0)))
                       - alpha) ** 2
    best, bf = 1.0, fun(1.0)
    for i in range(110):
        lam = 1e-7 + (10.0 - 1e-7) * i / 99.0 if i < 100 else 10.0 + 90.0 * (i - 100) / 9.0
        f = fun(lam)
        if f < bf:
            best, bf = lam, f
    lo, hi = max(best * 0.5, 1e-8), best * 2.0
    for _ in range(60):
        m1, m2 = lo + 0.382 * (hi - lo), lo + 0.618 * (hi - lo)
        if fun(m1) < fun(m2):
            hi = m2
        else:
            lo = m1
    lam = 0.5 * (lo + hi)
    if fun(lam) > 1e-6:
        raise ValueError("pc.cor1: failed to solve lambda")
    return lam


def pc_cor1_log_dens(theta, u, alpha):
    """priors.rs:662-683: density of rho = 2 e^theta / (1 + e^theta) - 1 with its Jacobian."""
    lam = pc_cor1_lambda(u, alpha)
    e = math.exp(theta)
    rho = 2.0 * e / (1.0 + e) - 1.0
    s = math.sqrt(1.0 - rho)
    return (math.log(lam) - lam * s - math.log(1.0 - math.exp(-math.sqrt(2.0) * lam)) - math.log(2.0 * s)
            + math.log(2.0) + theta - 2.0 * math.log1p(e))


def loggamma_log_dens(theta, shape, rate):
    """priors.rs:836-855 (rate convention, with the Jacobian of theta = log x)."""
    return shape * math.log(rate) - log_gamma(shape) + shape * theta - rate * math.exp(theta)


def pc_spde_log_dens(t1, t2, r0, alpha_r, s0, alpha_s, d=2.0):
    """priors.rs:127-147 (lambdas from quantiles) and 813-834 (density on log tau, log kappa)."""
    lam1 = -math.log(alpha_r) * r0 ** (d / 2.0)
    lam2 = -math.log(alpha_s) / s0
    log_rho = 0.5 * math.log(8.0) - t2
    log_sigma = -0.5 * math.log(4.0 * math.pi) - t1 - t2
    dh = d / 2.0
    s_rho = math.log(lam1 * dh) - dh * log_rho - lam1 * math.exp(-dh * log_rho)
    s_sig = math.log(lam2) + log_sigma - lam2 * math.exp(log_sigma)
    return s_rho + s_sig


def spde_coefs(log_tau, log_kappa):
    """spde.rs:70-140: Q = tau^2 (kappa^4 C + 2 kappa^2 G + G C^-1 G) coefficients."""
    t2 = math.exp(2 * log_tau)
    k2 = math.exp(2 * log_kappa)
    return np.array([t2 * k2 * k2, 2 * t2 * k2, t2])


def spde_neg_log_posterior(theta, model, a, y, max_iter=200, tol=1e-5, perm=None):
    """evaluate_neg_log_posterior (inla_stats/src/hyper_opt.rs:21-47) for the SPDE Gaussian model,
    theta = [log prec_eps, log tau, log kappa], default priors loggamma(1, 5e-5) + pc.spde(1, .05, 1, .01)."""
    q = model.matrix(spde_coefs(theta[1], theta[2]))
    try:
        r = laplace(q, a, "gaussian", y, p1=math.exp(theta[0]), max_iter=max_iter, tol=tol, perm=perm)
    except OracleError:
        return 1e12
    lp = loggamma_log_dens(theta[0], 1.0, 5e-5) + pc_spde_log_dens(theta[1], theta[2], 1.0, 0.05, 1.0, 0.01)
    return -(r["mlik"] + lp)


# ---------------------------------------------------------------------------
# meshes (crates/inla_fmesher/src/fmesher.rs), pure Python for small meshes
# ---------------------------------------------------------------------------

GEOM_EPSILON = 1e-15  # fmesher.rs:5


def _sa2(a, b, c):
    """signed_area2 (fmesher.rs:897-899)."""
    return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])


def mesh_neighbors(triangles):
    """build_mesh2d's edge map (fmesher.rs:122-139): nbr[t][e] across the edge opposite vertex e."""
    nbr = [[-1, -1, -1] for _ in triangles]
    open_edges = {}
    for t, tri in enumerate(triangles):
        for e in range(3):
            a, b = int(tri[(e + 1) % 3]), int(tri[(e + 2) % 3])
            if (b, a) in open_edges:
                ot, oe = open_edges.pop((b, a))
                nbr[t][e], nbr[ot][oe] = ot, t
            elif (a, b) in open_edges:
                raise OracleError(f"non-manifold edge detected between vertices {a} and {b}")
            else:
                open_edges[(a, b)] = (t, e)
    return nbr


def fem_blocks(vertices, triangles, triangle_scale=None, diffusion=(1.0, 0.0, 1.0)):
    """assemble_fem_blocks_diffusion_unchecked (fmesher.rs:544-626) with coalesce (fmesher.rs:89-107):
    dict of {(row, col): value} for c0, c1, g1, b1, and the areas."""
    hxx, hxy, hyy = diffusion
    nbr = mesh_neighbors(triangles)
    trip = {"c0": [], "c1": [], "g1": [], "b1": []}
    areas = []
    for t, tv in enumerate(triangles):
        s = [tuple(map(float, vertices[int(v)])) for v in tv]
        e = [(s[2][0] - s[1][0], s[2][1] - s[1][1]), (s[0][0] - s[2][0], s[0][1] - s[2][1]),
             (s[1][0] - s[0][0], s[1][1] - s[0][1])]
        area = 0.5 * abs(_sa2(s[0], s[1], s[2]))
        areas.append(area)
        fa = 0.5 * abs(e[0][0] * e[1][1] - e[0][1] * e[1][0])
        fa = area if fa <= GEOM_EPSILON else fa
        scale = 1.0 if triangle_scale is None else float(triangle_scale[t])
        eij = [[0.0] * 3 for _ in range(3)]
        for i in range(3):
            gi = (e[i][1], -e[i][0])
            for j in range(i, 3):
                gj = (e[j][1], -e[j][0])
                hx = hxx * gi[0] + hxy * gi[1]
                hy = hxy * gi[0] + hyy * gi[1]
                eij[i][j] = hx * gj[0] + hy * gj[1]
                eij[j][i] = eij[i][j]
        v = [int(x) for x in tv]
        for i in range(3):
            trip["c0"].append((v[i], v[i], area / 3.0))
            trip["c1"].append((v[i], v[i], area / 6.0))
            trip["g1"].append((v[i], v[i], scale * eij[i][i] / (4.0 * fa)))
            for j in range(i + 1, 3):
                trip["c1"] += [(v[i], v[j], area / 12.0), (v[j], v[i], area / 12.0)]
                vij = scale * eij[i][j] / (4.0 * fa)
                trip["g1"] += [(v[i], v[j], vij), (v[j], v[i], vij)]
        bnd = [nbr[t][k] < 0 for k in range(3)]
        if any(bnd):
            vij = -1.0 / (4.0 * fa)
            for i in range(3):
                for j in range(3):
                    for k in range(3):
                        if bnd[k] and i != k:
                            trip["b1"].append((v[i], v[j], scale * eij[k][j] * vij))
    out = {"areas": areas}
    for name, tr in trip.items():
        merged = {}
        for r, c, x in sorted(tr, key=lambda q: (q[0], q[1])):   # stable, then summed in order
            merged[(r, c)] = merged[(r, c)] + x if (r, c) in merged else x
        out[name] = merged
    return out


def locate_point(vertices, triangles, nbr, start, p):
    """locate_point_from (fmesher.rs:222-263) + barycentric_coords (822-831): (triangle, bary)."""
    cur, remaining = start, max(len(triangles) * 3, 1)
    while remaining > 0:
        remaining -= 1
        tv = [int(x) for x in triangles[cur]]
        a, b, c = (tuple(map(float, vertices[v])) for v in tv)
        orient = 1.0 if _sa2(a, b, c) >= 0.0 else -1.0
        most_negative, leaving = 0.0, None
        for e in range(3):
            side = orient * _sa2(tuple(map(float, vertices[tv[(e + 1) % 3]])),
                                 tuple(map(float, vertices[tv[(e + 2) % 3]])), p)
            if side < most_negative:
                most_negative, leaving = side, e
        if most_negative >= -GEOM_EPSILON:
            den = _sa2(a, b, c)
            w0 = _sa2(b, c, p) / den
            w1 = _sa2(c, a, p) / den
            return cur, (w0, w1, 1.0 - w0 - w1)
        if leaving is None or nbr[cur][leaving] < 0:
            return -1, None
        cur = nbr[cur][leaving]
    return -1, None


def projector_triplets(vertices, triangles, points):
    """observation_projector_triplets (fmesher.rs:168-219)."""
    nbr = mesh_neighbors(triangles)
    trips, start = [], 0
    for row, p in enumerate(points):
        t, w = locate_point(vertices, triangles, nbr, start, (float(p[0]), float(p[1])))
        if t < 0:
            raise OracleError(f"observation point ({p[0]}, {p[1]}) is outside the mesh")
        start = t
        for k in range(3):
            if abs(w[k]) > GEOM_EPSILON:
                trips.append((row, int(triangles[t][k]), w[k]))
    return trips


def spde_precision(c0_diag, g1, kappa, tau):
    """spde_precision_csc (crates/inla_stats/src/spde.rs:70-140) as a dict {(i, j): value}:
    tau^2 (kappa^4 C0 + 2 kappa^2 G1 + G1 C0^-1 G1), with (G1 C0^-1 G1)_ij summed over
    ascending k as sum_k (G1_ik (1 / c0_k)) G1_kj."""
    g = sp.csc_matrix(g1)
    n = g.shape[0]
    for v in c0_diag:
        if abs(v) < 1e-15:
            raise OracleError("Zero entry in mass matrix c0 diagonal")
    cinv = [1.0 / float(v) for v in c0_diag]
    cols = [dict() for _ in range(n)]
    for j in range(n):
        for p in range(g.indptr[j], g.indptr[j + 1]):
            cols[j][int(g.indices[p])] = cols[j].get(int(g.indices[p]), 0.0) + float(g.data[p])
    gcg = {}
    for j in range(n):
        for k in sorted(cols[j]):
            gkj = cols[j][k]
            for i, gik in cols[k].items():
                gcg[(i, j)] = gcg.get((i, j), 0.0) + (gik * cinv[k]) * gkj
    k2 = kappa * kappa
    k4 = k2 * k2
    q = {}
    for i in range(n):
        q[(i, i)] = k4 * float(c0_diag[i])
    for j in range(n):
        for i, v in cols[j].items():
            q[(i, j)] = q.get((i, j), 0.0) + 2.0 * k2 * v
    for key, v in gcg.items():
        q[key] = q.get(key, 0.0) + v
    t2 = tau * tau
    return {key: v * t2 for key, v in q.items()}, gcg


# ---------------------------------------------------------------------------
# one-dimensional marginals (crates/inla_stats/src/marginals.rs)
# ---------------------------------------------------------------------------

def _phi(x, mu, var):
    """marginals.rs:73-80."""
    if not (var > 0.0 and math.isfinite(var)):
        return 0.0
    s = math.sqrt(var)
    z = (x - mu) / s
    return math.exp(-0.5 * z * z) / (s * math.sqrt(2.0 * math.pi))


def _trapezoid(x, y):
    """Marginal1D::integrate (marginals.rs:20-30)."""
    s = 0.0
    for i in range(len(x) - 1):
        s += 0.5 * (y[i] + y[i + 1]) * (x[i + 1] - x[i])
    return s


def gaussian_mixture_marginal(means, vars_, weights, n_points=201, n_sd=4.0):
    """marginals.rs:83-135: (x, y) with unit trapezoid mass."""
    K = len(means)
    mu = 0.0
    for k in range(K):
        mu += weights[k] * means[k]
    var = 0.0
    for k in range(K):
        d = means[k] - mu
        var += weights[k] * (vars_[k] + d * d)
    if not (var > 0.0 and math.isfinite(var)):
        var = 1e-8
    half = max(n_sd, 1.0) * math.sqrt(var)
    lo, hi = mu - half, mu + half
    x, y = [], []
    for i in range(n_points):
        xi = lo + (hi - lo) * float(i) / float(n_points - 1)
        yi = 0.0
        for k in range(K):
            yi += weights[k] * _phi(xi, means[k], vars_[k])
        x.append(xi)
        y.append(yi)
    mass = _trapezoid(x, y)
    if mass > 0.0 and math.isfinite(mass):
        y = [v / mass for v in y]
    return np.array(x), np.array(y)


def hyperpar_marginal_from_nodes(theta_j, weights, n_points=201, n_sd=4.0):
    """marginals.rs:137-162."""
    mu = 0.0
    for k in range(len(theta_j)):
        mu += weights[k] * theta_j[k]
    v = 0.0
    for k in range(len(theta_j)):
        d = theta_j[k] - mu
        v += weights[k] * d * d
    h2 = max(v, 1e-8) * 1.0
    return gaussian_mixture_marginal(list(theta_j), [h2] * len(theta_j), weights, n_points, n_sd)


def marginal_quantiles(x, y, probs):
    """marginal_cdf + marginal_quantiles (marginals.rs:183-226)."""
    f = [0.0] * len(x)
    for i in range(len(x) - 1):
        f[i + 1] = f[i] + 0.5 * (y[i] + y[i + 1]) * (x[i + 1] - x[i])
    mass = f[-1]
    if mass > 0.0:
        f = [v / mass for v in f]
    out = []
    for p in probs:
        q = x[-1]
        for i in range(1, len(f)):
            if f[i] >= p:
                t = 0.0 if abs(f[i] - f[i - 1]) < 1e-15 else (p - f[i - 1]) / (f[i] - f[i - 1])
                q = x[i - 1] + t * (x[i] - x[i - 1])
                break
        out.append(q)
    return np.array(out)
