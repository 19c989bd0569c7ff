"""Seeded synthetic inputs for the INLA hot path (input side of the Laplace loop).

Each latent precision is written as a linear combination of fixed-pattern
component matrices, ``Q(theta) = sum_t c_t(theta) * M_t``, so that every
theta-point, Newton iterate and batched problem shares one symbolic analysis
and the device only refreshes values.

Reference behaviour restated here (inputs only; none of this is timed):

* SPDE precision ``tau^2 (kappa^4 C~ + 2 kappa^2 G + G C~^-1 G)`` —
  crates/inla_stats/src/spde.rs:70-140.
* P1 FEM blocks: lumped mass ``C~_ii = sum area/3`` and stiffness
  ``G_ij = e_i . e_j / (4 area)`` — crates/inla_fmesher/src/fmesher.rs:544-626.
* Barycentric projector rows, weights with ``|w| <= 1e-15`` dropped —
  crates/inla_fmesher/src/fmesher.rs:175-219, 822-831.
* Besag graph Laplacian — crates/inla_stats/src/besag.rs:127-152.
* AR1 conditional-precision form ``tau * tridiag(1, 1+rho^2, ..., 1; -rho)`` —
  crates/inla_stats/src/ar1.rs:9-69.
* ``scale.model`` — crates/inla_math/src/design.rs:140-195.
* Grouped effects: ``kron(Q_group, Q_main)``, group-major latent order with the
  main index fastest — crates/inla_stats/src/structured.rs:475-540; group AR1
  ``rho = 2 / (1 + e^-theta) - 1`` — structured.rs:348-356; per-group copies of
  the main model's component sum-to-zero rows — structured.rs:782-807, 884-963.
* Sum-to-zero constraint rows and block embedding —
  crates/inla_math/src/constraints.rs:49-68, 111-149.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

GEOM_EPSILON = 1e-15
SEED_BASE = 20261203


# ---------------------------------------------------------------------------
# meshes and FEM
# ---------------------------------------------------------------------------

def grid_mesh(nx: int, rng: np.random.Generator, jitter: float = 0.2):
    """Structured triangulation of the unit square from an ``nx x nx`` vertex grid.

    Interior vertices are jittered by ``U(+-jitter*h)`` per axis (x draws first,
    then y), boundary vertices stay on the boundary. Every cell is split on the
    same diagonal; triangles are counter-clockwise.
    """
    h = 1.0 / (nx - 1)
    gx, gy = np.meshgrid(np.arange(nx) * h, np.arange(nx) * h, indexing="xy")
    vx = gx.ravel().copy()
    vy = gy.ravel().copy()
    ii = np.arange(nx * nx) % nx
    jj = np.arange(nx * nx) // nx
    interior = (ii > 0) & (ii < nx - 1) & (jj > 0) & (jj < nx - 1)
    k = int(interior.sum())
    dx = rng.uniform(-jitter * h, jitter * h, size=k)
    dy = rng.uniform(-jitter * h, jitter * h, size=k)
    vx[interior] += dx
    vy[interior] += dy
    c = np.arange((nx - 1) * (nx - 1))
    ci = c % (nx - 1)
    cj = c // (nx - 1)
    v00 = cj * nx + ci
    v10 = v00 + 1
    v01 = v00 + nx
    v11 = v01 + 1
    t1 = np.stack([v00, v10, v11], axis=1)
    t2 = np.stack([v00, v11, v01], axis=1)
    tris = np.empty((2 * len(c), 3), dtype=np.int64)
    tris[0::2] = t1
    tris[1::2] = t2
    verts = np.stack([vx, vy], axis=1)
    return verts, tris


def fem_matrices(verts: np.ndarray, tris: np.ndarray):
    """Lumped mass diagonal ``c0`` and stiffness ``G`` (CSC) of P1 elements."""
    nv = len(verts)
    s0, s1, s2 = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    e0 = s2 - s1
    e1 = s0 - s2
    e2 = s1 - s0
    area2 = (s1[:, 0] - s0[:, 0]) * (s2[:, 1] - s0[:, 1]) - (s1[:, 1] - s0[:, 1]) * (s2[:, 0] - s0[:, 0])
    area = 0.5 * np.abs(area2)
    fa = 0.5 * np.abs(e0[:, 0] * e1[:, 1] - e0[:, 1] * e1[:, 0])
    fa = np.where(fa <= GEOM_EPSILON, area, fa)
    e = [e0, e1, e2]
    c0 = np.zeros(nv)
    for i in range(3):
        np.add.at(c0, tris[:, i], area / 3.0)
    rows, cols, vals = [], [], []
    for i in range(3):
        for j in range(3):
            eij = e[i][:, 0] * e[j][:, 0] + e[i][:, 1] * e[j][:, 1]
            rows.append(tris[:, i])
            cols.append(tris[:, j])
            vals.append(eij / (4.0 * fa))
    g = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nv, nv)).tocsc()
    g.sum_duplicates()
    g.sort_indices()
    return c0, g


def _signed_area2(ax, ay, bx, by, cx, cy):
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax)


def grid_projector(verts: np.ndarray, tris: np.ndarray, nx: int, pts: np.ndarray) -> sp.csr_matrix:
    """Barycentric projector for points inside the jittered grid mesh.

    Any triangle containing the point gives the same non-zero weights; the
    candidate triangles are those of the 3x3 cells around the point's
    unjittered cell.
    """
    h = 1.0 / (nx - 1)
    nc = nx - 1
    n = len(pts)
    ci0 = np.clip((pts[:, 0] / h).astype(np.int64), 0, nc - 1)
    cj0 = np.clip((pts[:, 1] / h).astype(np.int64), 0, nc - 1)
    found = np.zeros(n, dtype=bool)
    wts = np.zeros((n, 3))
    tv = np.zeros((n, 3), dtype=np.int64)
    for dj in (0, -1, 1):
        for di in (0, -1, 1):
            ci = np.clip(ci0 + di, 0, nc - 1)
            cj = np.clip(cj0 + dj, 0, nc - 1)
            for half in (0, 1):
                t = 2 * (cj * nc + ci) + half
                a, b, c = verts[tris[t, 0]], verts[tris[t, 1]], verts[tris[t, 2]]
                den = _signed_area2(a[:, 0], a[:, 1], b[:, 0], b[:, 1], c[:, 0], c[:, 1])
                w0 = _signed_area2(b[:, 0], b[:, 1], c[:, 0], c[:, 1], pts[:, 0], pts[:, 1]) / den
                w1 = _signed_area2(c[:, 0], c[:, 1], a[:, 0], a[:, 1], pts[:, 0], pts[:, 1]) / den
                w2 = 1.0 - w0 - w1
                inside = (w0 >= -GEOM_EPSILON) & (w1 >= -GEOM_EPSILON) & (w2 >= -GEOM_EPSILON)
                take = inside & ~found
                wts[take] = np.stack([w0, w1, w2], axis=1)[take]
                tv[take] = tris[t][take]
                found |= take
    if not found.all():
        raise ValueError("observation point outside the mesh")
    rows = np.repeat(np.arange(n), 3)
    w = wts.ravel()
    keep = np.abs(w) > GEOM_EPSILON
    a = sp.coo_matrix((w[keep], (rows[keep], tv.ravel()[keep])), shape=(n, len(verts))).tocsr()
    a.sum_duplicates()
    a.sort_indices()
    return a


# ---------------------------------------------------------------------------
# component model container
# ---------------------------------------------------------------------------

@dataclass
class LatentModel:
    """``Q(theta) = sum_t coef_t(theta) * comps[t]`` on one shared pattern.

    ``pattern`` is the full symmetric CSC pattern (both triangles, sorted
    indices, diagonal present) that every component is expressed on, and
    ``comp_values[t]`` holds component ``t``'s values on that pattern.
    """

    n: int
    pattern: sp.csc_matrix
    comp_values: np.ndarray  # (T, nnz)
    kind: str
    info: dict = field(default_factory=dict)

    @property
    def n_comp(self) -> int:
        return self.comp_values.shape[0]

    def values(self, coefs) -> np.ndarray:
        return np.asarray(coefs, dtype=np.float64) @ self.comp_values

    def matrix(self, coefs) -> sp.csc_matrix:
        q = self.pattern.copy()
        q.data = self.values(coefs)
        return q


def _on_pattern(pattern: sp.csc_matrix, m: sp.spmatrix) -> np.ndarray:
    """Values of ``m`` on ``pattern`` (zero where ``m`` has no entry)."""
    m = sp.csc_matrix(m)
    m.sum_duplicates()
    pc = pattern.tocoo()
    key_p = pc.col.astype(np.int64) * pattern.shape[0] + pc.row
    mc = m.tocoo()
    key_m = mc.col.astype(np.int64) * pattern.shape[0] + mc.row
    order = np.argsort(key_m)
    key_m = key_m[order]
    vals = mc.data[order]
    pos = np.searchsorted(key_m, key_p)
    pos = np.clip(pos, 0, max(len(key_m) - 1, 0))
    out = np.zeros(len(key_p))
    if len(key_m):
        hit = key_m[pos] == key_p
        out[hit] = vals[pos[hit]]
    return out


def union_pattern(n: int, mats) -> sp.csc_matrix:
    acc = sp.identity(n, format="csc") * 0.0
    acc = acc + sp.identity(n, format="csc")  # diagonal always present
    for m in mats:
        mm = sp.csc_matrix(m, copy=True)
        mm.data = np.ones_like(mm.data)
        acc = acc + abs(mm) + abs(mm.T)
    acc = sp.csc_matrix(acc)
    acc.sum_duplicates()
    acc.sort_indices()
    acc.data = np.ones_like(acc.data)
    return acc


def build_latent(n: int, comps, kind: str, extra_pattern=(), info=None) -> LatentModel:
    pat = union_pattern(n, list(comps) + list(extra_pattern))
    vals = np.stack([_on_pattern(pat, c) for c in comps])
    return LatentModel(n=n, pattern=pat, comp_values=vals, kind=kind, info=info or {})


def spde_components(c0: np.ndarray, g: sp.csc_matrix):
    """Components of ``tau^2 (kappa^4 C + 2 kappa^2 G + G C^-1 G)``."""
    cinv = sp.diags(1.0 / c0)
    gcg = (g @ cinv @ g).tocsc()
    return [sp.diags(c0).tocsc(), g.tocsc(), gcg]


def spde_coefs(log_tau: float, log_kappa: float):
    """Coefficients (and d/d log_tau, d/d log_kappa) for :func:`spde_components`."""
    t2 = np.exp(2 * log_tau)
    k2 = np.exp(2 * log_kappa)
    c = np.array([t2 * k2 * k2, 2 * t2 * k2, t2])
    d_tau = 2 * c
    d_kappa = np.array([4 * c[0], 2 * c[1], 0.0])
    return c, np.stack([d_tau, d_kappa])


# ---------------------------------------------------------------------------
# graphs
# ---------------------------------------------------------------------------

def lattice_adjacency(nr: int, nc: int) -> sp.csr_matrix:
    """Rook adjacency of an ``nr x nc`` lattice (row-major node numbering)."""
    idx = np.arange(nr * nc).reshape(nr, nc)
    a = np.concatenate([idx[:, :-1].ravel(), idx[:-1, :].ravel()])
    b = np.concatenate([idx[:, 1:].ravel(), idx[1:, :].ravel()])
    n = nr * nc
    m = sp.coo_matrix((np.ones(len(a)), (a, b)), shape=(n, n))
    return (m + m.T).tocsr()


def besag_structure(adj: sp.spmatrix) -> sp.csc_matrix:
    """Graph Laplacian ``R = D - W`` (intrinsic Besag structure), with a unit diagonal for
    regions without neighbours (besag.rs:127-152: singletons are N(0, 1 / tau))."""
    adj = sp.csr_matrix(adj)
    deg = np.asarray(adj.sum(axis=1)).ravel()
    deg = np.where(deg == 0, 1.0, deg)
    return (sp.diags(deg) - adj).tocsc()


def ar1_components(n: int):
    """``tau * (M0 + rho^2 M1 - rho M2)`` pieces of the AR1 conditional precision."""
    m0 = sp.identity(n, format="csc")
    d1 = np.ones(n)
    d1[0] = d1[-1] = 0.0
    m1 = sp.diags(d1).tocsc()
    off = np.ones(n - 1)
    m2 = sp.diags([off, off], [-1, 1]).tocsc()
    return m0, m1, m2


def ar1_precision(n: int, rho: float, tau: float) -> sp.csc_matrix:
    m0, m1, m2 = ar1_components(n)
    return (tau * (m0 + rho * rho * m1 - rho * m2)).tocsc()


# ---------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------

@dataclass
class SpdeProblem:
    model: LatentModel
    a: sp.csr_matrix       # n_obs x n projector
    y: np.ndarray
    verts: np.ndarray
    tris: np.ndarray
    truth: dict
    theta_init: np.ndarray  # [log prec_eps, log tau, log kappa]


def make_spde_problem(nx: int = 200, n_obs: int = 20_000, seed: int = SEED_BASE + 2,
                      range_true: float = 0.2, sigma_true: float = 1.0,
                      noise_sd: float = 0.1, family: str = "gaussian", nb_size: float = 5.0) -> SpdeProblem:
    """SPDE Matern alpha=2 on the jittered ``nx x nx`` grid with Gaussian data (or, with
    ``family="nbinomial"``, negative-binomial counts with size ``nb_size`` and mean
    ``exp(A x)``).

    Draw order: interior jitter x, jitter y, field innovations z (n), point
    locations (n_obs x 2), observation noise (n_obs) or counts. The field is an exact
    draw ``x = K^-1 C~^{1/2} z`` with ``K = tau (kappa^2 C~ + G)``, whose
    covariance ``K^-1 C~ K^-1`` is the SPDE ``Q^-1``.
    """
    rng = np.random.default_rng(seed)
    verts, tris = grid_mesh(nx, rng)
    c0, g = fem_matrices(verts, tris)
    comps = spde_components(c0, g)
    n = len(verts)
    kappa = np.sqrt(8.0) / range_true
    tau = 1.0 / (2.0 * np.sqrt(np.pi) * kappa * sigma_true)
    z = rng.standard_normal(n)
    k = (tau * (kappa * kappa * sp.diags(c0) + g)).tocsc()
    x = spla.spsolve(k, np.sqrt(c0) * z)
    pts = rng.uniform(0.0, 1.0, size=(n_obs, 2))
    a = grid_projector(verts, tris, nx, pts)
    if family == "nbinomial":
        mu = np.exp(a @ x)
        y = rng.negative_binomial(nb_size, nb_size / (nb_size + mu)).astype(float)
    else:
        y = a @ x + noise_sd * rng.standard_normal(n_obs)
    ata = (a.T @ a).tocsc()
    model = build_latent(n, comps, "spde", extra_pattern=[ata],
                         info={"nx": nx, "c0": c0})
    truth = {"log_prec": float(np.log(1.0 / noise_sd ** 2)), "log_tau": float(np.log(tau)),
             "log_kappa": float(np.log(kappa)), "x": x}
    return SpdeProblem(model=model, a=a, y=y, verts=verts, tris=tris, truth=truth,
                       theta_init=np.zeros(3))


# ---------------------------------------------------------------------------
# intrinsic models: scale.model and constraints
# ---------------------------------------------------------------------------

def scale_model(r: sp.spmatrix):
    """``scale_model_csc`` (design.rs:150-195): ``fac = exp(mean(log(diag(ginv(R)))))``
    over the positive finite entries, eigenvalues above ``sqrt(eps) * max(max_lam, 1)``
    kept; returns ``(fac * R, fac)``. (The reference diagonalizes by Jacobi sweeps, here
    by LAPACK: the factor agrees to rounding.)"""
    n = r.shape[0]
    if n == 1:
        return sp.identity(1, format="csc"), 1.0
    lam, v = np.linalg.eigh(np.asarray(sp.csr_matrix(r).todense()))
    max_lam = max(abs(max(float(lam.max()), 0.0)), 1.0)
    tol = np.sqrt(np.finfo(np.float64).eps) * max_lam
    keep = lam > tol
    d = (v[:, keep] ** 2) @ (1.0 / lam[keep])
    ok = (d > 0.0) & np.isfinite(d)
    if not ok.any():
        raise ValueError("scale_model: ginv has no positive diagonal")
    fac = float(np.exp(np.mean(np.log(d[ok]))))
    return (fac * sp.csc_matrix(r)).tocsc(), fac


def sum_to_zero_constraint(n: int, k: int = 1):
    """``sum_to_zero_constraint`` (constraints.rs:111-149): row 0 = 1/sqrt(n); row 1 (k=2)
    the centred index scaled to unit norm. Returns ``(C [k x n], e [k])``."""
    if n <= 0 or k not in (1, 2):
        raise ValueError("sum_to_zero_constraint: n > 0 and k in {1, 2}")
    c = np.zeros((k, n))
    c[0] = 1.0 / np.sqrt(n)
    if k == 2:
        v = np.arange(n, dtype=float) - (n - 1) / 2.0
        scale = np.sqrt(np.sum(v * v))
        if scale < 1e-14:
            raise ValueError("sum_to_zero_constraint: degenerate linear row")
        c[1] = v / scale
    return c, np.zeros(k)


def component_constraints(adj: sp.spmatrix):
    """component_constraints (structured.rs:782-806): one sum-to-zero row per connected
    component of more than one node, weight 1 / sqrt(size) on its nodes, components in order of
    their first node; singletons stay unconstrained. Returns ``(C [k x n], e [k])`` or None."""
    adj = sp.csr_matrix(adj)
    n = adj.shape[0]
    seen = np.zeros(n, dtype=bool)
    rows = []
    for s0 in range(n):
        if seen[s0]:
            continue
        comp, stack = [], [s0]
        seen[s0] = True
        while stack:
            u = stack.pop()
            comp.append(u)
            for v in adj.indices[adj.indptr[u]:adj.indptr[u + 1]]:
                if not seen[v]:
                    seen[v] = True
                    stack.append(v)
        if len(comp) > 1:
            r = np.zeros(n)
            r[comp] = 1.0 / np.sqrt(len(comp))
            rows.append(r)
    if not rows:
        return None
    return np.array(rows), np.zeros(len(rows))


def plane_constraint_2d(nrow: int, ncol: int):
    """``plane_constraint_2d`` (constraints.rs:219-266) for a column-major lattice
    (``node = j * nrow + i``): constant, row trend, column trend, each unit norm."""
    if nrow <= 0 or ncol <= 0:
        raise ValueError("plane_constraint_2d: nrow and ncol must be > 0")
    n = nrow * ncol
    j, i = np.meshgrid(np.arange(ncol), np.arange(nrow), indexing="ij")
    vi = (i.ravel() - (nrow - 1) / 2.0).astype(float)
    vj = (j.ravel() - (ncol - 1) / 2.0).astype(float)
    si, sj = np.sqrt(np.sum(vi * vi)), np.sqrt(np.sum(vj * vj))
    if si < 1e-14 or sj < 1e-14:
        raise ValueError("plane_constraint_2d: degenerate row/col trend")
    c = np.stack([np.full(n, 1.0 / np.sqrt(n)), vi / si, vj / sj])
    return c, np.zeros(3)


def embed_constraint(c: np.ndarray, full_n: int, offset: int) -> np.ndarray:
    """``ConstraintSpec::embed`` (constraints.rs:49-68): place the block at ``offset``."""
    c = np.atleast_2d(c)
    if offset + c.shape[1] > full_n:
        raise ValueError("embed: block exceeds full dimension")
    out = np.zeros((c.shape[0], full_n))
    out[:, offset:offset + c.shape[1]] = c
    return out


@dataclass
class BesagProblem:
    model: LatentModel
    a: sp.csr_matrix      # n_obs x n projector [1 | x | I]
    y: np.ndarray
    constraint: tuple     # (C [1 x n], e [1]): sum-to-zero on the region block
    scale: float          # scale.model factor of the Besag structure
    truth: dict


BESAG_FIXED_PREC = 1e-4  # precision of the intercept and covariate effects


def make_besag_problem(nr: int = 30, nc: int = 30, seed: int = SEED_BASE + 1, tau_true: float = 2.0,
                       beta0: float = 0.5, beta1: float = 0.3) -> BesagProblem:
    """Poisson GLMM ``y ~ 1 + x + f(region, besag, scale.model)`` on an ``nr x nc`` rook
    lattice with a sum-to-zero constraint on the Besag block.

    Latent layout [intercept, x-effect, region (nr*nc)] (fixed effects first, precision
    1e-4); ``Q(theta) = M0 + exp(theta) M1`` with ``M0 = diag(1e-4, 1e-4, 0, ...)`` and
    ``M1 = blockdiag(0, 0, fac * R)``. Draw order: covariate x (n_region), Besag
    innovations (n_region - 1, on the scaled structure's non-null eigenvectors, tau_true),
    Poisson counts.
    """
    rng = np.random.default_rng(seed)
    adj = lattice_adjacency(nr, nc)
    r = besag_structure(adj)
    rs, fac = scale_model(r)
    nreg = nr * nc
    n = nreg + 2
    x = rng.standard_normal(nreg)
    lam, v = np.linalg.eigh(np.asarray(rs.todense()))
    tol = np.sqrt(np.finfo(np.float64).eps) * max(float(lam.max()), 1.0)
    keep = lam > tol
    z = rng.standard_normal(int(keep.sum()))
    u = v[:, keep] @ (z / np.sqrt(tau_true * lam[keep]))
    eta = beta0 + beta1 * x + u
    y = rng.poisson(np.exp(eta)).astype(float)
    rows = np.repeat(np.arange(nreg), 3)
    cols = np.stack([np.zeros(nreg, dtype=int), np.ones(nreg, dtype=int), 2 + np.arange(nreg)], axis=1).ravel()
    vals = np.stack([np.ones(nreg), x, np.ones(nreg)], axis=1).ravel()
    a = sp.csr_matrix((vals, (rows, cols)), shape=(nreg, n))
    d0 = np.zeros(n)
    d0[:2] = BESAG_FIXED_PREC
    m0 = sp.diags(d0).tocsc()
    m1 = sp.block_diag([sp.csc_matrix((2, 2)), rs]).tocsc()
    ata = (a.T @ a).tocsc()
    model = build_latent(n, [m0, m1], "besag", extra_pattern=[ata], info={"nr": nr, "nc": nc})
    c, e = sum_to_zero_constraint(nreg, 1)
    cons = (embed_constraint(c, n, 2), e)
    truth = {"log_tau": float(np.log(tau_true)), "u": u, "beta": (beta0, beta1), "x": x}
    return BesagProblem(model=model, a=a, y=y, constraint=cons, scale=fac, truth=truth)


def besag_coefs(log_tau: float):
    """Coefficients of :func:`make_besag_problem`'s components and d/d log_tau."""
    t = float(np.exp(log_tau))
    return np.array([1.0, t]), np.array([[0.0, t]])


@dataclass
class GroupProblem:
    model: LatentModel
    a: sp.csr_matrix      # n_obs x n projector [1 | I | I]
    y: np.ndarray
    ntrials: float
    constraint: tuple     # (C [T x n], e [T]): sum-to-zero of the spatial block per time
    dims: tuple           # (n_space, T)
    truth: dict


def group_constraint(n_space: int, T: int, offset: int, n: int):
    """``grouped_constraints`` (structured.rs:884-963) for a connected Besag main model and an
    AR1 group model (no constraint of its own): row t is 1/sqrt(n_space) on time slice t."""
    c = np.zeros((T, n))
    w = 1.0 / np.sqrt(n_space)
    for t in range(T):
        c[t, offset + t * n_space:offset + (t + 1) * n_space] = w
    return c, np.zeros(T)


def make_group_problem(nr: int = 50, nc: int = 50, T: int = 40, seed: int = SEED_BASE + 3, rho: float = 0.8,
                       tau_b: float = 1.0, tau_g: float = 1.0, tau_iid: float = 4.0, beta0: float = 0.0,
                       ntrials: float = 10.0) -> GroupProblem:
    """Space-time group model: Besag on an ``nr x nc`` rook lattice grouped by AR1 over ``T``
    times, plus iid and an intercept; binomial likelihood with ``ntrials`` trials, one
    observation per space-time cell.

    Latent layout [intercept, group effect (T * n_space, group-major), iid (T * n_space)];
    ``Q(theta) = M_int + tau_b tau_g (K0 + rho^2 K1 - rho K2) + tau_iid M_iid`` with
    ``K_i = kron(AR1 piece_i, R)``. theta = [log tau_b, log tau_g, logit-type rho, log tau_iid].
    Draw order: per-eigenvector AR1 paths of the spatial field (n_space - 1 paths of length
    T), iid effects, binomial counts.
    """
    rng = np.random.default_rng(seed)
    r = besag_structure(lattice_adjacency(nr, nc))
    ns = nr * nc
    nst = ns * T
    n = 1 + 2 * nst
    lam, v = np.linalg.eigh(np.asarray(r.todense()))
    keep = lam > np.sqrt(np.finfo(np.float64).eps) * max(float(lam.max()), 1.0)
    lk, vk = lam[keep], v[:, keep]
    z = np.zeros((T, len(lk)))
    z[0] = rng.standard_normal(len(lk)) / np.sqrt(1.0 - rho * rho)
    for t in range(1, T):
        z[t] = rho * z[t - 1] + rng.standard_normal(len(lk))
    u = (z / np.sqrt(tau_b * tau_g * lk)) @ vk.T          # (T, ns), row t = time slice t
    w = rng.standard_normal(nst) / np.sqrt(tau_iid)
    eta = beta0 + u.ravel() + w
    y = rng.binomial(int(ntrials), 1.0 / (1.0 + np.exp(-eta))).astype(float)
    rows = np.repeat(np.arange(nst), 3)
    cols = np.stack([np.zeros(nst, dtype=np.int64), 1 + np.arange(nst), 1 + nst + np.arange(nst)], axis=1).ravel()
    a = sp.csr_matrix((np.ones(3 * nst), (rows, cols)), shape=(nst, n))
    m0, m1, m2 = ar1_components(T)
    z1 = sp.csc_matrix((1, 1))
    zst = sp.csc_matrix((nst, nst))
    ks = [sp.block_diag([z1, sp.kron(mi, r, format="csc"), zst]).tocsc() for mi in (m0, m1, m2)]
    dint = np.zeros(n)
    dint[0] = BESAG_FIXED_PREC
    m_int = sp.diags(dint).tocsc()
    m_iid = sp.diags(np.r_[np.zeros(1 + nst), np.ones(nst)]).tocsc()
    ata = (a.T @ a).tocsc()
    model = build_latent(n, [m_int] + ks + [m_iid], "besag_x_ar1", extra_pattern=[ata],
                         info={"nr": nr, "nc": nc, "T": T})
    cons = group_constraint(ns, T, 1, n)
    truth = {"rho": rho, "tau_b": tau_b, "tau_g": tau_g, "tau_iid": tau_iid, "u": u, "w": w}
    return GroupProblem(model=model, a=a, y=y, ntrials=ntrials, constraint=cons, dims=(ns, T), truth=truth)


def group_coefs(theta):
    """Coefficients of :func:`make_group_problem`'s components and their theta-derivatives
    (rho clamped to +-0.999 as structured.rs:353 does; the derivative is then 0)."""
    tb, tg, tr, ti = (float(v) for v in theta)
    s = np.exp(tb + tg)
    rho_raw = 2.0 / (1.0 + np.exp(-tr)) - 1.0
    rho = float(np.clip(rho_raw, -0.999, 0.999))
    drho = (1.0 - rho_raw * rho_raw) / 2.0 if rho == rho_raw else 0.0
    tau_iid = np.exp(ti)
    c = np.array([1.0, s, s * rho * rho, -s * rho, tau_iid])
    dc = np.zeros((4, 5))
    dc[0, 1:4] = c[1:4]
    dc[1, 1:4] = c[1:4]
    dc[2, 2] = s * 2.0 * rho * drho
    dc[2, 3] = -s * drho
    dc[3, 4] = tau_iid
    return c, dc


@dataclass
class MultiProblem:
    models: list          # LatentModel per model: [intercept, AR1 (n_k), iid (n_k)]
    a: list               # projectors [1 | I | I] (n_k x (2 n_k + 1))
    y: list
    truth: dict


def ar1_iid_model(nk: int) -> tuple:
    """Latent [intercept, AR1 (nk), iid (nk)] with components [M_int, K0, K1, K2, M_iid]
    (AR1 pieces of ar1_components) and the projector [1 | I | I]."""
    n = 1 + 2 * nk
    m0, m1, m2 = ar1_components(nk)
    z1, zk = sp.csc_matrix((1, 1)), sp.csc_matrix((nk, nk))
    ks = [sp.block_diag([z1, mi, zk]).tocsc() for mi in (m0, m1, m2)]
    d = np.zeros(n)
    d[0] = BESAG_FIXED_PREC
    m_int = sp.diags(d).tocsc()
    m_iid = sp.diags(np.r_[np.zeros(1 + nk), np.ones(nk)]).tocsc()
    rows = np.repeat(np.arange(nk), 3)
    cols = np.stack([np.zeros(nk, dtype=np.int64), 1 + np.arange(nk), 1 + nk + np.arange(nk)], axis=1).ravel()
    a = sp.csr_matrix((np.ones(3 * nk), (rows, cols)), shape=(nk, n))
    model = build_latent(n, [m_int] + ks + [m_iid], "ar1_iid", extra_pattern=[(a.T @ a).tocsc()], info={"nk": nk})
    return model, a


def make_multi_problem(G: int = 512, seed: int = SEED_BASE + 4, n_lo: int = 200, n_hi: int = 5000,
                       tau_iid: float = 10.0, beta0: float = 0.5) -> MultiProblem:
    """Uneven batch of independent Poisson models, each AR1(n_k) + iid(n_k) + intercept with
    n_obs = n_k: n_k = floor(exp(U(ln n_lo, ln n_hi))), rho_k ~ U(0.3, 0.95),
    tau_k ~ LogNormal(0, 0.5). Draw order: all n_k, all rho_k, all tau_k, then per model the
    AR1 path (stationary start), the iid effects and the counts."""
    rng = np.random.default_rng(seed)
    nks = np.floor(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), size=G))).astype(int)
    rhos = rng.uniform(0.3, 0.95, size=G)
    taus = rng.lognormal(0.0, 0.5, size=G)
    models, As, ys = [], [], []
    for nk, rho, tau in zip(nks, rhos, taus):
        model, a = ar1_iid_model(int(nk))
        e = rng.standard_normal(int(nk)) / np.sqrt(tau)
        x = np.empty(int(nk))
        x[0] = e[0] / np.sqrt(1.0 - rho * rho)
        for t in range(1, int(nk)):
            x[t] = rho * x[t - 1] + e[t]
        v = rng.standard_normal(int(nk)) / np.sqrt(tau_iid)
        y = rng.poisson(np.exp(beta0 + x + v)).astype(float)
        models.append(model)
        As.append(a)
        ys.append(y)
    return MultiProblem(models=models, a=As, y=ys,
                        truth={"n": nks, "rho": rhos, "tau": taus, "tau_iid": tau_iid, "beta0": beta0})


def ar1_iid_coefs(theta):
    """theta = [log tau, logit-type rho, log tau_iid] -> coefficients of :func:`ar1_iid_model`'s
    components [M_int, K0, K1, K2, M_iid] and their theta-derivatives (3 x 5); rho =
    2 / (1 + e^-theta) - 1 clamped to +-0.999 as structured.rs:348-356."""
    lt, tr, li = (float(v) for v in theta)
    tau = np.exp(lt)
    rho_raw = 2.0 / (1.0 + np.exp(-tr)) - 1.0
    rho = float(np.clip(rho_raw, -0.999, 0.999))
    drho = (1.0 - rho_raw * rho_raw) / 2.0 if rho == rho_raw else 0.0
    ti = np.exp(li)
    c = np.array([1.0, tau, tau * rho * rho, -tau * rho, ti])
    dc = np.zeros((3, 5))
    dc[0, 1:4] = c[1:4]
    dc[1, 2] = tau * 2.0 * rho * drho
    dc[1, 3] = -tau * drho
    dc[2, 4] = ti
    return c, dc
