"""Known-answer matrices restated from the reference's own unit tests.

* ``ar1_q(n, rho, tau)`` — crates/inla_math/src/sparse_ldlt.rs:573-588
* ``besag_ridge_q(adj, tau, ridge)`` — sparse_ldlt.rs:590-604
* ``besag_4cycle_chord`` / ``path6`` graphs — sparse_ldlt.rs:647-664
* ``mixture_major_fgn_like(64, 5)`` — sparse_ldlt.rs:527-548
* ``mixture_major_path_cliques(64, 5)`` — crates/inla_math/src/ordering.rs:169-189
* ``tridiagonal8`` — crates/inla_math/src/ldlt.rs:522-530
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _sym(n, trips):
    r = [t[0] for t in trips]
    c = [t[1] for t in trips]
    v = [t[2] for t in trips]
    m = sp.coo_matrix((v, (r, c)), shape=(n, n)).tocsc()
    m.sum_duplicates()
    m.sort_indices()
    return m


def ar1_q(n, rho, tau):
    trips = []
    for i in range(n):
        d = tau if (i == 0 or i == n - 1) else tau * (1.0 + rho * rho)
        trips.append((i, i, d))
        if i + 1 < n:
            trips.append((i, i + 1, -tau * rho))
            trips.append((i + 1, i, -tau * rho))
    return _sym(n, trips)


def besag_ridge_q(adj, tau, ridge):
    n = len(adj)
    trips = []
    for i in range(n):
        trips.append((i, i, tau * len(adj[i]) + ridge))
        for j in adj[i]:
            if j > i:
                trips.append((i, j, -tau))
                trips.append((j, i, -tau))
    return _sym(n, trips)


BESAG_4CYCLE_CHORD = [[1, 3], [0, 2, 3], [1, 3], [0, 1, 2]]
PATH6 = [[j for j in (i - 1, i + 1) if 0 <= j < 6] for i in range(6)]


def mixture_major_fgn_like(n_time, n_comp):
    n = n_time * n_comp
    trips = []
    for t in range(n_time):
        for c in range(n_comp):
            i = c * n_time + t
            trips.append((i, i, 6.0))
            for d in range(c + 1, n_comp):
                j = d * n_time + t
                trips += [(i, j, -0.4), (j, i, -0.4)]
            if t + 1 < n_time and c > 0:
                i2 = c * n_time + t + 1
                trips += [(i, i2, -1.2), (i2, i, -1.2)]
    return _sym(n, trips)


def mixture_major_path_cliques(n_time, n_comp):
    n = n_time * n_comp
    trips = []
    for t in range(n_time):
        for c in range(n_comp):
            i = c * n_time + t
            trips.append((i, i, 4.0))
            for d in range(c + 1, n_comp):
                j = d * n_time + t
                trips += [(i, j, -0.3), (j, i, -0.3)]
            if t + 1 < n_time and c > 0:
                i2 = c * n_time + t + 1
                trips += [(i, i2, -1.0), (i2, i, -1.0)]
    return _sym(n, trips)


def tridiagonal8():
    n = 8
    trips = []
    for i in range(n):
        trips.append((i, i, 2.5))
        if i + 1 < n:
            trips += [(i + 1, i, -0.7), (i, i + 1, -0.7)]
    return _sym(n, trips)


def identity(n, v):
    return sp.identity(n, format="csc") * v


def random_spd(n, density, seed):
    """Random sparse SPD matrix (diagonally dominant), full symmetric CSC."""
    rng = np.random.default_rng(seed)
    a = sp.random(n, n, density=density, random_state=rng, format="csc")
    a = a + a.T
    a.data = -np.abs(a.data)
    d = np.asarray(abs(a).sum(axis=1)).ravel() + 1.0 + rng.uniform(0, 1, n)
    q = (a + sp.diags(d)).tocsc()
    q.sum_duplicates()
    q.sort_indices()
    return q


def grid_laplacian(nr, nc, ridge=0.5, tau=1.0):
    """Besag lattice Laplacian (rook) plus a ridge."""
    idx = np.arange(nr * nc).reshape(nr, nc)
    adj = [[] for _ in range(nr * nc)]
    for r in range(nr):
        for c in range(nc):
            i = idx[r, c]
            if c + 1 < nc:
                adj[i].append(idx[r, c + 1]); adj[idx[r, c + 1]].append(i)
            if r + 1 < nr:
                adj[i].append(idx[r + 1, c]); adj[idx[r + 1, c]].append(i)
    return besag_ridge_q(adj, tau, ridge)


KNOWN_ANSWER = {
    "ar1_12": (lambda: ar1_q(12, 0.7, 2.5), 1e-9),
    "ar1_3": (lambda: ar1_q(3, 0.2, 1.0), 1e-10),
    "besag_4cycle_chord": (lambda: besag_ridge_q(BESAG_4CYCLE_CHORD, 1.5, 0.25), 1e-9),
    "besag_path6": (lambda: besag_ridge_q(PATH6, 1.0, 0.1), 1e-9),
    "tridiagonal8": (tridiagonal8, 1e-9),
    "identity3x2": (lambda: identity(3, 2.0), 1e-10),
}
