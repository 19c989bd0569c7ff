"""Generate ``golden.npz``: dense numpy answers for the known-answer fixtures.

The reference (Rust + faer) cannot be built in this environment, so the
golden vectors for the reference's own known-answer matrices
(tests/fixtures.py) are computed here with dense LAPACK through numpy:
``log|Q|``, ``Q^{-1} b`` for ``b = 1..n`` and ``diag(Q^{-1})``. Run:

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

from fixtures import KNOWN_ANSWER, grid_laplacian, random_spd  # noqa: E402


def cases():
    for name, (mk, _tol) in KNOWN_ANSWER.items():
        yield name, mk()
    yield "grid_7x9", grid_laplacian(7, 9, ridge=0.3, tau=1.7)
    yield "random_spd_40", random_spd(40, 0.08, 20261203)


def main():
    out = {}
    for name, q in cases():
        d = q.toarray()
        n = d.shape[0]
        sign, logdet = np.linalg.slogdet(d)
        assert sign > 0
        b = np.arange(1, n + 1, dtype=np.float64)
        inv = np.linalg.inv(d)
        out[f"{name}/logdet"] = np.array([logdet])
        out[f"{name}/solve"] = np.linalg.solve(d, b)
        out[f"{name}/diag_inv"] = np.diag(inv).copy()
        out[f"{name}/indptr"] = q.indptr.astype(np.int64)
        out[f"{name}/indices"] = q.indices.astype(np.int64)
        out[f"{name}/data"] = q.data.astype(np.float64)
    np.savez_compressed(HERE / "golden.npz", **out)
    print(f"wrote {HERE / 'golden.npz'} with {len(out)} arrays")


if __name__ == "__main__":
    main()
