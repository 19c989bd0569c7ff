"""The process-wide cache of symbolic analyses (host code, no GPU): analyses answered from the
cache equal fresh ones, through the public C ABI, and a different permutation or pattern is never
answered by another pattern's entry."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

from inla_b200 import GpuSolver, models
from inla_b200._lib import ORDER_AMD, ORDER_ND

ROOT = Path(__file__).resolve().parent.parent

SCRIPT = r"""
import json, sys
sys.path[:0] = [sys.argv[1] + '/rust-inla_b200']
from inla_b200 import GpuSolver, models
q = models.make_spde_problem(nx=40, n_obs=500).model.pattern
out = {}
for order in (%d, %d):
    s = GpuSolver(ordering=order)
    s.analyze(q)
    out[order] = [s.perm().tolist(), s.etree().tolist(), s.supernodes().tolist(), s.colcounts().tolist(),
                  {k: int(v) for k, v in s.info().items()}]
print(json.dumps(out))
""" % (ORDER_ND, ORDER_AMD)


def _summary(s):
    return [s.perm().tolist(), s.etree().tolist(), s.supernodes().tolist(), s.colcounts().tolist(),
            {k: int(v) for k, v in s.info().items()}]


def test_cached_analyses_equal_fresh_ones():
    q = models.make_spde_problem(nx=40, n_obs=500).model.pattern
    here = {}
    for order in (ORDER_ND, ORDER_AMD):
        first = GpuSolver(ordering=order)
        first.analyze(q)
        again = GpuSolver(ordering=order)
        again.analyze(q)                      # answered from the cache
        assert _summary(first) == _summary(again)
        here[str(order)] = _summary(again)
    env = dict(os.environ, INLA_NO_SYMBOLIC_CACHE="1")
    r = subprocess.run([sys.executable, "-c", SCRIPT, str(ROOT)], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    fresh = json.loads(r.stdout.strip().splitlines()[-1])
    assert fresh == here


def test_custom_permutations_are_not_confused():
    q = models.make_spde_problem(nx=20, n_obs=100).model.pattern
    n = q.shape[0]
    rng = np.random.default_rng(2)
    p1, p2 = np.arange(n), rng.permutation(n)
    res = []
    for p in (p1, p2, p1, p2):
        s = GpuSolver()
        s.set_perm(p)
        s.analyze(q)
        res.append(_summary(s))
    assert res[0] == res[2] and res[1] == res[3] and res[0] != res[1]
