"""The replicas-only multi-rank path of bench.py on CPU: two gloo ranks (no GPU), the
max-over-ranks time and the summed evaluations, and the reference arm's rank-0-only rule."""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        ms = [12.5, 30.0][rank]
        evals = [100, 157][rank]
        out.put((rank, bench.combine_over_ranks(dist, ms, evals, "cpu")))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_max_time_and_summed_evaluations():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got[0] == got[1] == (30.0, 257.0)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.combine_over_ranks(None, 7.0, 21, "cpu") == (7.0, 21.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    class Args:
        gpus, steps, warmup, cpu_seconds, nx, nobs = 2, 1, 0, 0.1, 10, 50

    assert bench.run_reference(Args(), 2, 1) == 0
    assert capsys.readouterr().out == ""


def test_dist_setup_without_torchrun_is_single_rank(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_setup(None) == (1, 0, 0, None)


def test_reference_arm_whole_fit_on_a_small_mesh():
    """The whole-fit timing of the reference arm (Nelder-Mead, FD Hessian, CCD nodes over
    threads) runs on a 15 x 15 mesh and lands on the oracle's own Nelder-Mead mode."""
    import types

    import numpy as np

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import bench
    import oracle as O

    p = bench.make_problem(types.SimpleNamespace(nx=15, nobs=120), standalone=True)
    perm = bench.cpu_perm(p)
    try:
        r = bench.cpu_whole_fit(p, 2, perm)
    finally:
        O.set_supernodal(False)  # the oracle's default, the form the parity tests pin
    mode_ref = O.nelder_mead(list(bench.THETA0), 0.1, 200, 1e-6,
                             lambda th: O.spde_neg_log_posterior(np.asarray(th), p.model, p.a, p.y, perm=perm))
    np.testing.assert_allclose(r["mode"], mode_ref, atol=1e-6)
    assert r["theta_evals"] > 15 and np.isfinite(r["mlik"]) and r["fit_s"] > 0


def test_other_config_fits_run_in_a_child_and_report_errors():
    """The extra fits run in a child process whose failure cannot stop the bench line: without a
    GPU both legs come back as errors in a JSON object."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("device present")
    sys.path.insert(0, str(ROOT))
    import bench

    r = bench.run_other_configs(timeout_s=300)
    assert set(r) == {"group_200k_ccd25", "multi_512_ccd15"}, r
    assert all("error" in v for v in r.values())


def test_reference_arm_line_on_a_tiny_mesh(capsys):
    """The whole reference arm on rank 0 (10 x 10 mesh): one JSON line with the GPU arm's config
    keys, the CPU-baseline description and the whole-fit timing."""
    import json

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import bench
    import oracle as O

    class Args:
        gpus, steps, warmup, cpu_seconds, nx, nobs, no_cpu_fit = 1, 1, 0, 0.1, 10, 50, False

    try:
        assert bench.run_reference(Args(), 1, 0) == 0
    finally:
        O.set_supernodal(False)
        O.set_threads(1)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["workload"] == "spde_200x200_gaussian_ccd15"
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_fit"]["theta_evals"] > 15
