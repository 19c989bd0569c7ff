#!/usr/bin/env python
"""Headline benchmark: full INLA fit of the SPDE Matern model on the jittered
200x200 mesh (n = 40 000 latent, 20 000 Gaussian observations, three
hyperparameters, CCD integration with 15 theta-points), FP64.

One step = one full fit (mode search + Hessian + CCD + marginal variances of
every latent node) with the batched + adjoint path: BFGS on exact adjoint
gradients with a batched line search, the reference's FD Hessian stencil in
one batch, the 15 CCD nodes in one batch. The metric is theta-evaluations
per second (full Laplace evaluations at one theta-point per second) and fit
seconds; the plain GPU drop-in (the reference's control flow: Nelder-Mead,
sequential FD Hessian, sequential CCD, one theta-point per evaluation) is
timed in the same run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: each rank fits an independent replica (replicas only, no
collective on the data path); value = all ranks' theta-evaluations / max
rank time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "rust-inla_b200"))

METRIC = "INLA fit s & θ-evals/s, SPDE n≈40k: batched+adjoint vs plain GPU (var ≤1e-8)"
UNIT = "theta-evals/s"
THETA0 = [0.0, 0.0, 0.0]  # reference defaults: family 0.0, spde [log tau, log kappa] = [0, 0]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=200)
    ap.add_argument("--nobs", type=int, default=20000)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain GPU drop-in fit")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-fit", action="store_true",
                    help="reference arm: skip timing the oracle's whole fit (NM + FD Hessian + CCD; minutes)")
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the fits of the grouped 200 001-node model and of the 512 uneven models")
    ap.add_argument("--other-configs-child", action="store_true", help=argparse.SUPPRESS)
    return ap.parse_args()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return ws, rank, local, pg


def combine_over_ranks(dist, ms, evals, device):
    """Whole-job figures of the replicas: the slowest rank's device time and the sum of every
    rank's theta-evaluations. Every rank takes the same two collectives in the same order."""
    if dist is None:
        return float(ms), float(evals)
    import torch

    tmax = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    tsum = torch.tensor([float(evals)], dtype=torch.float64, device=device)
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(tsum[0])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.proc:
            return out
        time.sleep(0.3)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if sm:
            out = {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                   "samples": len(sm)}
        return out


def make_problem(args, standalone: bool = False):
    """The seeded SPDE inputs. ``standalone`` loads the input generator (numpy / scipy only) by
    path, without importing the package that loads the CUDA library: the reference arm runs
    the CPU oracle alone."""
    if standalone:
        import importlib.util

        spec = importlib.util.spec_from_file_location("_bench_models", ROOT / "rust-inla_b200" / "inla_b200" / "models.py")
        models = importlib.util.module_from_spec(spec)
        sys.modules[spec.name] = models  # dataclasses resolve the module by name
        spec.loader.exec_module(models)
    else:
        from inla_b200 import models
    return models.make_spde_problem(nx=args.nx, n_obs=args.nobs)


# ---------------------------------------------------------------------------
# reference arm: the CPU oracle (restatement of the reference's CPU path)
# ---------------------------------------------------------------------------

def cpu_theta_evals(p, seconds: float, threads: int, perm, want_var: bool = False, count: int | None = None):
    """Oracle Laplace evaluations at CCD-like theta-points, `threads` in parallel (the reference
    maps its CCD nodes over Rayon workers, inference.rs:1387-1397). One evaluation = prior LDL^T
    + log-det, posterior LDL^T + log-det + solve (Gaussian closed-form mode) and mlik: the
    evaluation behind every Nelder-Mead step and FD-Hessian point of the reference's fit
    (hyper_opt.rs:21-47). With ``want_var`` it adds the Takahashi diagonal of the posterior
    (sparse_ldlt.rs:376-444), the extra work of a CCD node. Runs rounds of `threads`
    evaluations until `seconds` have passed (at least one round), or exactly `count`
    evaluations. Returns (evals, elapsed seconds)."""
    from concurrent.futures import ThreadPoolExecutor

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.set_supernodal(True)  # the supernodal form with per-pattern analyses, as the reference factorizes
    rng = np.random.default_rng(7)
    base = np.array([4.6, -3.9, 2.65])
    thetas = [base + 0.05 * rng.standard_normal(3) for _ in range(4096)]

    def one(k):
        th = thetas[k % len(thetas)]
        q = p.model.matrix(O.spde_coefs(th[1], th[2]))
        O.laplace(q, p.a, "gaussian", p.y, p1=math.exp(th[0]), perm=perm, want_var=want_var)
        return 1

    done = 0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        if count is not None:
            done = sum(ex.map(one, range(count)))
        else:
            while time.perf_counter() - t0 < seconds or done == 0:
                done += sum(ex.map(one, range(done, done + threads)))
    return done, time.perf_counter() - t0


def other_config_fits():
    """Fit seconds of two other workloads on this GPU, each a first fit (it includes the engine's
    per-batch-size autotuning and graph captures), wall clock between synchronizes:
    * the space x time group model (Besag 50 x 50 (x) AR1 T = 40 + iid + intercept, n = 200 001,
      binomial(10), one sum-to-zero row per time held bordered; CCD over 4 hyperparameters, 25 nodes);
    * 512 independent AR1 + iid + intercept Poisson models of 200 to 5 000 nodes, fitted in lockstep
      (per-model mode search, Hessian and CCD 15).
    Each entry holds its result or its error."""
    import torch

    from inla_b200 import models
    from inla_b200.laplace import PRIOR_PC_COR1, PRIOR_PC_PREC, LaplaceModel
    from inla_b200.multi import MultiModel

    out = {}
    try:
        t0 = time.perf_counter()
        p = models.make_group_problem()
        lm = LaplaceModel(p.model, a=p.a, family="binomial", y=p.y, p1=p.ntrials, max_batch=9)
        lm.set_constraints(*p.constraint)  # auto: bordered at this size
        priors = [(PRIOR_PC_PREC, 0, (1.0, 0.01)), (PRIOR_PC_PREC, 1, (1.0, 0.01)), (PRIOR_PC_COR1, 2, (0.5, 0.75)),
                  (PRIOR_PC_PREC, 3, (1.0, 0.01))]

        def tmap(th):
            c, dc = models.group_coefs(th)
            return c, dc, 1.0, np.zeros(4)

        torch.cuda.synchronize()
        t1 = time.perf_counter()
        r = lm.fit(np.array([0.0, 0.0, 1.5, 1.0]), theta_map=tmap, priors=priors, mode_search="newton", batched=True)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        out["group_200k_ccd25"] = {"fit_s": t2 - t1, "inputs_and_model_s": t1 - t0, "theta_evals": int(r["n_evals"]),
                                   "batches": int(r["n_batches"]), "mode": [float(v) for v in r["mode"]],
                                   "n_latent": int(p.model.n)}
        lm.close()
        del lm, p
    except Exception as e:  # reported, not raised: the main line must still print
        out["group_200k_ccd25"] = {"error": repr(e)[:300]}
    try:
        t0 = time.perf_counter()
        p = models.make_multi_problem()
        mm = MultiModel(p.models, p.a, p.y, family="poisson", max_batch=15)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        r = mm.fit(np.zeros((mm.G, 3)))
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        out["multi_512_ccd15"] = {"fit_s": t2 - t1, "inputs_and_model_s": t1 - t0, "models": int(mm.G),
                                  "batches": int(r["n_batches"]), "model_evals": int(r["n_model_evals"]),
                                  "all_status_ok": bool(np.all(r["status"] == 0))}
    except Exception as e:
        out["multi_512_ccd15"] = {"error": repr(e)[:300]}
    return out


def run_other_configs(timeout_s: float = 300.0):
    """other_config_fits in a child process, so that nothing in it can stop this line."""
    import subprocess

    try:
        r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--other-configs-child"], capture_output=True,
                           text=True, timeout=timeout_s)
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode == 0 and lines:
            return json.loads(lines[-1])
        return {"error": f"rc={r.returncode}: {(r.stderr or r.stdout)[-300:]}"}
    except Exception as e:
        return {"error": repr(e)[:300]}


def cpu_whole_fit(p, threads: int, perm):
    """The reference's whole fit restated by the oracle, wall-clock seconds per stage: Nelder-Mead
    from theta0 (hyper_opt.rs:15-183), one evaluation at a time with the threads inside each
    factorization; the FD Hessian (hyper_opt.rs:188-259, h = max(1e-4, 0.05 |theta|)), likewise; the CCD nodes with the Takahashi variances, mapped over `threads`
    as inference.rs:1387-1397 maps them over Rayon workers; the mixture (inference.rs:1419-1466)."""
    from concurrent.futures import ThreadPoolExecutor

    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    O.set_supernodal(True)
    O.set_threads(threads)  # one evaluation at a time: the threads work inside each factorization
    count = [0]

    def f(th):
        count[0] += 1
        return O.spde_neg_log_posterior(np.asarray(th), p.model, p.a, p.y, perm=perm)

    def node(theta):
        r = O.laplace(p.model.matrix(O.spde_coefs(theta[1], theta[2])), p.a, "gaussian", p.y,
                      p1=math.exp(theta[0]), perm=perm, want_var=True)
        lp = O.loggamma_log_dens(theta[0], 1.0, 5e-5) + O.pc_spde_log_dens(theta[1], theta[2], 1.0, 0.05, 1.0, 0.01)
        return r["x"], r["var"], r["mlik"] + lp

    t0 = time.perf_counter()
    mode = O.nelder_mead(list(THETA0), 0.1, 200, 1e-6, f)
    t1 = time.perf_counter()
    h = max(1e-4, max(0.05 * abs(t) for t in mode))
    hess = O.fd_hessian(mode, f, h)
    t2 = time.perf_counter()
    O.set_threads(1)  # the nodes run side by side, one thread each
    # the CCD nodes as integrate() places them, evaluated in parallel first
    lam, vec = np.linalg.eigh(np.linalg.inv(-np.asarray(hess)))
    z, _ = O.ccd_design(len(mode))
    thetas = [np.asarray(mode) + vec @ (np.sqrt(np.abs(lam)) * np.asarray(zk, dtype=float)) for zk in z]
    with ThreadPoolExecutor(max_workers=threads) as ex:
        done = dict(zip((tuple(t) for t in thetas), ex.map(node, thetas)))
    res = O.integrate(mode, hess, lambda th: done[tuple(th)] if tuple(th) in done else node(th), f0=1.0)
    t3 = time.perf_counter()
    return {"fit_s": t3 - t0, "stages_s": {"mode_search": t1 - t0, "hessian": t2 - t1, "nodes_and_mixture": t3 - t2},
            "theta_evals": count[0] + len(thetas), "mode": [float(v) for v in mode], "mlik": float(res["mlik"]),
            "threads": threads}


def cpu_perm(p):
    """The oracle's restatement of the reference's ordering choice on this pattern
    (ordering.rs:149-162 picks AMD here; the oracle's minimum-degree order stands in for
    faer's AMD). Computed once, outside the timed region."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    return O.reference_perm(p.model.pattern)


CPU_KIND_NOTE = ("CPU oracle: C restatement of rust-inla's path: a supernodal LDL^T (postordered "
                 "elimination tree, relaxed supernodes, dense panels; analysis cached per pattern as "
                 "the reference's pattern cache does) written here, not faer's own code, and the "
                 "reference's Takahashi recurrence")


def bench_config(p, args, ws):
    """The workload both arms run (same keys on both lines)."""
    return {"workload": "spde_200x200_gaussian_ccd15", "n_latent": int(p.model.n), "n_obs": args.nobs,
            "theta_dim": 3, "ccd_points": 15, "theta0": THETA0, "parallelism": f"replicas{ws}",
            "l2": "working set (front buffers, B x 213 MB) larger than L2; no flush needed"}


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    p = make_problem(args, standalone=True)
    threads = os.cpu_count() or 1
    perm = cpu_perm(p)
    per_step = max(args.cpu_seconds / max(args.steps, 1), 1.0)
    for _ in range(args.warmup):
        cpu_theta_evals(p, 0.0, threads, perm)
    ev, el = 0, 0.0
    for _ in range(args.steps):
        e, t = cpu_theta_evals(p, per_step, threads, perm)
        ev += e
        el += t
    value = ev / el
    # the CCD stage of the reference's fit: 15 node evaluations with marginal variances
    nccd, tccd = cpu_theta_evals(p, 0.0, threads, perm, want_var=True, count=15)
    whole = None if args.no_cpu_fit else cpu_whole_fit(p, threads, perm)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded SPDE 200x200 jittered mesh, 20k Gaussian obs)",
            "config": bench_config(p, args, ws),
            "ccd_stage_with_variances_s": tccd,
            **({"cpu_fit": whole} if whole else {}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{ev} oracle Laplace evaluations (prior + posterior LDL^T, solve, mlik: "
                                       f"the Nelder-Mead / FD-Hessian evaluation of the reference's fit) at "
                                       f"CCD-like theta-points, {threads} threads, minimum-degree order; then the 15 "
                                       f"CCD-node evaluations with the Takahashi diagonal in {tccd:.1f}s; "
                                       f"{CPU_KIND_NOTE}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def measured_dgemm_tflops(torch):
    """cuBLAS DGEMM throughput on this GPU (FP64 denominator of the roofline)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, 2 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def factor_roofline(p, torch, B=21, reps=10):
    """Average duration of the batched supernodal LDL^T launch sequence (B theta-points),
    CUDA events on the launching stream; algorithmic FLOPs F = sum_j (c_j^2 + 2 c_j) per problem."""
    import ctypes as C

    from inla_b200 import BatchSolver, GpuSolver, _lib, models
    from inla_b200._lib import check, lib

    c, _ = models.spde_coefs(math.log(0.02), math.log(14.14))
    q = (p.model.matrix(c) + 100.0 * (p.a.T @ p.a)).tocsc()
    q.sort_indices()
    bs = BatchSolver(q, max_batch=B)  # nested dissection, as in the fit
    s = GpuSolver(_lib.ORDER_ND)
    s.analyze(q)
    cc = s.colcounts().astype(np.float64) - 1.0
    flops = float(np.sum(cc * cc + 2 * cc))
    vals = torch.tensor(np.tile(q.data, (B, 1)), device="cuda")
    ld = torch.zeros(B, dtype=torch.float64, device="cuda")
    st = torch.zeros(B, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream

    def fac():
        check(lib().inla_batch_factorize_dev(bs._h, B, C.c_void_p(vals.data_ptr()), C.c_void_p(ld.data_ptr()),
                                             C.c_void_p(st.data_ptr()), C.c_void_p(stream)))

    for _ in range(3):
        fac()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fac()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del bs
    return {"flops_per_launch": flops * B, "ms": ms, "nnz_l": int(s.info()["nnz_l"]), "B": B}


TRAFFIC_SUMMARY = Path(__file__).resolve().parent / "profiles" / "traffic_factor_spde200.md"


def factor_traffic(B):
    """DRAM bytes (read + write) of one batched factorization of B problems, from the committed
    ncu summary (per-problem figure of a smaller capture; batch members use disjoint buffers)."""
    try:
        for line in TRAFFIC_SUMMARY.read_text().splitlines():
            if line.startswith("dram_bytes_per_problem:"):
                return int(line.split(":")[1]) * B, f"{TRAFFIC_SUMMARY.name} (per-problem DRAM bytes x {B})"
    except OSError:
        pass
    return None, "no ncu traffic summary"


def run_ours(args, ws, rank, local, dist):
    import torch

    from inla_b200 import lib as _l  # noqa: F401
    from inla_b200._lib import lib
    from inla_b200.laplace import LaplaceModel

    torch.cuda.set_device(local)
    p = make_problem(args)
    tc = time.perf_counter()
    lm = LaplaceModel(p.model, a=p.a, family="gaussian", y=p.y, max_batch=25)
    create_first_s = time.perf_counter() - tc  # includes the symbolic analysis the later creations reuse
    fit_kw = dict(mode_search="newton", batched=True, tol=1e-4)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        lm.fit(THETA0, **fit_kw)
    barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    launches0 = lib().inla_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    evals = 0
    fits = []
    for _ in range(args.steps):
        r = lm.fit(THETA0, **fit_kw)
        evals += r["n_evals"]
        fits.append(r)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    clocks = sampler.stop()
    launches = lib().inla_kernel_launches() - launches0
    ms_total, evals_all = combine_over_ranks(dist, e0.elapsed_time(e1), evals, "cuda")
    value = evals_all / (ms_total * 1e-3)
    last = fits[-1]

    # e2e through the public API with host buffers: model creation (H2D of the
    # pattern, components, projector and data, device tables; the symbolic analysis
    # of this pattern is the process-wide cached one, computed at the first
    # creation, create_first_s) + fit + D2H of results
    e2e_ms, e2e_evals = 0.0, 0
    nnz = p.model.pattern.nnz
    h2d = 8 * (p.model.comp_values.size + p.y.size + p.a.nnz) + 8 * (p.model.n + 1 + nnz) + 8 * (
        p.a.shape[0] + 1 + p.a.nnz)
    d2h = 8 * (2 * p.model.n + 3 + 9 + 64 * 4 + 6)
    e2e_parts = []  # per step: model creation, fit, release (seconds)
    for _ in range(args.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lm2 = LaplaceModel(p.model, a=p.a, family="gaussian", y=p.y, max_batch=25)
        t1 = time.perf_counter()
        r2 = lm2.fit(THETA0, **fit_kw)
        t2 = time.perf_counter()
        lm2.close()
        t3 = time.perf_counter()
        e2e_ms += (t3 - t0) * 1e3
        e2e_evals += r2["n_evals"]
        e2e_parts.append([round(t1 - t0, 4), round(t2 - t1, 4), round(t3 - t2, 4)])
    e2e_value = e2e_evals / (e2e_ms * 1e-3) if e2e_ms > 0 else None

    if rank != 0:
        return 0

    # the same fit with the forward-difference gradient stencil (m + 1 points per mode-search
    # batch instead of 2m + 1): fewer theta-evaluations, a shorter fit
    fwd = None
    if not args.no_plain:
        kw1 = dict(fit_kw, mode_search="newton1")
        lm.fit(THETA0, **kw1)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        for _ in range(3):
            r1 = lm.fit(THETA0, **kw1)
        f1.record()
        torch.cuda.synchronize()
        fwd = {"fit_s": f0.elapsed_time(f1) * 1e-3 / 3, "theta_evals_per_fit": r1["n_evals"],
               "max_abs_mode_diff": float(np.max(np.abs(r1["mode"] - last["mode"])))}

    # plain GPU drop-in: the reference's control flow, one theta-point per evaluation
    plain = None
    if not args.no_plain:
        t0 = time.perf_counter()
        rp = lm.fit(THETA0, mode_search="nm", batched=False)
        plain_s = time.perf_counter() - t0
        plain = {"fit_s": plain_s, "theta_evals": rp["n_evals"], "theta_evals_per_s": rp["n_evals"] / plain_s,
                 "mode": rp["mode"].tolist(), "mode_iters": rp["mode_iters"],
                 "max_rel_var_diff_vs_batched": float(np.max(np.abs(rp["var"] - last["var"]) / rp["var"])),
                 "max_abs_mean_diff_vs_batched": float(np.max(np.abs(rp["mean"] - last["mean"])))}

    # roofline: the batched supernodal factorization (dominant FP64 contraction)
    peak = measured_dgemm_tflops(torch)
    # the fit's mode-search batches factorize 10 problems (7 posterior theta-points and the 3 prior
    # representatives of their stencil); B = 21 is the larger batch for reference
    fr = factor_roofline(p, torch, B=10)
    fr21 = factor_roofline(p, torch, B=21)
    achieved = fr["flops_per_launch"] / (fr["ms"] * 1e-3) / 1e12
    traffic, tsrc = factor_traffic(fr["B"])
    roof = {"bound": "tensor",
            "kernel": "batched supernodal LDL^T at the fit's batch size (B=10 theta-points, nested dissection; "
                      "the schedule the engine picks for that size)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64; the measured-peaks file has no FP64 entry)",
            "traffic": traffic, "traffic_source": tsrc, "ms_per_launch": fr["ms"],
            "flops_per_launch": fr["flops_per_launch"],
            "b21": {"ms_per_launch": fr21["ms"], "achieved": fr21["flops_per_launch"] / (fr21["ms"] * 1e-3) / 1e12,
                    "frac": fr21["flops_per_launch"] / (fr21["ms"] * 1e-3) / 1e12 / peak}}

    cpu = None
    if ws == 1 and args.cpu_seconds > 0:
        threads = os.cpu_count() or 1
        perm = cpu_perm(p)
        cpu_theta_evals(p, 0.0, threads, perm, count=1)  # untimed: the per-pattern analyses
        ev, el = cpu_theta_evals(p, args.cpu_seconds, threads, perm)
        cpu = {"value": ev / el, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{ev} oracle Laplace evaluations (prior + posterior LDL^T, solve, mlik: the "
                         f"Nelder-Mead / FD-Hessian evaluation of the reference's fit) at CCD-like theta-points "
                         f"in {el:.1f}s, {threads} threads, minimum-degree order; {CPU_KIND_NOTE}"}

    others = None
    if ws == 1 and not args.no_other_configs:
        # the child's models need the device memory this process still holds: free the benchmark
        # model and hand the library's and torch's cached blocks back to the driver first
        lm.close()
        lib().inla_release_cached_memory()
        torch.cuda.empty_cache()
        others = run_other_configs()

    fit_s = ms_total * 1e-3 / args.steps
    # where one fit's time goes (host wall clock per phase, averaged over the timed fits)
    phases = {k: sum(f["phase_s"][k] for f in fits) / len(fits) for k in fits[0]["phase_s"]}
    phases["host_between_phases"] = sum(f["seconds"] for f in fits) / len(fits) - sum(phases.values())
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded SPDE 200x200 jittered mesh, 20k Gaussian obs; inputs resident in HBM)",
            "config": bench_config(p, args, ws),
            "method": "batched Newton on adjoint gradients (FD-of-gradient Hessian), full step first with "
                      "half / quarter steps on failure; FD Hessian and CCD nodes in one batch each",
            "fit_s": fit_s, "fit_breakdown_s": phases, "theta_evals_per_fit": evals / args.steps,
            "mode": last["mode"].tolist(),
            "plain_gpu": plain,
            "speedup_vs_plain_gpu": (plain["fit_s"] / fit_s) if plain else None,
            "forward_stencil_fit": fwd,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "fit_s": e2e_ms * 1e-3 / max(args.e2e_steps, 1), "create_fit_close_s": e2e_parts,
                    "create_first_s": round(create_first_s, 4),
                    "note": "model creation inside every e2e step; the symbolic analysis of the pattern and the "
                            "engine tables derived from it are the process-wide cached ones from the first creation "
                            "(create_first_s includes them); the first e2e step also maps fresh device memory, "
                            "because the timed model still holds its own"},
            "gpu_launches": int(launches), "clocks": clocks, "roofline": roof, "cpu_baseline": cpu,
            "other_configs": others}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.other_configs_child:
        print(json.dumps(other_config_fits()), flush=True)
        return 0
    ws, rank, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            return run_reference(args, ws, rank)
        return run_ours(args, ws, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
