"""Workload driver for profiling the hot-path kernels (run under ncu).

    python -m inla_b200.profile_ops --nx 200 --batch 15 --op factor|solve|selinv|all [--reps R]
    python -m inla_b200.profile_ops --nx 200 --batch 21 --op laplace-grad [--ordering amd|nd]
    python -m inla_b200.profile_ops --nx 600 --op mesh --npts 100000 [--reps R]

``factor``/``solve``/``selinv`` run the batched supernodal kernels on the SPDE
posterior precision ``Q(theta) + 100 A^T A`` (theta at the generating values);
``laplace-grad`` runs one batched Laplace evaluation with the adjoint trace
pieces (what one Newton iteration of the batched fit launches); ``mesh`` times the
host and device forms of the mesh tools (FEM blocks, SPDE components, projector) on
a jittered nx x nx mesh. Timings printed here are CUDA-event times on the launching
stream, except the device projector (it synchronizes: wall clock) and the host forms.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))


def main():
    import torch

    from inla_b200 import BatchSolver, models
    from inla_b200._lib import check, lib
    from inla_b200.laplace import LaplaceModel

    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=200)
    ap.add_argument("--batch", type=int, default=15)
    ap.add_argument("--op", default="all")
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--ordering", default="amd", choices=["amd", "nd"])
    ap.add_argument("--stencil", action="store_true",
                    help="laplace-grad batch shaped like one batched-Newton iteration: 3 candidates x "
                         "(centre, +-h per coordinate), so stencil points share prior factorizations")
    ap.add_argument("--panel-form", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="panel form of the level launches: -1 autotuned, 0 split, 1 fused, 2 look-ahead")
    ap.add_argument("--npts", type=int, default=20_000, help="observation points of the mesh op")
    a = ap.parse_args()
    from inla_b200 import _lib
    order = {"amd": _lib.ORDER_AMD, "nd": _lib.ORDER_ND}[a.ordering]
    if a.op == "mesh":
        print(json.dumps(time_mesh(a.nx, a.npts, max(a.reps, 1))), flush=True)
        return
    p = models.make_spde_problem(nx=a.nx, n_obs=a.nx * a.nx // 2)
    B = a.batch
    stream = torch.cuda.current_stream().cuda_stream

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / a.reps

    out = {"nx": a.nx, "B": B, "ordering": a.ordering}
    if a.op in ("factor", "solve", "selinv", "all"):
        c, _ = models.spde_coefs(math.log(0.02), math.log(14.14))
        q = (p.model.matrix(c) + 100.0 * (p.a.T @ p.a)).tocsc()
        q.sort_indices()
        check(lib().inla_set_panel_form(a.panel_form))
        bs = BatchSolver(q, max_batch=B, ordering=order)
        vals = torch.tensor(np.tile(q.data, (B, 1)), device="cuda")
        ld = torch.zeros(B, dtype=torch.float64, device="cuda")
        st = torch.zeros(B, dtype=torch.int32, device="cuda")
        x = torch.ones(B, q.shape[0], dtype=torch.float64, device="cuda")
        dg = torch.zeros_like(x)

        def fac():
            check(lib().inla_batch_factorize_dev(bs._h, B, C.c_void_p(vals.data_ptr()), C.c_void_p(ld.data_ptr()),
                                                 C.c_void_p(st.data_ptr()), C.c_void_p(stream)))

        def sol():
            check(lib().inla_batch_solve_dev(bs._h, B, C.c_void_p(x.data_ptr()), C.c_void_p(stream)))

        def sel():
            check(lib().inla_batch_diag_inv_dev(bs._h, B, C.c_void_p(dg.data_ptr()), C.c_void_p(stream)))

        fac()
        for name, fn in (("factor", fac), ("solve", sol), ("selinv", sel)):
            if a.op in (name, "all"):
                out[name + "_ms"] = timed(fn)
        del bs
    if a.op == "laplace-grad":
        lm = LaplaceModel(p.model, a=p.a, family="gaussian", y=p.y, max_batch=B, ordering=order)
        if a.stencil:
            base = np.array([4.6, -3.9, 2.6])
            pts = []
            for cnd in range(3):
                c0 = base + 0.1 * cnd
                pts.append(c0)
                for kk in range(3):
                    for sgn in (1, -1):
                        e = np.zeros(3)
                        e[kk] = sgn * 1e-3
                        pts.append(c0 + e)
            th = np.array(pts[:B])
        else:
            th = np.array([4.6, -3.9, 2.6]) + 0.01 * np.random.default_rng(0).standard_normal((B, 3))
        coefs = np.stack([models.spde_coefs(t[1], t[2])[0] for t in th])
        scale = np.exp(th[:, 0])
        out["laplace_grad_ms"] = timed(lambda: lm.eval(coefs, scale, gradient=True, mode=False))
    print(json.dumps(out), flush=True)


def time_mesh(nx, npts, reps):
    """Host forms against device forms of the mesh tools, milliseconds (device: after the first
    call, which builds the contribution lists and copies the mesh; best of ``reps``)."""
    import time

    import torch

    from inla_b200 import models
    from inla_b200.mesh import Mesh, SpdePlan, spde_components

    v, t = models.grid_mesh(nx, np.random.default_rng(13))
    m = Mesh(v, t)
    pts = np.random.default_rng(14).uniform(0.0, 1.0, size=(npts, 2))
    dpts = torch.tensor(pts, device="cuda")

    def wall(fn):
        t0 = time.perf_counter()
        r = fn()
        return r, 1e3 * (time.perf_counter() - t0)

    f, host_fem = wall(m.fem)
    _, host_spde = wall(lambda: spde_components(f["c0"].diagonal(), f["g1"]))
    _, host_proj = wall(lambda: m.projector(pts))
    d, first = wall(m.fem_device)
    cp, ri = m.fem_pattern("g1")
    plan = SpdePlan(len(v), cp, ri)
    plan.components(d["c0"], d["g1"])
    m.projector_device(dpts)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    dev_fem = dev_spde = dev_proj = float("inf")
    for _ in range(reps):
        ev[0].record()
        m.fem_device()
        ev[1].record()
        plan.components(d["c0"], d["g1"])
        ev[2].record()
        torch.cuda.synchronize()
        dev_fem = min(dev_fem, ev[0].elapsed_time(ev[1]))
        dev_spde = min(dev_spde, ev[1].elapsed_time(ev[2]))
        dev_proj = min(dev_proj, wall(lambda: m.projector_device(dpts))[1])
    return {"nx": nx, "triangles": len(t), "points": npts, "host_fem_ms": host_fem, "host_spde_ms": host_spde,
            "host_projector_ms": host_proj, "device_first_call_ms": first, "device_fem_ms": dev_fem,
            "device_spde_ms": dev_spde, "device_projector_ms": dev_proj}


if __name__ == "__main__":
    main()
