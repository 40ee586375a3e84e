"""Benchmark of the time-step hot path (one JSON line on rank 0).

Workload (N=1): flow past a fixed sphere at Re=300 -- domain 4x2x2, 4x2x2
level-0 blocks of 8^3 cells, levelMax 4 (mesh frozen after refinement around
the sphere and its wake: 2340 blocks, 1.198M cells), sphere radius 0.0625 at
(1,1,1) moving at +0.1 in x with the frame following it (uinf = -0.1),
nu = 0.1*0.125/300, WENO5, implicit penalization lambda=1e6, FP64 BiCGSTAB
with the two-level preconditioner (block-constant coarse space + exact
block inverse; --solver b200: the block inverse alone), reference
tolerances (-poissonTol 1e-6, -poissonTolRel 1e-4).  A "step" is one full
time step: calcMaxTimestep, AdvectionDiffusion (3 RK stages), Penalization,
PressureProjection (RHS, Poisson solve, mean removal, gradient update).
The timed steps follow the warm-up steps and --settle (50) more.

`value`  Mcell-steps/s with the fields resident in HBM (device time, CUDA
         events on the context's stream), L2 flushed between timed steps.
`e2e`    the same through the reference-facing C ABI with host buffers:
         per step velocity + pressure uploaded from pinned host memory, the
         step, velocity + pressure downloaded.
`poisson_to_tolerance`  one solve of the seeded right-hand side to 1e-6 and
         1e-10 (FP64 true residual) per solver; the learned network trained
         in the run on the flow's own pressure right-hand sides.
`learned_re1000`  the network trained above, inside every solver on the
         sphere at Re=1000, levelMax 5 (5000 blocks): one pressure
         right-hand side of that flow solved to 1e-6.
`swarm_batch`  64 independent penalized-ellipsoid cases (372-2659 blocks
         each, 37.5M cells) advanced together by cup_batch_step: 200 steps
         with the two-level solver and the bodies moving, 5 with the block
         inverse alone (FP64, and mixed precision) and the bodies held in
         place; step 0 also taken case by case for comparison.
`mesh_adaptation`  from the settled state, three rounds of one adaptation
         (vorticity tagging, refine/compress, field transfer), the two-level
         coarse space of the new mesh, and 20 steps on it (the reference
         adapts every 20 steps); timed apart from the steps, as the metric
         leaves adaptation out.
`--impl reference`  the reference's CPU path restated (oracle: upwind/WENO,
         penalization, projection with the pipelined BiCGSTAB + block CG of
         PoissonSolverAMR.cpp) on the host cores, one step per sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from cup3d_b200.workloads import (SPHERE_BODY, SPHERE_FLAGS, SPHERE_MESH, SPHERE_WORKLOAD as WORKLOAD,  # noqa: E402
                                  make_sphere_ctx, poisson_rhs)

# Algorithmic bytes per cell per launch (each array read once and written once,
# halos excluded, 8-byte reals).
ALG_BYTES = {
    "advect_stage_weno5": 8 * 10,       # mean over stages of 9S/12S/9S (R u, tmpV; W u, tmpV)
    "advect_stage_upwind5": 8 * 10,
    "pressure_rhs": 8 * 7,              # R u(3), chi, p_old; W lhs, phi
    "grad_update": 8 * 9,               # R phi, p_old, u(3); W u(3), p_new
    "bicg_a_pupdate_precond": 8 * 5,    # R r, p, nu; W p, z1
    "bicg_b_spmv_dot": 8 * 3,           # R z1, rhat; W nu
    "bicg_c_supdate_precond": 8 * 4,    # R r, nu; W r, z2
    "bicg_d_spmv_dots": 8 * 3,          # R z2, r; W t
    "bicg_e_xr_update_dots": 8 * 8,     # R x, z1, z2, r, t, rhat; W x, r
    "bicg_init": 8 * 6,
    "bicg_persistent": 8 * 22,          # per iteration: R/W of the three phases (40+40+96 B)
    "weighted_sum": 8 * 1,
    "max_u": 8 * 3,
}


# DRAM bytes (read + write) per cell and iteration of the persistent solver,
# measured by ncu (--set full) on 16 iterations of one solve on the sphere
# mesh (1,198,080 cells), per solver:
#   b200 (`python -m cup3d_b200.kernel_cases solve`): 147.7 MB + 594.2 MB,
#     most of the 176 algorithmic bytes hit in L2;
#   b200_twolevel (`... solve b200_twolevel`): 724.2 MB + 844.7 MB, the two
#     reads of the 21.9 MB A_c^-1 an iteration most of the growth.
MEASURED_TRAFFIC_PER_CELL_ITER = {("bicg_persistent", "b200"): 38.70, ("bicg_persistent", "b200_twolevel"): 81.8}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 100 ms by one
    `nvidia-smi -lms` process running across the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)  # first sample before the timed region starts

    def stop(self):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 7:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[0]) for r in rows) if v is not None]
        mx = [v for v in (num(r[1]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def train_learned(ctx, rhs_list, iters=(0, 1, 2, 3, 5, 8, 12), steps=600, batch=128, lr=1e-3):
    """Trains the block CNN on the residuals of plain solves of the flow's own
    pressure right-hand sides (rhs_list, collected during the run; the last one
    is held out), at the iterates `iters`.  The target of each block sample
    is the one-cell-overlap local solve's correction of its residual."""
    import torch
    level, index, _ = ctx.blocks()
    mb = int(np.where((index == 0).all(axis=1))[0][0])
    ctx.cnn_init(7)
    ctx.cnn_dataset_reserve(ctx.nb * len(rhs_list) * len(iters))
    for bh in rhs_list:
        b = torch.tensor(bh, device="cuda")
        for k in iters:
            xk = torch.zeros_like(b)
            if k > 0:
                ctx.set_poisson("b200", 0.0, 1e-30, k)
                ctx.poisson_solve_dev(b, xk)
            ax = torch.zeros_like(b)
            ctx.poisson_apply(xk, ax)
            r = b - ax
            r[mb * 512] = -ax[mb * 512]  # the mean-constraint row's right-hand side is zero
            ctx.cnn_dataset_add(r.contiguous())
    ctx.cnn_holdout(ctx.nb * len(iters))
    before = ctx.cnn_eval()
    losses = ctx.cnn_train(steps, batch, lr, 11)
    return {"pairs": f"residuals of plain BiCGSTAB iterates {list(iters)} on {len(rhs_list)} pressure right-hand "
                     f"sides of the sphere flow (the last held out)",
            "samples": ctx.cnn_dataset_size(), "steps": steps, "batch": batch, "lr": lr,
            "loss_first10": float(np.mean(losses[:10])), "loss_last10": float(np.mean(losses[-10:])),
            "held_out_rel_loss": [round(float(before), 4), round(float(ctx.cnn_eval()), 4)]}


SOLVERS = ("b200", "b200_mixed", "b200_twolevel", "b200_twolevel_mixed", "b200_schwarz", "b200_learned",
           "b200_learned_mixed")


def poisson_at_tolerance(ctx, stream, flush, rhs_list, reps=3):
    """Device time of one Poisson solve to a relative residual (FP64-checked
    true residual) for every solver, on the seeded right-hand side."""
    import torch
    b = torch.tensor(poisson_rhs(ctx), device="cuda")
    t0 = time.perf_counter()
    training = train_learned(ctx, rhs_list)
    torch.cuda.synchronize()
    training["seconds"] = round(time.perf_counter() - t0, 2)
    res = {"rhs": "PCG64(20261203) white noise + 8 Gaussian sources, h^3-weighted zero mean; x0 = 0",
           "training": training}
    for tol in (1e-6, 1e-10):
        for solver in SOLVERS:
            runs = []
            for _ in range(reps):
                x = torch.zeros_like(b)
                ctx.set_poisson(solver, 0.0, tol, 1000)
                with torch.cuda.stream(stream):
                    flush.fill_(1.0)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                rc, st = ctx.poisson_solve_dev(b, x)
                e1.record(stream)
                e1.synchronize()
                runs.append((e0.elapsed_time(e1), rc, st))
            runs.sort(key=lambda t: t[0])
            ms, rc, st = runs[len(runs) // 2]
            res[f"{solver}@{tol:g}"] = {"ms": round(ms, 3), "iterations": st["iterations"],
                                        "true_rel": float(f"{st['true_rel']:.3e}"), "fallback": st["fallback"],
                                        "status": st["status"], "rc": rc}
    base = res["b200@1e-06"]["ms"]
    res["speedup_vs_b200@1e-06"] = {k.split("@")[0]: round(base / v["ms"], 3)
                                    for k, v in res.items() if k.endswith("@1e-06")}
    ctx.set_poisson(ctx.solver_name, 1e-6, 1e-4, 1000)
    return res


def learned_re1000(src, flush, settle=30, reps=3):
    """The learned preconditioner's evaluation case: the network trained on
    the Re=300 flow (src's weights) inside the solvers of the sphere at
    Re=1000, levelMax 5 (5000 blocks, 2.56M cells).  That flow is stepped
    `settle` steps from rest with the two-level solver; its last pressure
    right-hand side is solved from zero to 1e-6 (FP64 true residual) by
    every solver, device time, L2 flushed before each solve."""
    import torch
    import cup3d_b200 as cup
    from cup3d_b200.workloads import SPHERE_RE1000_WORKLOAD, make_sphere_re1000_ctx
    ctx = make_sphere_re1000_ctx(torch.cuda.current_device(), "b200_twolevel")
    st_ = torch.cuda.ExternalStream(cup._lib.lib().cup_stream(ctx._p))
    its = []
    for k in range(settle):
        _, _, st = ctx.step(k)
        its.append(st["iterations"])
    level, index, _ = ctx.blocks()
    mb = int(np.where((index == 0).all(axis=1))[0][0])
    b = torch.tensor(ctx.download("lhs"), device="cuda")
    b[mb * 512] = 0.0  # the mean-constraint row
    ctx.cnn_init(7)
    ctx.cnn_set_params(src.cnn_get_params())
    res = {"workload": SPHERE_RE1000_WORKLOAD, "blocks": ctx.nb, "cells": ctx.nb * 512,
           "rhs": f"the pressure right-hand side of step {settle - 1} of the Re=1000 flow from rest; x0 = 0",
           "network": "trained on the Re=300 levelMax 4 flow (poisson_to_tolerance.training), not retrained",
           "settle_poisson_iterations": its[-5:]}
    for solver in SOLVERS:
        runs = []
        for _ in range(reps):
            x = torch.zeros_like(b)
            ctx.set_poisson(solver, 0.0, 1e-6, 1000)
            with torch.cuda.stream(st_):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st_)
            rc, st = ctx.poisson_solve_dev(b, x)
            e1.record(st_)
            e1.synchronize()
            runs.append((e0.elapsed_time(e1), rc, st))
        runs.sort(key=lambda t: t[0])
        ms, rc, st = runs[len(runs) // 2]
        res[f"{solver}@1e-06"] = {"ms": round(ms, 3), "iterations": st["iterations"],
                                  "true_rel": float(f"{st['true_rel']:.3e}"), "fallback": st["fallback"],
                                  "status": st["status"], "rc": rc}
    base = res["b200@1e-06"]["ms"]
    res["speedup_vs_b200@1e-06"] = {k.split("@")[0]: round(base / v["ms"], 3)
                                    for k, v in res.items() if k.endswith("@1e-06")}
    ctx.close()
    return res


def swarm_batch(flush, steps=5, solver="b200", moving=False):
    """The 64-case ellipsoid swarm advanced as one batch (cup_batch_step: one
    set of launches and one Poisson launch per step for all cases), against
    the same cases stepped one by one; device time from CUDA events on the
    stepping streams, L2 flushed before every timed step.  Kernel by kernel
    (-stepGraph 0) on both sides, so that no step pays a graph capture.
    solver: the Poisson solver of every case (b200_twolevel: each case's own
    coarse space, built when the batch is created, timed apart).  moving:
    every body moves with its velocity (each step advances the cases' poses
    and creates their chi again inside the timed step), else the bodies are
    held in place (-StaticObstacles 1)."""
    import torch
    import cup3d_b200 as cup
    from cup3d_b200.workloads import SWARM_WORKLOAD, make_swarm_ctx
    lib = cup._lib.lib()
    extra = f"-stepGraph 0 -poissonSolver {solver}" + (" -StaticObstacles 0" if moving else "")
    ctxs = [make_swarm_ctx(i, torch.cuda.current_device(), extra) for i in range(64)]
    t0 = time.perf_counter()
    batch = cup.Batch(ctxs)
    setup_s = time.perf_counter() - t0
    ncell = batch.nb * 512

    def timed(ctx, fn):
        st = torch.cuda.ExternalStream(lib.cup_stream(ctx._p))
        with torch.cuda.stream(st):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        out = fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    # step 0 of every case, one by one and as the batch, from the same state;
    # each case's coarse space built before (as the batch's is at creation)
    if solver in ("b200_twolevel", "b200_twolevel_mixed"):
        for c in ctxs:
            r = torch.ones(c.nb * 512, dtype=torch.float64, device="cuda")
            c.coarse_apply(r, torch.zeros_like(r))
    single_ms = 0.0
    for c in ctxs:
        single_ms += timed(c, lambda: c.step(0))[0]
    batch0_ms, (_, _, _, st0) = timed(batch, lambda: batch.step(0))
    ms, its = [], []
    for k in range(1, steps + 1):
        t, (_, _, _, st) = timed(batch, lambda: batch.step(k))
        ms.append(t)
        its.append([x["iterations"] for x in st])
    for c in ctxs:
        c.close()
    batch.close()
    return {
        "workload": SWARM_WORKLOAD, "cases": 64, "cells": ncell, "solver": solver,
        "bodies": "moving (chi created again every step)" if moving else "held in place",
        "batch_create_s": round(setup_s, 2),
        "metric": "Mcell-steps/s (batched time steps of all cases)",
        "precision": ("FP32 inner Poisson solves in FP64 refinement, FP64 elsewhere" if solver.endswith("_mixed")
                      else "FP64"),
        "value": round(ncell * steps / (sum(ms) * 1e-3) / 1e6, 3), "steps": f"1..{steps} after step 0",
        "ms_per_step": [round(x, 2) for x in ms] if len(ms) <= 10 else
                       {"first5": [round(x, 2) for x in ms[:5]], "last5": [round(x, 2) for x in ms[-5:]],
                        "mean": round(sum(ms) / len(ms), 2)},
        "poisson_iterations_mean_max": [[round(sum(i) / len(i), 1), max(i)] for i in its] if len(its) <= 10 else
                                       {"first": [round(sum(its[0]) / len(its[0]), 1), max(its[0])],
                                        "last": [round(sum(its[-1]) / len(its[-1]), 1), max(its[-1])]},
        "step0": {"batch_ms": round(batch0_ms, 2), "one_by_one_ms": round(single_ms, 2),
                  "speedup": round(single_ms / batch0_ms, 3),
                  "poisson_iterations_mean_max": [round(sum(x["iterations"] for x in st0) / 64, 1),
                                                  max(x["iterations"] for x in st0)]},
    }


def obstacle_creation(reps=7):
    """Obstacle creation (CreateObstacles) on the host path (cup_obstacle_sphere:
    signed distance and chi on the host, then the upload) against the device
    path (cup_obstacle_sphere_dev: four kernels and one 96-byte read of the
    slot count and kinematics): wall time of the call, median of reps, for the
    sphere on the sphere mesh and for swarm case 0's ellipsoid.  Both paths
    give the same slot list and chi bit for bit."""
    import torch
    import cup3d_b200 as cup
    from cup3d_b200.workloads import SWARM_AXES, make_swarm_ctx, swarm_case
    lib = cup._lib.lib()
    dev = torch.cuda.current_device()
    out = {}
    sphere = make_sphere_ctx(dev)
    p = swarm_case(0)
    swarm = make_swarm_ctx(0, dev)
    cases = {
        "sphere": (sphere, lambda on: sphere.obstacle_sphere(**SPHERE_BODY, on_device=on)),
        "swarm_case0_ellipsoid": (swarm, lambda on: swarm.obstacle_ellipsoid(p["center"], SWARM_AXES, p["quat"],
                                                                              vel=p["vel"], on_device=on)),
    }
    for name, (ctx, make) in cases.items():
        st = torch.cuda.ExternalStream(lib.cup_stream(ctx._p))
        res = {"blocks": ctx.nb}
        for on in (False, True):
            make(on)  # warm
            wall, dev_ms = [], []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(st)
                t0 = time.perf_counter()
                make(on)
                wall.append((time.perf_counter() - t0) * 1e3)
                e1.record(st)
                e1.synchronize()
                dev_ms.append(e0.elapsed_time(e1))
            res["device" if on else "host"] = {"wall_ms": round(float(np.median(wall)), 4),
                                               "stream_ms": round(float(np.median(dev_ms)), 4)}
        res["slots"] = int((ctx.get_obstacle()[0] >= 0).sum())
        res["speedup_wall"] = round(res["host"]["wall_ms"] / res["device"]["wall_ms"], 2)
        out[name] = res
    return out


def mesh_adaptation(ctx, stream, step0, rounds=3, every=20):
    """Mesh adaptation on the reference's cadence (Simulation.cpp:385: every
    20 steps), timed apart from the steps, which the metric leaves it out of.
    From the settled sphere state, `rounds` times: one adaptation
    (cup_adapt_mesh: device vorticity indicator, host refine/compress with
    2:1 balance, device field transfer, chi created again), the two-level
    coarse space of the new mesh (A_c through the device operator, blocked
    inverse; built by the first coarse application), then `every` steps on
    the new mesh.  Wall time of the calls, device time of the steps.  Also
    the dense inverse alone on the final mesh's A_c: the blocked form, and
    the column-wise pivoted form (forced by a cyclic shift of the rows, so
    its time includes the failed blocked attempt)."""
    import torch
    out = []
    step = step0
    for _ in range(rounds):
        nb0 = ctx.nb
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        changed = ctx.adapt_mesh()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        r = torch.ones(ctx.nb * 512, dtype=torch.float64, device="cuda")
        z = torch.zeros_like(r)
        ctx.coarse_apply(r, z)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        its = []
        e0.record(stream)
        for _ in range(every):
            _, rc, st = ctx.step(step)
            step += 1
            its.append(st["iterations"])
        e1.record(stream)
        e1.synchronize()
        out.append({"changed": bool(changed), "blocks_before": nb0, "blocks_after": ctx.nb,
                    "adapt_ms": round((t1 - t0) * 1e3, 3), "coarse_build_ms": round((t2 - t1) * 1e3, 3),
                    "step_ms": round(e0.elapsed_time(e1) / every, 4),
                    "poisson_iterations_mean": round(float(np.mean(its)), 2)})
    Ac, _ = ctx.coarse_matrix()
    level, index, _ = ctx.blocks()
    mb = int(np.where((index == 0).all(axis=1))[0][0])
    inv = {}
    for name, mat, last in (("blocked", Ac, mb), ("column_pivoted", np.roll(Ac, 1, axis=0), -1)):
        a = torch.tensor(mat, device="cuda")
        ctx.dense_inverse(a.clone(), last)  # warm
        ts = []
        for _ in range(3):
            b = a.clone()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            piv = ctx.dense_inverse(b, last)
            ts.append((time.perf_counter() - t0) * 1e3)
        inv[name] = {"ms": round(float(np.median(ts)), 3), "pivoted": bool(piv)}
    amort = np.mean([o["adapt_ms"] + o["coarse_build_ms"] for o in out]) / every
    return {"cadence_steps": every, "rounds": out, "amortized_ms_per_step": round(float(amort), 4),
            "dense_inverse": dict(inv, n=int(len(Ac)))}


def run_b200(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    import cup3d_b200 as cup
    ctx = make_sphere_ctx(local, args.solver)
    ctx.solver_name = args.solver
    nb = ctx.nb
    ncell = nb * 512
    stream = torch.cuda.ExternalStream(cup._lib.lib().cup_stream(ctx._p))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    step = 0
    # untimed: the warm-up steps, then settling steps past the start of the
    # CFL ramp; the flow's pressure right-hand sides of some of them are kept
    # as training data of the learned preconditioner
    rhs_list = []
    for k in range(args.warmup + args.settle):
        ctx.step(step)
        step += 1
        if k % 4 == 3 and len(rhs_list) < 12:
            rhs_list.append(ctx.download("lhs"))
    # The timed pass, the per-kernel pass and the end-to-end pass all run the
    # same K steps from the same state (velocity and pressure are the whole
    # state carried between steps), so their Poisson solves do the same work.
    first_step = step
    vel_h = torch.empty(3 * ncell, dtype=torch.float64).pin_memory()
    pres_h = torch.empty(ncell, dtype=torch.float64).pin_memory()
    vel0 = ctx.download("vel")
    pres0 = ctx.download("pres")

    def restore():
        ctx.upload("vel", vel0)
        ctx.upload("pres", pres0)
        torch.cuda.synchronize()
        return first_step
    # ---- timed region: device-resident --------------------------------------
    clocks = ClockSampler(local)
    clocks.start()
    times = []
    iters = []
    solve_ms = []
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)  # L2 flush outside the timed events
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dt, rc, st = ctx.step(step)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        iters.append(st["iterations"])
        solve_ms.append(st["milliseconds"])
        step += 1
    torch.cuda.synchronize()
    clk = clocks.stop()
    # ---- per-kernel pass: the same K steps again with CUDA events around every
    # launch (kept out of the timed region above, whose number it would lower)
    step = restore()
    ctx.profile(True)
    prof_iters = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        _, _, st = ctx.step(step)
        prof_iters.append(st["iterations"])
        step += 1
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    total_ms = sum(times)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * ncell * args.steps / (total_ms * 1e-3) / 1e6
    # launches in the timed region: the per-kernel pass's count with its
    # BiCGSTAB launches (5 kernels per iteration, issued in chunks of 8
    # iterations between host convergence checks) replaced by the timed steps'
    def bicg_launches(its):
        return sum(5 * 8 * ((k + 7) // 8) for k in its)
    per_phase = any(k.startswith("bicg_a") for k in prof)
    launches = sum(v[0] for v in prof.values())
    if per_phase:
        launches += bicg_launches(iters) - bicg_launches(prof_iters)
    # roofline of the dominant kernel (largest total device time)
    peak, peak_kind = measured_peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][1])
    dom_name, (dom_n, dom_ms) = dom
    per_launch_ms = dom_ms / max(dom_n, 1)
    if dom_name == "bicg_persistent":
        # one launch per solve, 176 B/cell per iteration; the two-level solver
        # adds two coarse corrections per iteration: a read-modify-write of z
        # (16 B/cell) and a row of A_c^-1 per block (8 nb^2 bytes) each
        per_cell = ALG_BYTES[dom_name] + (32 if args.solver == "b200_twolevel" else 0)
        per_iter = per_cell * ncell + (16 * nb * nb if args.solver == "b200_twolevel" else 0)
        alg_bytes = int(per_iter * sum(prof_iters) / max(dom_n, 1))
    else:
        alg_bytes = ALG_BYTES.get(dom_name, 0) * ncell
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9 if alg_bytes else None
    traffic = None
    if (dom_name, args.solver) in MEASURED_TRAFFIC_PER_CELL_ITER:
        traffic = int(MEASURED_TRAFFIC_PER_CELL_ITER[dom_name, args.solver] * ncell * sum(prof_iters) / max(dom_n, 1))
    # ---- e2e through the C ABI with host buffers: the same K steps, the state
    # uploaded from pinned host memory before and downloaded after every step
    step = restore()
    vel_h.numpy()[:] = vel0
    pres_h.numpy()[:] = pres0
    e2e_iters = []
    lib = cup._lib.lib()
    import ctypes as C
    vp = C.cast(vel_h.data_ptr(), cup._lib._D)
    pp = C.cast(pres_h.data_ptr(), cup._lib._D)
    e2e_ms = 0.0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cup._lib.check(lib.cup_upload_field(ctx._p, 0, vp), ctx._p)
        cup._lib.check(lib.cup_upload_field(ctx._p, 1, pp), ctx._p)
        _, _, st = ctx.step(step)
        e2e_iters.append(st["iterations"])
        cup._lib.check(lib.cup_download_field(ctx._p, 0, vp), ctx._p)
        cup._lib.check(lib.cup_download_field(ctx._p, 1, pp), ctx._p)
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        step += 1
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * ncell * args.steps / (e2e_ms * 1e-3) / 1e6
    line = {
        "metric": "Mcell-steps/s (whole time step, sphere Re=300 AMR, FP64)",
        "value": round(value, 3),
        "unit": "Mcell-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(total_ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded, generated in-process)",
        "config": {"workload": WORKLOAD, "blocks": nb, "cells": ncell, "levels_used": [1, 2, 3],
                   "poisson": f"{args.solver}: FP64 BiCGSTAB, "
                              + ("two-level preconditioner (block-constant coarse space + exact block inverse)"
                                 if args.solver == "b200_twolevel" else "exact block inverse")
                              + ", tol 1e-6 abs / 1e-4 rel (PoissonErrorTol / PoissonErrorTolRel)",
                   "parallelism": f"replicas x{world}", "l2": "flushed (256 MB write) between timed steps",
                   "first_timed_step": args.warmup + args.settle},
        "poisson": {"iterations_per_step": iters, "solve_ms_per_step": [round(x, 3) for x in solve_ms]},
        "kernels": {"pass": f"the same {args.steps} steps again with per-launch CUDA events "
                            f"(Poisson iterations {prof_iters})",
                    **{k: {"launches": v[0], "ms": round(v[1], 4)}
                       for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])}},
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1) if achieved else None,
                     "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4) if achieved else None,
                     "peak_source": peak_kind, "alg_bytes_per_launch": alg_bytes,
                     "launch_ms": round(per_launch_ms, 5), "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per iteration (16-iteration "
                                       "capture), scaled by the iterations of the launch" if traffic else None},
        "e2e": {"value": round(e2e_value, 3), "unit": "Mcell-steps/s", "poisson_iterations": e2e_iters,
                "h2d_bytes_per_step": 4 * 8 * ncell, "d2h_bytes_per_step": 4 * 8 * ncell},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if not args.no_poisson:
        line["poisson_to_tolerance"] = poisson_at_tolerance(ctx, stream, flush, rhs_list)
        if rank == 0:
            line["learned_re1000"] = learned_re1000(ctx, flush)
    if rank == 0 and not args.no_swarm:
        # the swarm's 200 steps with moving bodies and the two-level solver,
        # FP64 and mixed precision; 5 steps with the block inverse alone (FP64,
        # mixed precision), bodies in place, for comparison
        line["swarm_batch"] = {s: swarm_batch(flush, steps=n, solver=s, moving=mv)
                               for s, n, mv in (("b200", 5, False), ("b200_mixed", 5, False),
                                                ("b200_twolevel", 200, True),
                                                ("b200_twolevel_mixed", 200, True))}
    if rank == 0 and not args.no_obstacle:
        line["obstacle_creation"] = obstacle_creation()
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(ctx, args, (vel0, pres0), first_step)
    if rank == 0 and not args.no_adapt:
        # last: it changes the context's mesh
        line["mesh_adaptation"] = mesh_adaptation(ctx, stream, restore())
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_reference_step(ctx_host_state, m, slot, chi_o, udef_o, kin, chi, step, uinf, nu, cfl, lam):
    """One step of the reference CPU path restated in the oracle (timed)."""
    import oracle
    vel, pres = ctx_host_state
    umax = m.max_u(vel, uinf)
    dt = oracle.dt(m.hmin, nu, cfl, umax, step, 100)
    t0 = time.perf_counter()
    vel = m.advect_diffuse(vel, dt, nu, uinf=uinf, scheme=1)
    vel, _ = m.penalize(vel, chi, slot, chi_o, udef_o, kin, dt, lam=lam, implicit=1)
    vel, pres, info = m.pressure_project(vel, pres, dt, step, chi=chi, slot=slot, chi_o=chi_o, udef_o=udef_o,
                                         solver=1, tol=1e-6, tol_rel=1e-4)
    return time.perf_counter() - t0, (vel, pres), info


def cpu_baseline(ctx, args, state, step):
    """One step of the oracle's restatement of the reference CPU path, from the
    state of the first timed step."""
    import oracle
    level, index, _ = ctx.blocks()
    m = oracle.Mesh(level, index, [4, 2, 2], 4, [0, 0, 0], 4.0)
    slot, chi_o, udef_o, kin = ctx.get_obstacle()
    chi = ctx.download("chi")
    secs, _, info = cpu_reference_step(state, m, slot, chi_o, udef_o, kin, chi, step,
                                       (-0.1, 0.0, 0.0), 4.1666666666666667e-05, 0.3, 1e6)
    return {"value": round(m.n / secs / 1e6, 4), "unit": "Mcell-steps/s", "cores": os.cpu_count(),
            "cpu_model": cpu_model(), "kind": "port",
            "sample": f"1 full time step of the same workload from the state of the first timed step "
                      f"(oracle, OpenMP, pipelined BiCGSTAB + block CG, {info['iterations']} iterations, "
                      f"{secs:.2f} s)"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    """The reference's CPU path restated (oracle) on the host cores, on its
    own inputs: the mesh leaves from the pure-Python generator and the sphere
    from the oracle's CreateObstacles, so the library is never loaded."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    from cup3d_b200.workloads import sphere_wake_leaves
    leaves = sphere_wake_leaves()
    m = oracle.Mesh(leaves[:, 0], leaves[:, 1:], [4, 2, 2], 4, [0, 0, 0], 4.0)
    ob = m.create_obstacle("sphere", SPHERE_BODY["center"], SPHERE_BODY["radius"])
    slot, chi_o, chi = ob["slot"], ob["chi_o"], ob["chi"]
    udef_o = np.zeros(3 * len(chi_o))
    kin = np.concatenate([ob["com"], SPHERE_BODY["vel"], [0.0, 0.0, 0.0]])
    vel = np.zeros(3 * m.n)
    pres = np.zeros(m.n)
    state = (vel, pres)
    step = 0
    for _ in range(args.warmup):
        _, state, _ = cpu_reference_step(state, m, slot, chi_o, udef_o, kin, chi, step, (-0.1, 0, 0),
                                         4.1666666666666667e-05, 0.3, 1e6)
        step += 1
    total = 0.0
    for _ in range(args.steps):
        secs, state, _ = cpu_reference_step(state, m, slot, chi_o, udef_o, kin, chi, step, (-0.1, 0, 0),
                                            4.1666666666666667e-05, 0.3, 1e6)
        total += secs
        step += 1
    value = m.n * args.steps / total / 1e6
    line = {
        "impl": "reference",
        "metric": "Mcell-steps/s (whole time step, sphere Re=300 AMR, FP64)",
        "value": round(value, 4), "unit": "Mcell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * total / args.steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "blocks": m.nb, "cells": m.n},
        "cpu_baseline": {"value": round(value, 4), "unit": "Mcell-steps/s", "cores": os.cpu_count(),
                         "cpu_model": cpu_model(), "kind": "port",
                         "sample": "full time steps from rest on the frozen sphere mesh (oracle restatement of the "
                                   "reference CPU path, OpenMP over blocks; mesh and sphere built by the oracle "
                                   "side, not the library)"},
        "e2e": {"value": round(value, 4), "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--solver", default="b200_twolevel", choices=["b200", "b200_twolevel"],
                    help="Poisson solver of the timed steps")
    ap.add_argument("--settle", type=int, default=50, help="untimed steps after the warm-up")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-poisson", action="store_true", help="skip the Poisson-to-tolerance comparison")
    ap.add_argument("--no-swarm", action="store_true", help="skip the batched ellipsoid-swarm measurement")
    ap.add_argument("--no-obstacle", action="store_true", help="skip the obstacle-creation measurement")
    ap.add_argument("--no-adapt", action="store_true", help="skip the mesh-adaptation measurement")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
