"""Batched Poisson solves (cup_batch_*): independent cases in one launch.

* each case of a batch meets the standard of a case solved alone: FP64
  residual on the oracle's operator within the tolerance, solution within
  1e-8 of the oracle's, iteration count within 25% of the oracle's (the
  batch sums each case's dot products over that case's block groups, in
  another order than the single-case solver);
* a case with a zero right-hand side stops at once and keeps x0 = 0 while
  the others run on;
* with more than four blocks per block group (three copies of the sphere
  mesh) the batch stages block tables on the way; every case's FP64
  residual on its own context's device operator is within the tolerance;
* the single-case entry points refuse a batch;
* time steps of a batch (own dt, obstacle, mean and solve per case) match
  the same cases stepped one by one, and replayed from a CUDA graph they
  match the kernel-by-kernel batch step bit for bit;
* with moving bodies each case's pose and chi follow those of the case
  stepped alone, chi bit for bit.
"""
import numpy as np
import pytest

import cup3d_b200 as cup
from tests.meshes import make_ctx, oracle_mesh

pytestmark = pytest.mark.gpu

FLAGS = "-poissonTol 0 -poissonTolRel 1e-10"


def torch_dev(a):
    import torch
    return torch.tensor(np.asarray(a, np.float64), device="cuda")


def compatible_rhs(m, seed):
    b = np.random.default_rng(seed).standard_normal(m.n)
    hh = np.repeat(m.h, 512)
    return b - np.sum(b * hh ** 3) / np.sum(hh ** 3)


def mean_row_zeroed(ctx, m, b):
    bb = b.copy()
    if ctx.cfg.mean_constraint in (1, 3):
        mb = int(np.where((ctx.blocks()[1] == 0).all(axis=1))[0][0])
        bb[mb * 512] = 0.0
    return bb


def split(batch, x):
    out = []
    for k in range(batch.ncase):
        first, n = batch.case_blocks(k)
        out.append(x[first * 512:(first + n) * 512])
    return out


def test_batch_cases_match_oracle():
    names = ["tgv32", "amr2_free", "amr3_mixed", "amr3_periodic"]
    ctxs = [make_ctx(n, device=0, extra=FLAGS) for n in names]
    meshes = [oracle_mesh(c) for c in ctxs]
    bs = [compatible_rhs(m, 20 + k) for k, m in enumerate(meshes)]
    batch = cup.Batch(ctxs)
    assert batch.ncase == 4
    assert [batch.case_blocks(k)[1] for k in range(4)] == [m.nb for m in meshes]
    bd, xd = torch_dev(np.concatenate(bs)), torch_dev(np.zeros(sum(m.n for m in meshes)))
    rc, stats = batch.poisson_solve_dev(bd, xd)
    assert rc == 0
    xs = split(batch, xd.cpu().numpy())
    for k, (ctx, m, b, x, st) in enumerate(zip(ctxs, meshes, bs, xs, stats)):
        assert st["status"] == 1, (k, st)
        x_ref, st_ref = m.bicgstab_gpu(b, tol=0.0, tol_rel=1e-10)
        bb = mean_row_zeroed(ctx, m, b)
        mc = ctx.cfg.mean_constraint
        assert np.linalg.norm(bb - m.apply(x, mean_constraint=mc)) <= 1.05e-10 * np.linalg.norm(bb), k
        assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref), k
        assert abs(st["iterations"] - st_ref["iterations"]) <= max(3, st_ref["iterations"] // 4), (k, st, st_ref)
    with pytest.raises(cup.CupError):
        batch.poisson_solve()


def test_batch_mixed_precision_solve():
    # -poissonSolver b200_mixed on a batch: FP32 inner solves of all cases in
    # one launch inside FP64 refinement per case.  Each case reaches the FP64
    # true residual on the oracle's operator, its solution agrees with the
    # FP64 batched solve, and a case whose right-hand side is zero stays at
    # x = 0 while the others refine.
    names = ["tgv32", "amr2_free", "amr3_mixed"]
    sols = {}
    for solver in ("b200", "b200_mixed"):
        ctxs = [make_ctx(n, device=0, extra=FLAGS + f" -poissonSolver {solver}") for n in names]
        meshes = [oracle_mesh(c) for c in ctxs]
        bs = [compatible_rhs(m, 40 + k) for k, m in enumerate(meshes)]
        bs[1] = np.zeros_like(bs[1])
        batch = cup.Batch(ctxs)
        bd, xd = torch_dev(np.concatenate(bs)), torch_dev(np.zeros(sum(m.n for m in meshes)))
        rc, stats = batch.poisson_solve_dev(bd, xd)
        assert rc == 0, (solver, stats)
        xs = split(batch, xd.cpu().numpy())
        for k, (ctx, m, b, x, st) in enumerate(zip(ctxs, meshes, bs, xs, stats)):
            assert st["status"] == 1, (solver, k, st)
            bb = mean_row_zeroed(ctx, m, b)
            res = np.linalg.norm(bb - m.apply(x, mean_constraint=ctx.cfg.mean_constraint))
            assert res <= 1.05e-10 * max(np.linalg.norm(bb), 1e-300) or k == 1, (solver, k, res)
        assert not np.any(xs[1]), solver
        sols[solver] = (xs, stats)
    print("iterations FP64 / mixed (inner):", [s["iterations"] for s in sols["b200"][1]],
          [s["iterations"] for s in sols["b200_mixed"][1]])
    for k in (0, 2):
        x64, x32 = sols["b200"][0][k], sols["b200_mixed"][0][k]
        assert np.linalg.norm(x32 - x64) <= 1e-8 * np.linalg.norm(x64), k


def test_batch_refuses_single_case_solvers():
    # the learned, Schwarz and pipelined solvers are single-case only: a
    # batch solve with one of them is an error, not a silent other solver
    ctxs = [make_ctx(n, device=0, extra=FLAGS) for n in ("tgv32", "amr2_free")]
    batch = cup.Batch(ctxs)
    n = sum(c.nb * 512 for c in ctxs)
    bd, xd = torch_dev(np.zeros(n)), torch_dev(np.zeros(n))
    for solver in ("b200_learned", "b200_learned_mixed", "b200_schwarz", "b200_pipelined"):
        batch.set_poisson(solver, 0.0, 1e-8, 100)
        with pytest.raises(cup.CupError):
            batch.poisson_solve_dev(bd, xd)
    batch.set_poisson("b200", 0.0, 1e-8, 100)
    rc, stats = batch.poisson_solve_dev(bd, xd)
    assert rc == 0


def test_batch_zero_rhs_case_stops_at_once():
    ctxs = [make_ctx(n, device=0, extra=FLAGS) for n in ["amr2_free", "tgv32", "amr3_mixed"]]
    meshes = [oracle_mesh(c) for c in ctxs]
    bs = [compatible_rhs(meshes[0], 5), np.zeros(meshes[1].n), compatible_rhs(meshes[2], 6)]
    batch = cup.Batch(ctxs)
    bd, xd = torch_dev(np.concatenate(bs)), torch_dev(np.zeros(sum(m.n for m in meshes)))
    rc, stats = batch.poisson_solve_dev(bd, xd)
    xs = split(batch, xd.cpu().numpy())
    assert rc == 0
    assert stats[1]["iterations"] == 0 and stats[1]["status"] == 1
    assert np.abs(xs[1]).max() == 0.0
    for k in (0, 2):
        assert stats[k]["status"] == 1 and stats[k]["iterations"] > 10
        x_ref, _ = meshes[k].bicgstab_gpu(bs[k], tol=0.0, tol_rel=1e-10)
        assert np.linalg.norm(xs[k] - x_ref) <= 1e-8 * np.linalg.norm(x_ref), k


def test_batch_staged_tables_solve_every_case():
    # three copies of the sphere mesh (7020 blocks): about six blocks per
    # block group, so most groups stage block tables on the way.  At 1e-10
    # the sphere solve's iteration count moves with the summation order
    # (restarts land elsewhere), so each case is checked by its FP64
    # residual on the device operator of its own context.
    from cup3d_b200.workloads import make_sphere_ctx
    ctxs = [make_sphere_ctx(0) for _ in range(3)]
    for c in ctxs:
        c.set_poisson("b200", 0.0, 1e-10, 1000)
    n = ctxs[0].nb * 512
    hh = np.repeat(ctxs[0].blocks()[2], 512)
    bs = []
    for k in range(3):
        b = np.random.default_rng(40 + k).standard_normal(n)
        bs.append(b - np.sum(b * hh ** 3) / np.sum(hh ** 3))
    batch = cup.Batch(ctxs)
    assert batch.nb > 4 * 148 * 2 * 4  # more than four blocks per block group
    bd, xd = torch_dev(np.concatenate(bs)), torch_dev(np.zeros(3 * n))
    rc, stats = batch.poisson_solve_dev(bd, xd)
    assert rc == 0
    xs = split(batch, xd.cpu().numpy())
    mb = int(np.where((ctxs[0].blocks()[1] == 0).all(axis=1))[0][0])
    for k in range(3):
        assert stats[k]["status"] == 1, (k, stats[k])
        xk = torch_dev(xs[k])
        yk = torch_dev(np.zeros(n))
        ctxs[k].poisson_apply(xk, yk, ctxs[k].cfg.mean_constraint)
        bb = bs[k].copy()
        bb[mb * 512] = 0.0
        assert np.linalg.norm(bb - yk.cpu().numpy()) <= 1.05e-10 * np.linalg.norm(bb), k


def _smooth_velocity(ctx, phase):
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    return np.concatenate([np.sin(2 * x + phase) * np.cos(3 * y), 0.5 * np.cos(x - phase) * np.sin(2 * z),
                           0.3 * np.sin(y + z + phase)])


def _step_cases(extra="", static=True):
    flags = ("-poissonTol 0 -poissonTolRel 1e-11 -nu 0.01 -CFL 0.3 -rampup 0 -advection weno5 "
             f"-StaticObstacles {1 if static else 0} " + extra)
    a = make_ctx("tgv32", device=0, extra=flags)
    xyz, _ = a.cell_centres()
    x, y, z = xyz.T
    a.upload("vel", np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), 0 * x]))
    b = make_ctx("amr2_free", device=0, extra=flags)
    b.upload("vel", _smooth_velocity(b, 0.3))
    b.obstacle_sphere((0.5, 0.45, 0.55), 0.15, vel=(0.1, 0.0, 0.0))
    c = make_ctx("amr3_mixed", device=0, extra=flags)
    c.upload("vel", _smooth_velocity(c, 1.1))
    q = np.array([0.9, 0.1, 0.3, 0.3])
    c.obstacle_ellipsoid((1.0, 0.5, 0.75), (0.2, 0.1, 0.1), q / np.linalg.norm(q), vel=(0.0, 0.05, 0.0))
    return [a, b, c]


def test_batch_steps_match_single_cases():
    # each case stepped alone (cup_compute_dt, cup_advect_diffuse,
    # cup_penalize, cup_pressure_project) against the same cases stepped
    # together, through two steps.  The Poisson solves to 1e-11 sum their
    # dot products in another order, so the fields differ at that level:
    # dt bit for bit in the first step (max |u| does not depend on the
    # order) and within 1e-10 after; the single cases then step with the
    # batch's dt; velocities within 1e-8 of max|u|, forces within 1e-8 of
    # their size, pressure within 1e-7 of max|p|
    singles = _step_cases()
    batch = cup.Batch(_step_cases())
    for step in range(2):
        rc, dts, forces, stats = batch.step(step)
        assert rc == 0 and all(s["status"] == 1 for s in stats)
        for k, s in enumerate(singles):
            dt1 = s.compute_dt(step)
            assert (dt1 == dts[k]) if step == 0 else abs(dt1 - dts[k]) <= 1e-10 * dt1, (step, k, dt1, dts[k])
            dt = dts[k]
            s.advect_diffuse(dt)
            f = s.penalize(dt) if k > 0 else np.zeros(6)
            s.pressure_project(dt, step)
            u1 = s.download("vel").reshape(3, -1)
            ub = batch.case_field("vel", k)
            scale = np.abs(u1).max()
            assert np.abs(ub - u1).max() <= 1e-8 * scale, (step, k, np.abs(ub - u1).max() / scale)
            assert np.abs(forces[k] - f).max() <= 1e-8 * max(np.abs(f).max(), 1e-30), (step, k, forces[k], f)
            p1 = s.download("pres")
            pb = batch.case_field("pres", k)[0]
            assert np.abs(pb - p1).max() <= 1e-7 * np.abs(p1).max(), (step, k)


def test_captured_batch_steps_match_launched_batch_steps():
    # the batch step replayed as a CUDA graph (per-case dt on the device)
    # against the same step launched kernel by kernel: bit for bit
    batches = [cup.Batch(_step_cases(f"-stepGraph {g}")) for g in (1, 0)]
    for step in range(4):
        out = [b.step(step) for b in batches]
        (rc1, dt1, f1, st1), (rc0, dt0, f0, st0) = out
        assert rc1 == rc0 and np.array_equal(dt1, dt0) and np.array_equal(f1, f0), step
        assert [s["iterations"] for s in st1] == [s["iterations"] for s in st0], step
        assert np.array_equal(batches[0].download("vel"), batches[1].download("vel")), step
        assert np.array_equal(batches[0].download("pres"), batches[1].download("pres")), step


@pytest.mark.parametrize("solver", ["b200", "b200_twolevel_mixed"])
def test_moving_batch_matches_single_cases(solver):
    # bodies that move (-StaticObstacles 0): every batch step advances each
    # case's pose with the case's own dt and BDF2 history and creates all
    # bodies again on the flattened mesh; each case stepped alone by
    # cup_step with the batch's dt moves its body the same way.  chi bit for
    # bit at every step (the same creation arithmetic), velocity within 1e-7
    # of max |u| and pressure within 1e-6 of max |p| (solves to 1e-10 that sum
    # in other orders), with the FP64 block inverse and with the two-level
    # preconditioner in mixed precision
    # (a relative 1e-10: at 1e-11 a case's solve can stall on rounding)
    flags = f"-poissonTolRel 1e-10 -poissonSolver {solver}"
    singles = _step_cases("-stepGraph 0 " + flags, static=False)
    batch = cup.Batch(_step_cases(flags, static=False))
    chi0 = [batch.case_field("chi", k)[0].copy() for k in range(batch.ncase)]
    # steps 0-2: Euler, then BDF2 poses
    for step in range(3):
        rc, dts, forces, stats = batch.step(step)
        assert rc == 0 and all(s["status"] == 1 for s in stats), (step, stats)
        for k, s in enumerate(singles):
            dt1, rc1, st1 = s.step(step, dt=dts[k])
            assert rc1 >= 0 and dt1 == dts[k], (step, k, rc1, st1)
            assert np.array_equal(batch.case_field("chi", k)[0], s.download("chi")), (step, k)
            u1 = s.download("vel").reshape(3, -1)
            ub = batch.case_field("vel", k)
            scale = np.abs(u1).max()
            assert np.abs(ub - u1).max() <= 1e-7 * scale, (step, k, np.abs(ub - u1).max() / scale)
            p1 = s.download("pres")
            pb = batch.case_field("pres", k)[0]
            assert np.abs(pb - p1).max() <= 1e-6 * np.abs(p1).max(), (step, k)
    # the bodies moved: chi changed in the cases with a body
    assert np.array_equal(batch.case_field("chi", 0)[0], chi0[0])
    for k in (1, 2):
        assert not np.array_equal(batch.case_field("chi", k)[0], chi0[k]), k


def test_batch_with_a_single_block_case():
    # a one-block periodic case (every face its own neighbour) next to an AMR
    # case: both solved in the same launch, each to the oracle's standard
    one = cup.Context(cup.config("-bpdx 1 -bpdy 1 -bpdz 1 -levelMax 1 -extent 1 -BC_x periodic -BC_y periodic "
                                 "-BC_z periodic " + FLAGS, device=0))
    one.set_mesh_uniform()
    amr = make_ctx("amr2_free", device=0, extra=FLAGS)
    meshes = [oracle_mesh(one), oracle_mesh(amr)]
    bs = [compatible_rhs(m, 60 + k) for k, m in enumerate(meshes)]
    batch = cup.Batch([one, amr])
    bd, xd = torch_dev(np.concatenate(bs)), torch_dev(np.zeros(sum(m.n for m in meshes)))
    rc, stats = batch.poisson_solve_dev(bd, xd)
    assert rc == 0
    for m, b, x, st in zip(meshes, bs, split(batch, xd.cpu().numpy()), stats):
        x_ref, _ = m.bicgstab_gpu(b, tol=0.0, tol_rel=1e-10)
        assert st["status"] == 1
        assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
