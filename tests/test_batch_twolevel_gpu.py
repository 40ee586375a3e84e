"""The two-level preconditioner in a batch of cases (cup_batch_create with
-poissonSolver b200_twolevel): each case keeps its own coarse space (built on
its own context, packed block-diagonally), and the batched solver adds each
case's coarse correction to that case's blocks.

* every case converges to the FP64 tolerance on the oracle's operator, to the
  solution of the same case solved alone with the two-level solver (within
  1e-8), in about as many iterations (the batch sums each case's dot products
  over its block groups, in another order), and in fewer iterations than the
  batched block-inverse solver;
* batch time steps with it, replayed from a CUDA graph, equal the launched
  batch steps bit for bit.
"""
import numpy as np
import pytest

import cup3d_b200 as cup
from tests.meshes import make_ctx, oracle_mesh
from tests.test_batch_gpu import _step_cases, compatible_rhs, mean_row_zeroed, split, torch_dev

pytestmark = pytest.mark.gpu

NAMES = ["tgv32", "amr2_free", "amr3_mixed", "amr3_periodic"]


def _batch(solver):
    flags = f"-poissonTol 0 -poissonTolRel 1e-10 -poissonSolver {solver}"
    ctxs = [make_ctx(n, device=0, extra=flags) for n in NAMES]
    return ctxs, cup.Batch(ctxs)


def test_batched_twolevel_matches_cases_alone():
    ctxs, batch = _batch("b200_twolevel")
    meshes = [oracle_mesh(c) for c in ctxs]
    bs = [compatible_rhs(m, 40 + k) for k, m in enumerate(meshes)]
    bd, xd = torch_dev(np.concatenate(bs)), torch_dev(np.zeros(sum(m.n for m in meshes)))
    rc, stats = batch.poisson_solve_dev(bd, xd)
    assert rc == 0
    xs = split(batch, xd.cpu().numpy())
    _, plain = _batch("b200")
    xp = torch_dev(np.zeros(sum(m.n for m in meshes)))
    rcp, stats_plain = plain.poisson_solve_dev(torch_dev(np.concatenate(bs)), xp)
    assert rcp == 0
    for k, (ctx, m, b, x, st) in enumerate(zip(ctxs, meshes, bs, xs, stats)):
        assert st["status"] == 1, (k, st)
        bb = mean_row_zeroed(ctx, m, b)
        mc = ctx.cfg.mean_constraint
        assert np.linalg.norm(bb - m.apply(x, mean_constraint=mc)) <= 1.05e-10 * np.linalg.norm(bb), k
        xa = torch_dev(np.zeros(m.n))
        rca, sta = ctx.poisson_solve_dev(torch_dev(b), xa)
        assert rca == 0 and sta["status"] == 1
        xa = xa.cpu().numpy()
        print(NAMES[k], "iterations: batched two-level", st["iterations"], "alone", sta["iterations"],
              "batched block inverse", stats_plain[k]["iterations"])
        assert np.linalg.norm(x - xa) <= 1e-8 * np.linalg.norm(xa), k
        assert abs(st["iterations"] - sta["iterations"]) <= max(2, sta["iterations"] // 10), (k, st, sta)
        assert st["iterations"] < stats_plain[k]["iterations"], k


def test_captured_batched_twolevel_steps_match_launched():
    batches = [cup.Batch(_step_cases(f"-stepGraph {g} -poissonSolver b200_twolevel")) for g in (1, 0)]
    for step in range(3):
        out = [b.step(step) for b in batches]
        (rc1, dt1, f1, st1), (rc0, dt0, f0, st0) = out
        assert rc1 == rc0 == 0 and np.array_equal(dt1, dt0) and np.array_equal(f1, f0), step
        assert [s["iterations"] for s in st1] == [s["iterations"] for s in st0], step
        assert np.array_equal(batches[0].download("vel"), batches[1].download("vel")), step
        assert np.array_equal(batches[0].download("pres"), batches[1].download("pres")), step


def test_batched_twolevel_mixed_precision():
    # -poissonSolver b200_twolevel_mixed on a batch: FP32 batched inner solves
    # with each case's coarse correction, FP64 refinement per case.  Every case
    # meets the FP64 tolerance on the oracle's operator, agrees with the FP64
    # batched two-level solve, and needs fewer inner iterations than the
    # batched block inverse in mixed precision.
    sols = {}
    for solver in ("b200_twolevel", "b200_twolevel_mixed", "b200_mixed"):
        ctxs, batch = _batch(solver)
        meshes = [oracle_mesh(c) for c in ctxs]
        bs = [compatible_rhs(m, 40 + k) for k, m in enumerate(meshes)]
        bd, xd = torch_dev(np.concatenate(bs)), torch_dev(np.zeros(sum(m.n for m in meshes)))
        rc, stats = batch.poisson_solve_dev(bd, xd)
        assert rc == 0, (solver, stats)
        xs = split(batch, xd.cpu().numpy())
        for k, (ctx, m, b, x, st) in enumerate(zip(ctxs, meshes, bs, xs, stats)):
            assert st["status"] == 1, (solver, k, st)
            bb = mean_row_zeroed(ctx, m, b)
            res = np.linalg.norm(bb - m.apply(x, mean_constraint=ctx.cfg.mean_constraint))
            assert res <= 1.05e-10 * np.linalg.norm(bb), (solver, k, res)
        sols[solver] = (xs, [s["iterations"] for s in stats])
    print("iterations two-level FP64 / two-level mixed / block inverse mixed:",
          *(sols[s][1] for s in ("b200_twolevel", "b200_twolevel_mixed", "b200_mixed")))
    for k in range(len(NAMES)):
        x64, x32 = sols["b200_twolevel"][0][k], sols["b200_twolevel_mixed"][0][k]
        assert np.linalg.norm(x32 - x64) <= 1e-8 * np.linalg.norm(x64), k
    assert sum(sols["b200_twolevel_mixed"][1]) < sum(sols["b200_mixed"][1]), sols
