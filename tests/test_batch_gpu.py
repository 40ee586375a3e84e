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
* the single-case entry points refuse a batch.
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
