"""Mesh adaptation on the device (cup_adapt_indicator, cup_adapt_mesh) against
the oracle's restatement (Simulation::adaptMesh, Simulation.cpp:128-149):

* the per-block indicator (vorticity magnitude with GradChiOnTmp's marks)
  within 1e-12 of the oracle's, the interface marks equal;
* the adapted leaf list equal to the oracle's decision, bit for bit, and the
  velocity and pressure moved onto it as the oracle moves them;
* the flow past the sphere from -levelStart 3 with -Rtol 1 -Ctol 0.1: the
  initial refinement (Simulation::initialGridRefinement) and steps with the
  reference's cadence (every 20 steps) run, and two runs give the same meshes.
"""
import numpy as np
import pytest

import cup3d_b200 as cup
from tests.meshes import cell_centres, make_ctx, oracle_mesh

pytestmark = pytest.mark.gpu


def _flow(ctx):
    xyz, _ = cell_centres(ctx)
    x, y, z = xyz.T
    k = 2 * np.pi
    return np.concatenate([np.sin(k * x) * np.cos(k * y) + 0.3 * np.sin(3 * k * z),
                           -np.cos(k * x) * np.sin(k * y) + 0.2 * np.cos(2 * k * x),
                           0.4 * np.sin(k * (x + y)) * np.cos(k * z)])


def _setup(rtol, ctol, extra=""):
    ctx = make_ctx("amr2_free", device=0, extra=f"-Rtol {rtol} -Ctol {ctol} {extra}")
    ctx.obstacle_sphere((0.41, 0.52, 0.47), 0.18)
    ctx.upload("vel", _flow(ctx))
    xyz, _ = cell_centres(ctx)
    ctx.upload("pres", np.cos(3 * xyz[:, 0]) * np.sin(2 * xyz[:, 2]))
    return ctx


def _leaves(ctx):
    level, index, _ = ctx.blocks()
    return np.column_stack([level, index]).astype(np.int32)


@pytest.mark.parametrize("extra", ["", "-levelMaxVorticity 1"])
def test_indicator_matches_oracle(extra):
    ctx = _setup(1.0, 0.1, extra)
    m = oracle_mesh(ctx)
    got = ctx.adapt_indicator()
    lmv = ctx.cfg.level_max_vorticity if ctx.cfg.level_max_vorticity > 0 else ctx.cfg.level_max
    ref = m.adapt_indicator(ctx.download("vel"), ctx.download("chi"), ctx.cfg.level_max, lmv, 1.0, 0.1)
    iface = ref == 1e10
    assert 0 < iface.sum() < m.nb
    assert np.array_equal(got == 1e10, iface)
    assert np.abs(got - ref)[~iface].max() <= 1e-12 * np.abs(ref[~iface]).max()
    assert (ref[~iface] > 0).any()


def test_adapt_mesh_matches_oracle():
    probe = _setup(1.0, 0.1)
    ind = probe.adapt_indicator()
    vals = np.sort(ind[ind < 1e10])
    rtol, ctol = float(vals[int(0.7 * len(vals))]), float(vals[int(0.3 * len(vals))])
    ctx = _setup(rtol, ctol)
    m0 = oracle_mesh(ctx)
    vel0, pres0 = ctx.download("vel"), ctx.download("pres")
    ref_leaves = m0.adapt_leaves(ctx.adapt_indicator(), rtol, ctol)
    assert ctx.adapt_mesh()
    got = _leaves(ctx)
    assert sorted(map(tuple, got)) == sorted(map(tuple, ref_leaves))
    levels0, levels1 = m0.level, got[:, 0]
    assert levels1.max() > levels0.max() or len(got) != m0.nb
    m1 = oracle_mesh(ctx)
    vref = m0.adapt_transfer(m1, vel0, 3, True)
    pref = m0.adapt_transfer(m1, pres0, 1, False)
    v, p = ctx.download("vel"), ctx.download("pres")
    assert np.abs(v - vref).max() <= 1e-14 * np.abs(vref).max()
    assert np.abs(p - pref).max() <= 1e-14 * np.abs(pref).max()
    # the body is on the new mesh: chi as the oracle creates it there
    ob = m1.create_obstacle("sphere", (0.41, 0.52, 0.47), 0.18)
    assert np.array_equal(ctx.download("chi"), ob["chi"])
    assert np.all(ctx.download("lhs") == 0.0)


def test_consecutive_adaptations_match_oracle():
    # refine (new storage), compress with the flow scaled down (the storage
    # the first adaptation sized: each field's other buffer, the other table
    # set), refine again (within that storage); every transfer compared with
    # the oracle's.  No body: its interface marks would keep blocks refined.
    def setup(rtol, ctol):
        ctx = make_ctx("amr2_free", device=0, extra=f"-Rtol {rtol} -Ctol {ctol}")
        ctx.upload("vel", _flow(ctx))
        xyz, _ = cell_centres(ctx)
        ctx.upload("pres", np.cos(3 * xyz[:, 0]) * np.sin(2 * xyz[:, 2]))
        return ctx
    vals = np.sort(setup(1.0, 0.1).adapt_indicator())
    rtol, ctol = float(vals[int(0.6 * len(vals))]), float(vals[int(0.4 * len(vals))])
    ctx = setup(rtol, ctol)
    sizes = [ctx.nb]
    for scale in (1.0, 0.01, 1.0):
        ctx.upload("vel", _flow(ctx) * scale)
        m0 = oracle_mesh(ctx)
        vel0, pres0 = ctx.download("vel"), ctx.download("pres")
        ref_leaves = m0.adapt_leaves(ctx.adapt_indicator(), rtol, ctol)
        assert ctx.adapt_mesh()
        got = _leaves(ctx)
        assert sorted(map(tuple, got)) == sorted(map(tuple, ref_leaves))
        m1 = oracle_mesh(ctx)
        vref = m0.adapt_transfer(m1, vel0, 3, True)
        pref = m0.adapt_transfer(m1, pres0, 1, False)
        assert np.abs(ctx.download("vel") - vref).max() <= 1e-14 * np.abs(vref).max()
        assert np.abs(ctx.download("pres") - pref).max() <= 1e-14 * np.abs(pref).max()
        assert np.all(ctx.download("lhs") == 0.0)
        sizes.append(ctx.nb)
    print("blocks through the adaptations:", sizes)
    assert sizes[1] > sizes[0] and sizes[2] < sizes[1] and sizes[3] > sizes[2]
    # a step on the last mesh
    dt, rc, st = ctx.step(1)
    assert rc >= 0, st


def _sphere_run(steps):
    from cup3d_b200.workloads import SPHERE_BODY, SPHERE_FLAGS
    ctx = cup.Context(cup.config(SPHERE_FLAGS + " -levelStart 3 -Rtol 1 -Ctol 0.1 -stepGraph 0", device=0))
    ctx.set_mesh_uniform()
    assert ctx.nb == 32 * 16 * 16
    ctx.obstacle_sphere(**SPHERE_BODY)
    meshes = []
    for _ in range(ctx.cfg.level_max):  # initialGridRefinement with a static body
        ctx.adapt_mesh()
    meshes.append(_leaves(ctx))
    for step in range(steps):
        if step % 20 == 0 or step < 10:
            if ctx.adapt_mesh():
                meshes.append(_leaves(ctx))
        dt, rc, st = ctx.step(step)
        assert rc >= 0 and st["status"] == 1, (step, st)
    return ctx, meshes


def test_sphere_flow_adapts_deterministically():
    a, ma = _sphere_run(25)
    b, mb = _sphere_run(25)
    assert len(ma) == len(mb) and all(np.array_equal(x, y) for x, y in zip(ma, mb))
    assert np.array_equal(a.download("vel"), b.download("vel"))
    # far from the body the mesh has coarsened; at the body it is at the finest level
    final = ma[-1]
    assert final[:, 0].min() == 0 and final[:, 0].max() == 3
    assert len(final) < 32 * 16 * 16
