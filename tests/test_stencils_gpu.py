"""Parity of the device time-step operators (C ABI) against the CPU oracle.

Tolerances (FP64 both sides, different summation and fused-multiply-add order):
  * advection-diffusion, penalization: 1e-12 of max|u|;
  * pressure projection / full step (Poisson solved to 1e-11 relative on both
    sides): 5e-10 of max|u| for velocity, 1e-9 of max|p| for pressure; the
    difference left is the solves' convergence (the operators alone agree to 1e-12,
    see the RHS and advection tests).
"""
import numpy as np
import pytest

import oracle
from tests.meshes import cell_centres, make_ctx, oracle_mesh

pytestmark = pytest.mark.gpu


def smooth_velocity(ctx, amp=1.0):
    xyz, _ = cell_centres(ctx)
    L = ctx.cfg.extent
    k = 2 * np.pi / L
    x, y, z = xyz.T
    u = np.sin(k * x) * np.cos(k * y) * np.cos(k * z) + 0.3 * np.sin(2 * k * y + 0.4)
    v = -np.cos(k * x) * np.sin(k * y) * np.cos(k * z) + 0.2 * np.cos(k * z)
    w = 0.1 * np.sin(k * x + k * y) + 0.05 * np.cos(3 * k * z)
    return amp * np.concatenate([u, v, w])


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("scheme", [0, 1])
@pytest.mark.parametrize("name", ["tgv32", "amr2_free", "amr3_mixed"])
def test_advect_diffuse_matches_oracle(name, scheme):
    ctx = make_ctx(name, device=0, extra="-nu 0.01 -uinfx 0.1 -uinfy -0.05 -advection " +
                   ("weno5" if scheme else "upwind5"))
    m = oracle_mesh(ctx)
    vel = smooth_velocity(ctx)
    dt = 0.2 * m.hmin / np.abs(vel).max()
    ctx.upload("vel", vel)
    ctx.advect_diffuse(dt)
    got = ctx.download("vel")
    ref = m.advect_diffuse(vel, dt, 0.01, uinf=(0.1, -0.05, 0.0), scheme=scheme)
    assert rel(got, ref) < 1e-12
    assert rel(got, vel) > 1e-6  # the step did something


def _sphere_case(name="amr2_free", center=(0.41, 0.52, 0.47), r=0.18):
    ctx = make_ctx(name, device=0, extra="-nu 0.001 -lambda 1e6")
    ctx.obstacle_sphere(center, r, vel=(0.1, -0.02, 0.03), omega=(0.0, 0.5, -0.2))
    m = oracle_mesh(ctx)
    slot, chi_o, udef_o, kin = ctx.get_obstacle()
    chi = ctx.download("chi")
    return ctx, m, slot, chi_o, udef_o, kin, chi


def test_sphere_obstacle_volume():
    # like tests/python/test_obstacles.py: chi integrates to the sphere volume
    ctx, m, slot, chi_o, udef_o, kin, chi = _sphere_case()
    hh = np.repeat(m.h, 512)
    vol = np.sum(chi * hh ** 3)
    assert abs(vol - 4 / 3 * np.pi * 0.18 ** 3) < 0.02 * 4 / 3 * np.pi * 0.18 ** 3
    assert np.allclose(kin[:3], (0.41, 0.52, 0.47), atol=2e-3)


def test_penalization_matches_oracle():
    ctx, m, slot, chi_o, udef_o, kin, chi = _sphere_case()
    vel = smooth_velocity(ctx, 0.3)
    ctx.upload("vel", vel)
    dt = 1e-3
    F = ctx.penalize(dt)
    got = ctx.download("vel")
    ref, Fref = m.penalize(vel, chi, slot, chi_o, udef_o, kin, dt, lam=1e6, implicit=1)
    assert rel(got, ref) < 1e-12
    assert np.abs(F - Fref).max() <= 1e-11 * np.abs(Fref).max()


@pytest.mark.parametrize("step", [1, 5])
@pytest.mark.parametrize("name", ["tgv32", "amr3_mixed", "sphere"])
def test_pressure_project_matches_oracle(name, step):
    extra = "-poissonTol 0 -poissonTolRel 1e-11"
    if name == "sphere":
        ctx, m, slot, chi_o, udef_o, kin, chi = _sphere_case()
        ctx2 = make_ctx("amr2_free", device=0, extra=extra)
        ctx2.set_obstacle(np.where(slot >= 0)[0][np.argsort(slot[slot >= 0])], chi_o, udef_o, kin)
        ctx2.upload("chi", chi)
        ctx = ctx2
        obst = dict(chi=chi, slot=slot, chi_o=chi_o, udef_o=udef_o)
    else:
        ctx = make_ctx(name, device=0, extra=extra)
        m = oracle_mesh(ctx)
        obst = {}
    vel = smooth_velocity(ctx)
    xyz, _ = cell_centres(ctx)
    p0 = 0.1 * np.sin(xyz[:, 0] * 3.0) * np.cos(xyz[:, 1] * 2.0)
    ctx.upload("vel", vel)
    ctx.upload("pres", p0)
    dt = 0.2 * m.hmin / np.abs(vel).max()
    rc, st = ctx.pressure_project(dt, step)
    assert rc == 0 and st["status"] == 1
    got_v, got_p = ctx.download("vel"), ctx.download("pres")
    ref_v, ref_p, info = m.pressure_project(vel, p0, dt, step, tol=0.0, tol_rel=1e-11, **obst)
    assert info["converged"]
    assert rel(got_v, ref_v) < 5e-10
    assert np.abs(got_p - ref_p).max() < 1e-9 * np.abs(ref_p).max()


@pytest.mark.parametrize("step", [1, 5])
def test_split_projection_equals_fused(step):
    # PressureProjection as the reference runs it: RHS, then PoissonSolverBase::solve()
    # on sim.lhs / sim.pres (the increment), then mean, p += p_old and gradient
    # (PressureProjection.cpp:331-468): the same results as the fused call
    extra = "-poissonTol 0 -poissonTolRel 1e-11"
    outs = []
    for split in (False, True):
        ctx = make_ctx("amr3_mixed", device=0, extra=extra)
        vel = smooth_velocity(ctx)
        xyz, _ = cell_centres(ctx)
        p0 = 0.1 * np.sin(xyz[:, 0] * 3.0) * np.cos(xyz[:, 1] * 2.0)
        ctx.upload("vel", vel)
        ctx.upload("pres", p0)
        dt = 0.2 * oracle_mesh(ctx).hmin / np.abs(vel).max()
        if split:
            ctx.pressure_rhs(dt, step)
            assert np.all(ctx.download("pres") == 0.0)  # the increment starts at zero
            rc, st = ctx.poisson_solve()
            ctx.pressure_finish(dt, step)
        else:
            rc, st = ctx.pressure_project(dt, step)
        assert rc == 0 and st["status"] == 1
        outs.append((ctx.download("vel"), ctx.download("pres")))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    with pytest.raises(Exception, match="no projection open"):
        ctx.pressure_finish(1e-3, step)


def test_tgv_steps_match_oracle():
    # Taylor-Green: u = sin x cos y cos z, v = -cos x sin y cos z, w = 0 on [0,2pi]^3,
    # nu = 0.01, CFL 0.3, upwind5, FP64; Poisson converged tightly on both sides
    flags = "-nu 0.01 -CFL 0.3 -rampup 0 -poissonTol 0 -poissonTolRel 1e-11"
    ctx = make_ctx("tgv32", device=0, extra=flags)
    m = oracle_mesh(ctx)
    xyz, _ = cell_centres(ctx)
    x, y, z = xyz.T
    vel = np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), 0 * x])
    pres = np.zeros(m.n)
    ctx.upload("vel", vel)
    ref_v = vel.copy()
    for step in range(4):
        dt_gpu, rc, st = ctx.step(step)
        dt_ref = oracle.dt(m.hmin, 0.01, 0.3, m.max_u(ref_v), step, 0)
        assert abs(dt_gpu - dt_ref) <= 1e-12 * dt_ref
        ref_v = m.advect_diffuse(ref_v, dt_ref, 0.01)
        ref_v, pres, info = m.pressure_project(ref_v, pres, dt_ref, step, tol=0.0, tol_rel=1e-11)
        got = ctx.download("vel")
        assert rel(got, ref_v) < 5e-10, step
    assert rel(ctx.download("pres"), pres) < 1e-9


@pytest.mark.parametrize("step", [1, 5])
@pytest.mark.parametrize("name", ["tgv32", "amr3_mixed", "sphere"])
def test_pressure_rhs_matches_oracle(name, step):
    # KernelPressureRHS + kernelUpdateTmpV (+ KernelDivPressure for step > 2)
    # with flux correction, alone: 1e-12 of max|rhs|
    obst = {}
    if name == "sphere":
        ctx, m, slot, chi_o, udef_o, kin, chi = _sphere_case()
        obst = dict(chi=chi, slot=slot, chi_o=chi_o, udef_o=udef_o)
    else:
        ctx = make_ctx(name, device=0)
        m = oracle_mesh(ctx)
    vel = smooth_velocity(ctx)
    xyz, _ = cell_centres(ctx)
    p0 = 0.1 * np.sin(xyz[:, 0] * 3.0) * np.cos(xyz[:, 1] * 2.0)
    ctx.upload("vel", vel)
    ctx.upload("pres", p0)
    dt = 0.2 * m.hmin / np.abs(vel).max()
    ctx.pressure_rhs(dt, step)
    got = ctx.download("lhs")
    ref = m.pressure_rhs(vel, p0, dt, step, **obst)
    assert rel(got, ref) < 1e-12
