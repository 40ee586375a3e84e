"""Captured time steps (cup_step with the CFL dt and the plain solver replays
a CUDA graph of the whole step) against the same steps launched kernel by
kernel (-stepGraph 0): the same kernels in the same order, with dt computed
on the device by the host's operations, so dt, iteration counts, velocity and
pressure agree bit for bit, through the CFL ramp, both buffer parities and
the step where the p_old term switches on; new solver settings are captured
anew.
"""
import numpy as np
import pytest

from tests.meshes import make_ctx

pytestmark = pytest.mark.gpu


def _pair(name, extra):
    out = []
    for g in (1, 0):
        ctx = make_ctx(name, device=0, extra=extra + f" -stepGraph {g}")
        xyz, _ = ctx.cell_centres()
        x, y, z = xyz.T
        ctx.upload("vel", np.concatenate([np.sin(2 * x) * np.cos(y), np.cos(x) * np.sin(3 * z), 0.2 * np.sin(y + z)]))
        out.append(ctx)
    return out


@pytest.mark.parametrize("name,extra,body", [
    ("tgv32", "-nu 0.01 -CFL 0.3 -rampup 0", None),
    ("amr2_free", "-nu 0.001 -CFL 0.4 -rampup 3 -advection weno5 -StaticObstacles 1", ((0.5, 0.45, 0.55), 0.15)),
])
def test_captured_steps_match_launched_steps(name, extra, body):
    g, p = _pair(name, extra)
    if body:
        for c in (g, p):
            c.obstacle_sphere(body[0], body[1], vel=(0.1, 0.0, 0.0))
    for step in range(6):
        dt_g, rc_g, st_g = g.step(step)
        dt_p, rc_p, st_p = p.step(step)
        assert rc_g == rc_p and dt_g == dt_p, (step, dt_g, dt_p)
        assert st_g["iterations"] == st_p["iterations"] and st_g["status"] == st_p["status"], (step, st_g, st_p)
        assert np.array_equal(g.download("vel"), p.download("vel")), step
        assert np.array_equal(g.download("pres"), p.download("pres")), step


def test_captured_steps_follow_new_solver_settings():
    g, p = _pair("amr2_free", "-nu 0.001 -CFL 0.3 -rampup 0")
    for c in (g, p):
        c.step(0)
        c.set_poisson("b200", 0.0, 1e-9, 1000)
    _, _, st_g = g.step(1)
    _, _, st_p = p.step(1)
    assert st_g["iterations"] == st_p["iterations"] > 10
    assert np.array_equal(g.download("vel"), p.download("vel"))


def test_autotune_changes_only_the_launch_shape():
    # cup_autotune times launch grids on the context's own fields; the chosen
    # grids leave the stencils' results unchanged and the solver's up to its
    # summation order: two steps of a tuned and an untuned context agree to
    # within what a solve to 1e-11 allows
    extra = "-nu 0.001 -CFL 0.3 -rampup 0 -poissonTol 0 -poissonTolRel 1e-11"
    a, b = (make_ctx("amr3_periodic", device=0, extra=extra) for _ in range(2))
    for c in (a, b):
        xyz, _ = c.cell_centres()
        x, y, z = (2 * np.pi * t for t in xyz.T)
        c.upload("vel", np.concatenate([np.sin(x) * np.cos(y), np.cos(z) * np.sin(x), 0.3 * np.sin(y)]))
    choice, ms = a.autotune()
    sms = 148
    assert all(choice[k] >= 1 for k in choice), choice
    assert all(ms[k] > 0 for k in ("advect", "pressure_rhs", "grad_update", "solver")), ms
    for step in range(2):
        dta, _, sta = a.step(step)
        dtb, _, stb = b.step(step)
        assert abs(dta - dtb) <= 1e-12 * dtb
        ua, ub = a.download("vel"), b.download("vel")
        assert np.abs(ua - ub).max() <= 1e-9 * np.abs(ub).max(), step
