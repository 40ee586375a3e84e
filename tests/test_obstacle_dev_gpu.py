"""Obstacle creation on the device (cup_obstacle_sphere_dev /
cup_obstacle_ellipsoid_dev) against the host creation (obstacles.cpp, the
restatement of Sphere.cpp / ObstaclesCreate.cpp:18-121):

* slot list, chi, udef and the grid chi field bit for bit; centre of mass
  within 1e-14 of the domain size (the moments are summed in another order);
* on the sphere mesh (2340 blocks, four levels), on AMR test meshes with a
  rotated ellipsoid, with a body that leaves no cell on the mesh, and with a
  body cut by the domain boundary;
* a time step after device creation equals the one after host creation:
  velocity and pressure bit for bit (the near-body flags and udef layout the
  kernels read; the body does not rotate, so the centre of mass does not
  enter the velocity), force and torque within 1e-12 of their size (the
  torque arm uses the centre of mass); the same for a batch built from
  device-created bodies.
"""
import numpy as np
import pytest

import cup3d_b200 as cup
from tests.meshes import make_ctx

pytestmark = pytest.mark.gpu


def _obstacle_state(ctx):
    slot, chi, udef, kin = ctx.get_obstacle()
    return slot, chi, udef, kin, ctx.download("chi")


def _assert_same(a, b, extent):
    slot_a, chi_a, udef_a, kin_a, g_a = a
    slot_b, chi_b, udef_b, kin_b, g_b = b
    assert np.array_equal(slot_a, slot_b)
    assert np.array_equal(chi_a, chi_b)
    assert np.array_equal(udef_a, udef_b)
    assert np.array_equal(g_a, g_b)
    assert np.abs(kin_a[:3] - kin_b[:3]).max() <= 1e-14 * extent
    assert np.array_equal(kin_a[3:], kin_b[3:])


def test_sphere_on_the_sphere_mesh():
    from cup3d_b200.workloads import SPHERE_BODY, make_sphere_ctx
    ctx = make_sphere_ctx(0)
    host = _obstacle_state(ctx)
    assert (host[0] >= 0).sum() >= 8
    ctx.obstacle_sphere(**SPHERE_BODY, on_device=True)
    _assert_same(host, _obstacle_state(ctx), 4.0)


@pytest.mark.parametrize("name", ["amr2_free", "amr3_mixed", "amr3_periodic"])
def test_ellipsoid_on_amr_meshes(name):
    ctx = make_ctx(name, device=0)
    q = np.array([0.9, 0.1, 0.3, 0.3])
    q /= np.linalg.norm(q)
    args = dict(center=(0.6, 0.45, 0.5), axes=(0.2, 0.1, 0.08), quat=q, vel=(0.1, 0.02, 0.0), omega=(0.0, 0.3, 0.1))
    ctx.obstacle_ellipsoid(**args)
    host = _obstacle_state(ctx)
    assert (host[0] >= 0).sum() > 0
    ctx.obstacle_ellipsoid(**args, on_device=True)
    _assert_same(host, _obstacle_state(ctx), 1.0)


def test_body_off_the_mesh_and_body_cut_by_the_boundary():
    ctx = make_ctx("amr2_free", device=0)
    ctx.obstacle_sphere((5.0, 5.0, 5.0), 0.1, on_device=True)
    slot, chi, _, _ = ctx.get_obstacle()
    assert (slot < 0).all() and chi.size == 0
    assert np.abs(ctx.download("chi")).max() == 0.0
    ctx.obstacle_sphere((0.02, 0.5, 0.5), 0.15)
    host = _obstacle_state(ctx)
    ctx.obstacle_sphere((0.02, 0.5, 0.5), 0.15, on_device=True)
    _assert_same(host, _obstacle_state(ctx), 1.0)


def _stepped(on_device):
    flags = "-poissonTol 0 -poissonTolRel 1e-8 -nu 0.01 -CFL 0.3 -rampup 0 -advection weno5 -stepGraph 0"
    ctx = make_ctx("amr2_free", device=0, extra=flags)
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    ctx.upload("vel", np.concatenate([np.sin(2 * x) * np.cos(3 * y), 0.5 * np.cos(x) * np.sin(2 * z), 0.3 * np.sin(y + z)]))
    ctx.obstacle_sphere((0.5, 0.45, 0.55), 0.15, vel=(0.1, 0.0, 0.0), on_device=on_device)
    return ctx


def _close(f0, f1):
    f0, f1 = np.asarray(f0), np.asarray(f1)
    return np.abs(f0 - f1).max() <= 1e-12 * max(np.abs(f0).max(), 1e-300)


def test_step_after_device_creation_equals_step_after_host_creation():
    a, b = _stepped(False), _stepped(True)
    for step in range(2):
        outs = []
        for ctx in (a, b):
            dt = ctx.compute_dt(step)
            ctx.advect_diffuse(dt)
            f = ctx.penalize(dt)
            ctx.pressure_project(dt, step)
            outs.append((dt, f, ctx.download("vel"), ctx.download("pres")))
        (dt0, f0, u0, p0), (dt1, f1, u1, p1) = outs
        assert dt0 == dt1 and _close(f0, f1), step
        assert np.array_equal(u0, u1) and np.array_equal(p0, p1), step


def test_batch_of_device_created_bodies():
    batches = [cup.Batch([_stepped(dev), _stepped(dev)]) for dev in (False, True)]
    for step in range(2):
        (rc0, dt0, f0, _), (rc1, dt1, f1, _) = (bt.step(step) for bt in batches)
        assert rc0 == rc1 == 0 and np.array_equal(dt0, dt1), step
        assert all(_close(a, b) for a, b in zip(f0, f1)), step
        assert np.array_equal(batches[0].download("vel"), batches[1].download("vel")), step
