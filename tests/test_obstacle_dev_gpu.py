"""Obstacle creation on the host (cup_obstacle_sphere / cup_obstacle_ellipsoid)
and on the device (cup_obstacle_sphere_dev / cup_obstacle_ellipsoid_dev):

* both against the oracle's CreateObstacles (ObstaclesCreate.cpp:18-148,
  Sphere.cpp:19-51, Ellipsoid.cpp:22-300): slot list, chi and grid chi bit for
  bit, centre of mass to rounding, on the benchmarked sphere mesh, AMR meshes
  with a rotated ellipsoid and the reference's own sphere moment case
  (tests/python/test_obstacles.py:7-74) with its tolerances;
* device against host:

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


def _assert_matches_oracle(ctx, kind, centre, shape, quat=(1.0, 0.0, 0.0, 0.0), extent=1.0):
    """The context's obstacle (slot list, chi, zero udef, grid chi, centre of
    mass) against the oracle's CreateObstacles on the same mesh."""
    from tests.meshes import oracle_mesh
    ref = oracle_mesh(ctx).create_obstacle(kind, centre, shape, quat)
    slot, chi, udef, kin, grid = _obstacle_state(ctx)
    assert np.array_equal(slot, ref["slot"])
    assert np.array_equal(chi, ref["chi_o"])
    assert np.array_equal(grid, ref["chi"])
    assert np.all(udef == 0.0)
    assert np.abs(kin[:3] - ref["com"]).max() <= 1e-14 * extent


@pytest.mark.parametrize("on_device", [False, True])
def test_sphere_creation_matches_oracle(on_device):
    # the benchmarked sphere on its 2340-block, four-level mesh
    from cup3d_b200.workloads import SPHERE_BODY, make_sphere_ctx
    ctx = make_sphere_ctx(0)
    ctx.obstacle_sphere(**SPHERE_BODY, on_device=on_device)
    _assert_matches_oracle(ctx, "sphere", SPHERE_BODY["center"], SPHERE_BODY["radius"], extent=4.0)


@pytest.mark.parametrize("on_device", [False, True])
@pytest.mark.parametrize("name", ["amr2_free", "amr3_mixed", "amr3_periodic"])
def test_ellipsoid_creation_matches_oracle(name, on_device):
    ctx = make_ctx(name, device=0)
    q = np.array([0.9, 0.1, 0.3, 0.3])
    q /= np.linalg.norm(q)
    ctx.obstacle_ellipsoid((0.6, 0.45, 0.5), (0.2, 0.1, 0.08), q, on_device=on_device)
    _assert_matches_oracle(ctx, "ellipsoid", (0.6, 0.45, 0.5), (0.2, 0.1, 0.08), q)


@pytest.mark.parametrize("on_device", [False, True])
def test_reference_sphere_moment_case(on_device):
    # tests/python/test_obstacles.py:7-74: Sphere L=3 at (3.125, 2.5, 2.5) on
    # 8x4x4 blocks, extent 10, levelMax 2, chi on the level-1 grid; the
    # product's chi equals the oracle's and meets the reference's tolerances
    from tests.test_obstacle_moments import BPD, CTR, R, _moments, _uniform_level1
    level, index = _uniform_level1()
    ctx = cup.Context(cup.config(f"-bpdx {BPD[0]} -bpdy {BPD[1]} -bpdz {BPD[2]} -levelMax 2 -extent 10",
                                 device=0))
    ctx.set_mesh(level, index)
    ctx.obstacle_sphere(CTR, R, on_device=on_device)
    _assert_matches_oracle(ctx, "sphere", CTR, R, extent=10.0)
    from tests.meshes import oracle_mesh
    mo = _moments(oracle_mesh(ctx), ctx.download("chi"))
    assert round(mo["M"] - 4 / 3 * np.pi * R ** 3, 3) == 0
    for k in ("Mx", "My", "Mz", "Mxy", "Myz", "Mzx"):
        assert abs(mo[k]) < 1e-9, k
    for k in ("Mxx", "Myy", "Mzz"):
        assert round(mo[k] - 4 / 15 * np.pi * R ** 5, 1) == 0, k


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


def _pose_update(b, uinf, step, coef, dt, step_2nd_start=2):
    """Obstacle::update (Obstacle.cpp:306-368) restated: Euler for the first
    step_2nd_start steps, BDF2 with coefU after, quaternion renormalised."""
    w, q = b["omega"], b["quat"]
    dqdt = [0.5 * (-w[0] * q[1] - w[1] * q[2] - w[2] * q[3]),
            0.5 * (+w[0] * q[0] + w[1] * q[3] - w[2] * q[2]),
            0.5 * (-w[0] * q[3] + w[1] * q[0] + w[2] * q[1]),
            0.5 * (+w[0] * q[2] - w[1] * q[1] + w[2] * q[0])]
    if step < step_2nd_start:
        b["old_pos"], b["old_quat"] = list(b["pos"]), list(q)
        b["pos"] = [b["pos"][d] + dt * (b["vel"][d] + uinf[d]) for d in range(3)]
        q = [q[i] + dt * dqdt[i] for i in range(4)]
    else:
        aux = 1.0 / coef[0]
        tp, tq = list(b["pos"]), list(q)
        b["pos"] = [aux * (dt * (b["vel"][d] + uinf[d]) + (-coef[1] * b["pos"][d] - coef[2] * b["old_pos"][d]))
                    for d in range(3)]
        q = [aux * (dt * dqdt[i] + (-coef[1] * q[i] - coef[2] * b["old_quat"][i])) for i in range(4)]
        b["old_pos"], b["old_quat"] = tp, tq
    inv = 1.0 / np.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    b["quat"] = [x * inv for x in q]


@pytest.mark.parametrize("on_device", [True, False])
def test_moving_body_is_recreated_at_its_integrated_pose(on_device):
    # CreateObstacles every step: the pose integrated by Obstacle::update with
    # the step's dt (Euler in steps 0-1, BDF2 with the default coefU in step
    # 2, with coefU of the last two dts in step 3), then chi at that pose:
    # bit for bit the host creation at the pose restated here
    flags = "-poissonTol 0 -poissonTolRel 1e-6 -nu 0.01 -CFL 0.3 -rampup 0 -advection weno5"
    ctx = make_ctx("amr2_free", device=0, extra=flags)
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    ctx.upload("vel", np.concatenate([np.sin(2 * x) * np.cos(3 * y), 0.5 * np.cos(x) * np.sin(2 * z), 0.3 * np.sin(y + z)]))
    q0 = np.array([0.9, 0.1, 0.3, 0.3])
    q0 = list(q0 / np.linalg.norm(q0))
    body = dict(pos=[0.45, 0.5, 0.5], quat=q0, old_pos=[0.45, 0.5, 0.5], old_quat=list(q0), vel=[3.0, -1.0, 0.5],
                omega=[5.0, -3.0, 2.0])
    axes = (0.2, 0.1, 0.08)
    ctx.obstacle_ellipsoid(body["pos"], axes, body["quat"], vel=body["vel"], omega=body["omega"], on_device=on_device)
    chi0 = ctx.download("chi")
    coef, dt_prev = [1.5, -2.0, 0.5], 0.0
    for step in range(4):
        dt, rc, st = ctx.step(step)
        assert rc >= 0 and st["status"] == 1, (step, rc, st)
        if step > 2 and dt_prev > 0:
            a, b = dt_prev, dt
            c1, c2 = -(a + b) / (a * b), b / (a + b) / a
            coef = [-b * (c1 + c2), b * c1, b * c2]
        dt_prev = dt
        _pose_update(body, (0.0, 0.0, 0.0), step, coef, dt)
    ref = make_ctx("amr2_free", device=0)
    ref.obstacle_ellipsoid(body["pos"], axes, body["quat"], vel=body["vel"], omega=body["omega"])
    slot, chi, _, kin = ctx.get_obstacle()
    slot_r, chi_r, _, kin_r = ref.get_obstacle()
    assert np.abs(ctx.download("chi") - chi0).max() > 0.5  # the body has moved by more than a cell
    assert np.array_equal(slot, slot_r) and np.array_equal(chi, chi_r)
    assert np.abs(kin[:3] - kin_r[:3]).max() <= 1e-14
    assert np.array_equal(ctx.download("chi"), ref.download("chi"))


def test_static_and_comoving_bodies_stay():
    # -StaticObstacles 1, or a body whose velocity + uinf and angular velocity
    # are zero (the sphere in its own frame): chi is never re-created
    for flags, vel, uinf in (("-StaticObstacles 1", (0.2, 0.0, 0.0), 0.0), ("", (0.1, 0.0, 0.0), -0.1)):
        ctx = make_ctx("amr2_free", device=0, extra=f"-rampup 0 -uinfx {uinf} {flags}")
        ctx.obstacle_sphere((0.5, 0.5, 0.5), 0.15, vel=vel, on_device=True)
        before = _obstacle_state(ctx)
        for step in range(3):
            _, rc, _ = ctx.step(step)
            assert rc >= 0
        _assert_same(before, _obstacle_state(ctx), 1.0)


def _momenta_restated(ctx, lam, dt, implicit):
    """KernelIntegrateFluidMomenta + kernelFinalizeObstacleVel
    (ObstaclesUpdate.cpp:25-186) in numpy: the 29 integrals of the body."""
    slot, chi, udef, kin = ctx.get_obstacle()
    xyz, hh = ctx.cell_centres()
    u = ctx.download("vel").reshape(3, -1)
    ns = len(chi) // 512
    M = np.zeros(29)
    for b in np.where(slot >= 0)[0]:
        s = slot[b]
        X = chi[s * 512:(s + 1) * 512]
        m = X > 0
        if not m.any():
            continue
        p = (xyz[b * 512:(b + 1) * 512][m] - kin[:3]).T
        dv = hh[b * 512] ** 3
        Xd = X[m] * dv
        ub = u[:, b * 512:(b + 1) * 512][:, m]
        M[0] += Xd.sum()
        M[1:4] += (Xd * ub).sum(1)
        M[4:7] += (Xd * np.cross(p.T, ub.T).T).sum(1)
        M[7] += (Xd * (p[1] ** 2 + p[2] ** 2)).sum()
        M[8] += (Xd * (p[0] ** 2 + p[2] ** 2)).sum()
        M[9] += (Xd * (p[0] ** 2 + p[1] ** 2)).sum()
        M[10] -= (Xd * p[0] * p[1]).sum()
        M[11] -= (Xd * p[0] * p[2]).sum()
        M[12] -= (Xd * p[1] * p[2]).sum()
        if implicit:
            X1 = (X[m] > 0.5).astype(float)
            pf = dv * lam * dt * X1 / (1 + X1 * lam * dt)
            du = ub - np.stack([udef[(d * ns + s) * 512:(d * ns + s + 1) * 512][m] for d in range(3)])
            M[13] += pf.sum()
            M[14:17] += (pf * p).sum(1)
            M[17] += (pf * (p[1] ** 2 + p[2] ** 2)).sum()
            M[18] += (pf * (p[0] ** 2 + p[2] ** 2)).sum()
            M[19] += (pf * (p[0] ** 2 + p[1] ** 2)).sum()
            M[20] -= (pf * p[0] * p[1]).sum()
            M[21] -= (pf * p[0] * p[2]).sum()
            M[22] -= (pf * p[1] * p[2]).sum()
            M[23:26] += (pf * du).sum(1)
            M[26:29] += (pf * np.cross(p.T, du.T).T).sum(1)
    return M, kin


def _velocities_restated(M, kin, implicit, free_t, free_r, dt):
    """Obstacle::computeVelocities (Obstacle.cpp:143-269) with numpy's solver."""
    if implicit:
        pm, cm, J, lm, am = M[13], M[14:17], M[17:23], M[23:26], M[26:29]
    else:
        pm, cm, J, lm, am = M[0], np.zeros(3), M[7:13], M[1:4], M[4:7]
    A = np.array([[pm, 0, 0, 0, cm[2], -cm[1]], [0, pm, 0, -cm[2], 0, cm[0]], [0, 0, pm, cm[1], -cm[0], 0],
                  [0, -cm[2], cm[1], J[0], J[3], J[4]], [cm[2], 0, -cm[0], J[3], J[1], J[5]],
                  [-cm[1], cm[0], 0, J[4], J[5], J[2]]], dtype=float)
    rhs = np.concatenate([lm, am]).astype(float)
    vel0, om0 = kin[3:6], kin[6:9]
    for d in range(3):
        if not free_t[d]:
            A[d, [j for j in range(6) if j != d]] = 0
            rhs[d] = pm * vel0[d]
        if not free_r[d]:
            r = 3 + d
            A[r, [j for j in range(6) if j != r]] = 0
            rhs[r] = A[r, r] * om0[d]
    x = np.linalg.solve(A, rhs)
    vel = np.where(free_t, x[:3], vel0)
    om = np.where(free_r, x[3:], om0)
    Jm = M[7:13]
    dAv = (x[3:] - om0) / dt
    torque = np.array([Jm[0] * dAv[0] + Jm[3] * dAv[1] + Jm[4] * dAv[2], Jm[3] * dAv[0] + Jm[1] * dAv[1] + Jm[5] * dAv[2],
                       Jm[4] * dAv[0] + Jm[5] * dAv[1] + Jm[2] * dAv[2]])
    return vel, om, M[0] * (x[:3] - vel0) / dt, torque


@pytest.mark.parametrize("implicit,free_t,free_r", [(1, (1, 1, 1), (1, 1, 1)), (1, (1, 0, 1), (0, 0, 1)),
                                                    (0, (1, 1, 1), (1, 1, 1))])
def test_free_body_velocities_match_restated_momentum_integration(implicit, free_t, free_r):
    lam, dt = 1e6, 2e-3
    ctx = make_ctx("amr3_periodic", device=0, extra=f"-lambda {lam} -implicitPenalization {implicit}")
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    ctx.upload("vel", np.concatenate([np.sin(2 * np.pi * y), 0.5 * np.cos(2 * np.pi * z), 0.3 * np.sin(2 * np.pi * x)]))
    q = np.array([0.8, 0.2, -0.4, 0.4])
    ctx.obstacle_ellipsoid((0.55, 0.45, 0.5), (0.2, 0.12, 0.08), q / np.linalg.norm(q), vel=(0.1, -0.05, 0.02),
                           omega=(0.3, 0.0, -0.2), on_device=True)
    ctx.obstacle_free(free_t, free_r)
    M, kin = _momenta_restated(ctx, lam, dt, implicit)
    vel, om, force, torque = _velocities_restated(M, kin, implicit, np.array(free_t, bool), np.array(free_r, bool), dt)
    out = ctx.update_obstacles(dt)
    for key, ref in (("vel", vel), ("omega", om), ("force", force), ("torque", torque)):
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(out[key] - ref).max() <= 1e-10 * scale, (key, out[key], ref)
    assert np.array_equal(ctx.get_obstacle()[3][3:6], out["vel"])


def test_free_body_takes_the_uniform_flow_and_moves_with_it():
    # a free sphere in uniform flow: its velocity becomes the flow's and
    # cup_step carries it along (UpdateObstacles, then Obstacle::update)
    ctx = make_ctx("amr2_free", device=0, extra="-rampup 0 -CFL 0.3 -nu 0.001")
    n = ctx.nb * 512
    ctx.upload("vel", np.concatenate([np.full(n, 0.3), np.zeros(n), np.zeros(n)]))
    ctx.obstacle_sphere((0.4, 0.5, 0.5), 0.12, on_device=True)
    ctx.obstacle_free()
    out = ctx.update_obstacles(1e-3)
    assert abs(out["vel"][0] - 0.3) <= 1e-12 and np.abs(out["vel"][1:]).max() <= 1e-12
    assert np.abs(out["omega"]).max() <= 1e-10
    chi0 = ctx.download("chi")
    for step in range(3):
        _, rc, _ = ctx.step(step)
        assert rc >= 0
    assert np.abs(ctx.download("chi") - chi0).max() > 0.1


def test_frame_follows_a_free_body():
    # a sphere free along x in a uniform flow u = 0.3, with the frame of
    # reference fixed on it along x (bFixFrameOfRef): UpdateObstacles gives it
    # the flow's velocity, the next step sets uinf_x = -0.3 (updateUinf), and
    # the body stays where it is on the grid.  A periodic domain: on a
    # free-space box the projection removes a uniform through-flow.
    ctx = make_ctx("amr3_periodic", device=0, extra="-rampup 0 -CFL 0.3 -nu 0.001")
    n = ctx.nb * 512
    ctx.upload("vel", np.concatenate([np.full(n, 0.3), np.zeros(n), np.zeros(n)]))
    ctx.obstacle_sphere((0.4, 0.5, 0.5), 0.12, on_device=True)
    ctx.obstacle_free((1, 0, 0), (0, 0, 0))
    ctx.obstacle_fix_frame((1, 0, 0))
    assert np.array_equal(ctx.uinf(), [-0.0, 0.0, 0.0])
    chi0 = ctx.download("chi")
    for step in range(3):
        _, rc, _ = ctx.step(step)
        assert rc >= 0
    vel = ctx.get_obstacle()[3][3:6]
    assert abs(vel[0] - 0.3) <= 1e-3 and vel[1] == 0.0 and vel[2] == 0.0
    u = ctx.uinf()
    assert u[1] == 0.0 and u[2] == 0.0 and abs(u[0] + 0.3) <= 1e-3
    # the pose moved only by the difference between the velocity of one step and
    # the frame velocity set at the start of the next (at most the drift of one
    # step's velocity change), far below a cell
    assert np.abs(ctx.download("chi") - chi0).max() < 0.05
