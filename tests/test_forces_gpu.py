"""Surface forces (cup_compute_forces, ComputeForces of FluidSolidForces.cpp)
against the oracle's restatement on the same fields: a fixed sphere and a
rotated ellipsoid in the sphere workload's flow after a few time steps (AMR
mesh, WENO5, penalization).  The surface points, the one-sided velocity
gradients and the per-block sums are the same arithmetic (no fused
multiply-adds on either side); the sums over the points differ in order, so
the 19 quantities agree to 1e-10 relative to the largest of their kind."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _run(body):
    import cup3d_b200 as cup
    from cup3d_b200.workloads import SPHERE_FLAGS, SPHERE_MESH
    ctx = cup.Context(cup.config(SPHERE_FLAGS + " -stepGraph 0", device=0))
    ctx.set_mesh_sphere_wake(**SPHERE_MESH)
    c = np.array(SPHERE_MESH["center"])
    # the body moves at 0.1 against the frame's -0.1: at rest in the frame,
    # in a flow of 0.1 past it
    v = (0.1, 0.0, 0.0)
    if body == "sphere":
        ctx.obstacle_sphere(c, 0.0625, vel=v)
    else:
        q = np.array([0.9, 0.3, -0.2, 0.25]); q /= np.linalg.norm(q)
        ctx.obstacle_ellipsoid(c, (0.08, 0.05, 0.04), q, vel=v)
    for step in range(3):
        dt, rc, st = ctx.step(step)
        assert rc == 0
    f = ctx.compute_forces()
    level, index, _ = ctx.blocks()
    m = oracle.Mesh(level, index, [4, 2, 2], 4, [0, 0, 0], 4.0)
    slot, chi_o, udef_o, kin = ctx.get_obstacle()
    bos = np.argsort(np.where(slot >= 0, slot, 1 << 30))[:int((slot >= 0).sum())]
    if body == "sphere":
        nrm = m.obstacle_surface("sphere", c, 0.0625, bos, chi_o)
    else:
        nrm = m.obstacle_surface("ellipsoid", c, (0.08, 0.05, 0.04), bos, chi_o, quat=q)
    ref, bad = m.compute_forces(ctx.download("vel"), ctx.download("pres"), ctx.download("chi"), bos, nrm, udef_o,
                                ctx.cfg.nu, kin)
    return f, ref, bad


@pytest.mark.parametrize("body", ["sphere", "ellipsoid"])
def test_surface_forces_match_oracle(body):
    f, ref, bad = _run(body)
    assert bad == 0
    got = f["raw"][:19]
    print(body, "surface force", got[0:3], "pressure", got[3:6], "viscous", got[6:9], "drag", got[12])
    for a, b in ((0, 12), (12, 19)):  # vectors, then the scalar sums
        scale = np.abs(ref[a:b]).max()
        assert np.abs(got[a:b] - ref[a:b]).max() <= 1e-10 * scale, (got[a:b], ref[a:b])
    assert np.isfinite(f["raw"]).all()
    assert np.abs(got[0:3]).max() > 0 and f["drag"] > 0  # a flow past the body
