"""ComputeDissipation on the device (cup_compute_dissipation) against the
oracle's restatement (ComputeDissipation.cpp:17-109): the 20 diagnostics on
AMR meshes with coarse-fine faces, walls and periodic faces, with a body's chi
weighting the power terms; each within 1e-11 of the largest term of its kind
(the sums run in another order).  On the Taylor-Green field the kinetic
energy is (2 pi)^3 / 8."""
import numpy as np
import pytest

from tests.meshes import make_ctx, oracle_mesh

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["amr2_free", "amr3_mixed", "amr3_periodic"])
def test_dissipation_matches_oracle(name):
    ctx = make_ctx(name, device=0, extra="-nu 0.003")
    m = oracle_mesh(ctx)
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    vel = np.concatenate([np.sin(2 * x) * np.cos(3 * y), 0.5 * np.cos(x) * np.sin(2 * z), 0.3 * np.sin(y + z) + x * y])
    pres = np.cos(x + 2 * y) * np.sin(z)
    ctx.upload("vel", vel)
    ctx.upload("pres", pres)
    ctx.obstacle_sphere((0.5, 0.45, 0.55), 0.2)
    chi = ctx.download("chi")
    dev = ctx.dissipation()
    ref = m.dissipation(vel, pres, chi, 0.003)
    # groups of terms of one kind share a scale
    for sl in (slice(0, 3), slice(3, 6), slice(6, 9), slice(9, 12), slice(12, 15), slice(15, 16), slice(16, 17),
               slice(17, 18), slice(18, 19), slice(19, 20)):
        scale = max(np.abs(ref[sl]).max(), 1e-300)
        assert np.abs(dev[sl] - ref[sl]).max() <= 1e-11 * scale, (sl, dev[sl], ref[sl])


def test_taylor_green_kinetic_energy():
    ctx = make_ctx("tgv32", device=0)
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    ctx.upload("vel", np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), 0 * x]))
    q = ctx.dissipation()
    assert abs(q[18] - np.pi ** 3) <= 1e-12 * np.pi ** 3
    assert np.abs(q[6:9]).max() <= 1e-12
