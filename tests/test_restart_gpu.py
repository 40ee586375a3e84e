"""Restart files (cup_write_restart / cup_read_restart; Simulation::serialize
and deserialize, SimulationData.cpp:200-297, Obstacle.cpp:443-504):

* a run with a moving, rotating ellipsoid (BDF2 pose history) and a free
  sphere is saved after three steps, restored into a fresh context and stepped
  on: velocity, pressure, chi and the body's kinematics equal those of the
  uninterrupted run bit for bit (the property the reference's own restart
  comment asks for);
* field.restart and shape_0.restart carry the reference's keys in its order.
"""
import numpy as np
import pytest

from tests.meshes import make_ctx

pytestmark = pytest.mark.gpu

FLAGS = "-poissonTol 0 -poissonTolRel 1e-8 -nu 0.01 -CFL 0.3 -rampup 0 -advection weno5 -uinfy 0.05"


def _start(body):
    ctx = make_ctx("amr2_free", device=0, extra=FLAGS)
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    ctx.upload("vel", np.concatenate([np.sin(2 * x) * np.cos(3 * y), 0.5 * np.cos(x) * np.sin(2 * z), 0.3 * np.sin(y + z)]))
    if body == "ellipsoid":
        q = np.array([0.9, 0.1, 0.3, 0.3])
        ctx.obstacle_ellipsoid((0.45, 0.5, 0.5), (0.2, 0.1, 0.08), q / np.linalg.norm(q), vel=(2.0, -1.0, 0.5),
                               omega=(4.0, -2.0, 1.0), on_device=True)
    else:
        ctx.obstacle_sphere((0.5, 0.45, 0.55), 0.12)
        ctx.obstacle_free((1, 1, 0), (0, 0, 1))
    return ctx


def _state(ctx):
    return [ctx.download("vel"), ctx.download("pres"), ctx.download("chi"), ctx.get_obstacle()[3]]


@pytest.mark.parametrize("body", ["ellipsoid", "free_sphere"])
def test_restarted_run_continues_bit_for_bit(body, tmp_path):
    a = _start(body)
    t = 0.0
    for step in range(3):
        dt, rc, _ = a.step(step)
        assert rc >= 0
        t += dt
    a.write_restart(tmp_path, 3, t)
    b = make_ctx("amr2_free", device=0, extra=FLAGS)
    assert b.read_restart(tmp_path, 3) == t
    for x, y in zip(_state(a), _state(b)):
        assert np.array_equal(x, y)
    for step in range(3, 6):
        (dta, rca, sta), (dtb, rcb, stb) = a.step(step), b.step(step)
        assert dta == dtb and rca == rcb and sta["iterations"] == stb["iterations"], step
        for x, y in zip(_state(a), _state(b)):
            assert np.array_equal(x, y), step


def test_restart_text_files_follow_the_reference_keys(tmp_path):
    a = _start("ellipsoid")
    a.step(0)
    a.write_restart(tmp_path, 1, 0.25)
    field = (tmp_path / "field.restart").read_text().split("\n")
    assert [ln.split(":")[0] for ln in field[:6]] == ["time", "stepid", "uinfx", "uinfy", "uinfz", "dt"]
    assert field[1] == "stepid: 1" and float(field[3].split()[1]) == 0.05
    shape = [ln.split(":")[0] for ln in (tmp_path / "shape_0.restart").read_text().split("\n")[:26]]
    assert shape == (["x", "y", "z", "xAbs", "yAbs", "zAbs"] + [f"quat_{i}" for i in range(4)] +
                     ["u_x", "u_y", "u_z", "omega_x", "omega_y", "omega_z"] +
                     [f"old_position_{i}" for i in range(3)] + [f"old_absPos_{i}" for i in range(3)] +
                     [f"old_quaternion_{i}" for i in range(4)])
    assert (tmp_path / "restart_000000001.cupf").stat().st_size == 8 + 4 + 16 * a.nb + 32 * 512 * a.nb + 24


def test_restart_without_fix_frame_keys_restores(tmp_path):
    # shape_0.restart files written before the fix_frame_* keys existed: the
    # body restores with no axis fixed, and the run continues as before
    a = _start("ellipsoid")
    t = 0.0
    for step in range(2):
        dt, rc, _ = a.step(step)
        t += dt
    a.write_restart(tmp_path, 2, t)
    shape = tmp_path / "shape_0.restart"
    lines = shape.read_text().split("\n")
    assert any(ln.startswith("fix_frame_") for ln in lines)
    shape.write_text("\n".join(ln for ln in lines if not ln.startswith("fix_frame_")))
    b = make_ctx("amr2_free", device=0, extra=FLAGS)
    assert b.read_restart(tmp_path, 2) == t
    for step in range(2, 4):
        (dta, _, _), (dtb, _, _) = a.step(step), b.step(step)
        assert dta == dtb
        for x, y in zip(_state(a), _state(b)):
            assert np.array_equal(x, y), step
