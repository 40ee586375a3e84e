"""The oracle and the host mesh code against the committed golden fixtures
(tests/golden/, made by tests/golden/make_golden.py).

* block order and face tables after the space-filling-curve ordering: bit-exact;
* oracle operator rows and block inverse on the sampled entries: 1e-13 relative;
* oracle solve to 1e-10: the same iteration count (the oracle's sums run in
  a fixed order for any thread count), solution within 1e-8 relative;
* Taylor-Green 32^3 steps: dt within 1e-12, velocity within 5e-10 of
  max|u| (the Poisson solve is converged to 1e-11).
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
from tests.meshes import make_ctx, oracle_mesh

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ["tgv32", "amr2_free", "amr3_mixed", "amr3_periodic"]


def load(name):
    return np.load(GOLDEN / name)


@pytest.mark.parametrize("name", CASES)
def test_mesh_order_and_faces_match_golden(name):
    g = load(f"mesh_{name}.npz")
    ctx = make_ctx(name)
    level, index, h = ctx.blocks()
    kinds, nbrs = ctx.faces()
    assert np.array_equal(level, g["level"]) and np.array_equal(index, g["index"])
    assert np.array_equal(h, g["h"])
    assert np.array_equal(kinds, g["kinds"]) and np.array_equal(nbrs, g["nbrs"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_poisson_matches_golden(name):
    g = load(f"poisson_{name}.npz")
    m = oracle_mesh(make_ctx(name))
    x = np.random.default_rng(42).standard_normal(m.n)
    idx = g["idx"]
    y = m.apply(x, mean_constraint=1)
    assert np.abs(y[idx] - g["y"]).max() <= 1e-13 * np.abs(g["y"]).max()
    assert abs(np.linalg.norm(y) - g["y_norm"]) <= 1e-13 * g["y_norm"]
    z = m.precond_pinv(x, oracle.pinv())
    assert np.abs(z[idx] - g["z"]).max() <= 1e-13 * np.abs(g["z"]).max()


@pytest.mark.parametrize("name", ["amr2_free", "amr3_mixed"])
def test_oracle_solve_matches_golden(name):
    g = load(f"poisson_{name}.npz")
    m = oracle_mesh(make_ctx(name))
    hh = np.repeat(m.h, 512)
    b = np.random.default_rng(9).standard_normal(m.n)
    b -= np.sum(b * hh ** 3) / np.sum(hh ** 3)
    xs, st = m.bicgstab_gpu(b, tol=0.0, tol_rel=1e-10)
    it = int(g["solve_iterations"])
    assert st["iterations"] == it
    assert np.abs(xs[g["idx"]] - g["x"]).max() <= 1e-8 * np.abs(g["x"]).max()


def test_oracle_tgv_steps_match_golden():
    g = load("tgv32_steps.npz")
    ctx = make_ctx("tgv32", extra="-nu 0.01 -CFL 0.3 -rampup 0")
    m = oracle_mesh(ctx)
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    vel = np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), 0 * x])
    pres = np.zeros(m.n)
    idx = g["idx"]
    for step in range(4):
        dt = oracle.dt(m.hmin, 0.01, 0.3, m.max_u(vel), step, 0)
        assert abs(dt - float(g[f"dt{step}"])) <= 1e-12 * dt
        vel = m.advect_diffuse(vel, dt, 0.01)
        vel, pres, _ = m.pressure_project(vel, pres, dt, step, tol=0.0, tol_rel=1e-11)
        assert np.abs(vel[idx] - g[f"vel{step}"]).max() <= 5e-10 * np.abs(g[f"vel{step}"]).max(), step
