"""Generates the committed golden fixtures of tests/golden/ from the CPU oracle
and the product's host mesh code (no GPU needed).

    python tests/golden/make_golden.py

The reference itself cannot run here (its Cubism submodule is absent and it
needs MPI), so the fixtures pin the oracle and the host mesh code to fixed
values, and the GPU tests compare the device path against the same values:

* mesh_<case>.npz     leaf order (level, index) after cup_set_mesh's space-filling-
                      curve ordering (bit-exact) and the face tables;
* poisson_<case>.npz  y = A x (mean constraint 1) and z = P_inv x for a seeded x:
                      norms and 512 sampled entries; a solve to 1e-10: iterations,
                      solution norm and samples;
* tgv32_steps.npz     the Taylor-Green case (32^3, nu 0.01, CFL 0.3, upwind5,
                      Poisson to 1e-11): dt and velocity samples/norms after 1..4 steps.

All of these fixtures are self-pinned: they record what this repository's
oracle and host mesh code compute, so they catch regressions but say nothing
about the reference by themselves.  What ties the oracle to the reference's
own tests and values is elsewhere:

* tests/test_obstacle_moments.py  the reference's sphere chi-moment test
                      (tests/python/test_obstacles.py:7-74) with its tolerances;
* tests/test_oracle_kat.py        the reference's periodic ghost-shift test
                      (tests/cubismup3d/TestBoundaries.cpp:19-104) and known
                      answers built from the reference's formulas (stencil
                      exactness, P_inv L = I, RK3 coefficients).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from tests.meshes import make_ctx, oracle_mesh  # noqa: E402

POISSON_CASES = ["tgv32", "amr2_free", "amr3_mixed", "amr3_periodic"]
NSAMPLE = 512


def sample_index(n, seed):
    return np.sort(np.random.default_rng(seed).choice(n, size=min(NSAMPLE, n), replace=False)).astype(np.int64)


def tgv_velocity(ctx):
    xyz, _ = ctx.cell_centres()
    x, y, z = xyz.T
    return np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), 0 * x])


def poisson_case(name):
    ctx = make_ctx(name)
    level, index, h = ctx.blocks()
    kinds, nbrs = ctx.faces()
    np.savez_compressed(HERE / f"mesh_{name}.npz", level=level, index=index, h=h, kinds=kinds, nbrs=nbrs)
    m = oracle_mesh(ctx)
    x = np.random.default_rng(42).standard_normal(m.n)
    idx = sample_index(m.n, 1)
    y = m.apply(x, mean_constraint=1)
    z = m.precond_pinv(x, oracle.pinv())
    hh = np.repeat(m.h, 512)
    b = np.random.default_rng(9).standard_normal(m.n)
    b -= np.sum(b * hh ** 3) / np.sum(hh ** 3)
    xs, st = m.bicgstab_gpu(b, tol=0.0, tol_rel=1e-10)
    np.savez_compressed(HERE / f"poisson_{name}.npz", idx=idx, y=y[idx], y_norm=np.linalg.norm(y),
                        z=z[idx], z_norm=np.linalg.norm(z), solve_iterations=st["iterations"],
                        solve_restarts=st["restarts"], x=xs[idx], x_norm=np.linalg.norm(xs))


def tgv_steps():
    flags = "-nu 0.01 -CFL 0.3 -rampup 0 -poissonTol 0 -poissonTolRel 1e-11"
    ctx = make_ctx("tgv32", extra=flags)
    m = oracle_mesh(ctx)
    vel = tgv_velocity(ctx)
    pres = np.zeros(m.n)
    idx = sample_index(3 * m.n, 2)
    out = {"idx": idx}
    for step in range(4):
        dt = oracle.dt(m.hmin, 0.01, 0.3, m.max_u(vel), step, 0)
        vel = m.advect_diffuse(vel, dt, 0.01)
        vel, pres, info = m.pressure_project(vel, pres, dt, step, tol=0.0, tol_rel=1e-11)
        out[f"dt{step}"] = dt
        out[f"vel{step}"] = vel[idx]
        out[f"vel_norm{step}"] = np.linalg.norm(vel)
        out[f"pres_norm{step}"] = np.linalg.norm(pres)
    np.savez_compressed(HERE / "tgv32_steps.npz", **out)


if __name__ == "__main__":
    for name in POISSON_CASES:
        poisson_case(name)
    tgv_steps()
    for p in sorted(HERE.glob("*.npz")):
        print(p.name, p.stat().st_size)
