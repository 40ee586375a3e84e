"""The reference CPU solver's pipelined BiCGSTAB on the device ("b200_pipelined",
one persistent launch) against the oracle's restatement of it
(orc_bicgstab_pipelined, PoissonSolverAMR.cpp:13-358) on the same operator
and right-hand side: the same residual replacements, restarts and stopping
test, so the iteration counts agree to within two (the sums of the dot
products differ in order) and both solutions satisfy the FP64 tolerance;
their difference is within the tolerance's reach."""
import numpy as np
import pytest

from tests.meshes import make_ctx, oracle_mesh

pytestmark = pytest.mark.gpu


def torch_dev(a):
    import torch
    return torch.tensor(np.asarray(a, np.float64), device="cuda")


def rhs(m, seed):
    b = np.random.default_rng(seed).standard_normal(m.n)
    hh = np.repeat(m.h, 512)
    return b - np.sum(b * hh ** 3) / np.sum(hh ** 3)


@pytest.mark.parametrize("name", ["tgv32", "amr2_free", "amr3_mixed"])
def test_pipelined_matches_oracle(name):
    ctx = make_ctx(name, device=0)
    m = oracle_mesh(ctx)
    b = rhs(m, 21)
    tol = 1e-8
    # precond 0: the exact block inverse (the device's preconditioner; the
    # reference's block CG converges to it)
    x_o, st_o = m.bicgstab_pipelined(b, tol=0.0, tol_rel=tol, precond=0)
    bd, xd = torch_dev(b), torch_dev(np.zeros(m.n))
    ctx.set_poisson("b200_pipelined", 0.0, tol, 1000)
    rc, st = ctx.poisson_solve_dev(bd, xd)
    assert rc == 0 and st["status"] == 1, st
    assert st["true_rel"] <= 1.5 * tol, st
    print(name, "pipelined iterations", st["iterations"], "oracle", st_o["iterations"],
          f"{st['milliseconds']:.2f} ms")
    assert st_o["converged"]
    assert abs(st["iterations"] - st_o["iterations"]) <= 2, (st, st_o)
    x = xd.cpu().numpy()
    assert np.linalg.norm(x - x_o) <= 1e-6 * np.linalg.norm(x_o)


def test_pipelined_on_sphere_mesh():
    from cup3d_b200.workloads import make_sphere_ctx, poisson_rhs
    ctx = make_sphere_ctx(0)
    b = poisson_rhs(ctx)
    out = {}
    for solver in ("b200", "b200_pipelined"):
        bd, xd = torch_dev(b), torch_dev(np.zeros(len(b)))
        ctx.set_poisson(solver, 0.0, 1e-6, 1000)
        ctx.poisson_solve_dev(bd, xd)
        bd, xd = torch_dev(b), torch_dev(np.zeros(len(b)))
        rc, st = ctx.poisson_solve_dev(bd, xd)
        assert rc == 0 and st["status"] == 1 and st["true_rel"] <= 1.5e-6, (solver, st)
        out[solver] = (st["iterations"], round(st["milliseconds"], 3))
    print("sphere mesh to 1e-6 (iterations, ms):", out)
