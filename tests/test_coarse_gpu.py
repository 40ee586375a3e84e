"""Coarse space of the two-level solvers (cup_coarse_matrix, cup_coarse_apply_dev)
and the two-level solve "b200_twolevel":

* A_c from the device operator and the block colouring equals P^T A P of the
  oracle's operator matrix (P constant over each block) to 1e-12, on meshes
  with periodic, wall and free-space faces and coarse-fine interfaces, for the
  mean-constraint modes 1 and 2;
* z = P A_c^-1 P^T r matches a dense solve with the oracle's A_c;
* on the benchmarked sphere mesh with its seeded right-hand side, the
  two-level solve reaches the FP64-checked tolerance in a fraction of the
  block-Jacobi iterations.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import cup3d_b200 as cup
from tests.meshes import make_ctx, oracle_mesh

pytestmark = pytest.mark.gpu


def torch_dev(a):
    import torch
    return torch.tensor(np.asarray(a, np.float64), device="cuda")


def oracle_ac(ctx, m, mode):
    rp, ci, v = m.csr(mode)
    A = sp.csr_matrix((v, ci, rp), shape=(m.n, m.n)).tolil()
    level, index, h = ctx.blocks()
    hh3 = np.repeat(h, 512) ** 3
    if mode == 1:  # the mean row: sum x h^3 on the first cell of block (0,0,0)
        mb = int(np.where((index == 0).all(axis=1))[0][0])
        A[mb * 512, :] = hh3
    A = A.tocsr()
    x = np.random.default_rng(0).standard_normal(m.n)
    ax = A @ x
    if mode == 2:  # every row adds (sum x h^3) h^3, a dense rank-one term the CSR leaves out
        ax = ax + np.sum(x * hh3) * hh3
    assert np.abs(ax - m.apply(x, mode)).max() <= 1e-12 * np.abs(m.apply(x, mode)).max()
    P = sp.csr_matrix((np.ones(m.n), (np.arange(m.n), np.repeat(np.arange(m.nb), 512))), shape=(m.n, m.nb))
    Ac = (P.T @ A @ P).toarray()
    if mode == 2:
        w = 512.0 * h ** 3
        Ac += np.outer(w, w)
    return Ac


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("name", ["tgv32", "amr2_free", "amr3_mixed", "amr3_periodic"])
def test_coarse_matrix_matches_oracle(name, mode):
    ctx = make_ctx(name, device=0, extra=f"-bMeanConstraint {mode}")
    m = oracle_mesh(ctx)
    got, colours = ctx.coarse_matrix()
    ref = oracle_ac(ctx, m, mode)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max(), (np.abs(got - ref).max(), colours)
    assert colours >= 7


def test_coarse_apply_matches_dense_solve():
    ctx = make_ctx("amr3_mixed", device=0)
    m = oracle_mesh(ctx)
    Ac = oracle_ac(ctx, m, 1)
    r = np.random.default_rng(5).standard_normal(m.n)
    rd, zd = torch_dev(r), torch_dev(np.zeros(m.n))
    ctx.coarse_apply(rd, zd)
    yc = np.linalg.solve(Ac, r.reshape(m.nb, 512).sum(axis=1))
    ref = np.repeat(yc, 512)
    # A_c^-1 is kept in FP32
    assert np.abs(zd.cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max()


def test_twolevel_solve_on_sphere_mesh():
    from cup3d_b200.workloads import make_sphere_ctx, poisson_rhs
    ctx = make_sphere_ctx(0)
    m = oracle_mesh(ctx)
    b = poisson_rhs(ctx)
    level, index, _ = ctx.blocks()
    mb = int(np.where((index == 0).all(axis=1))[0][0])
    bm = b.copy()
    bm[mb * 512] = 0.0
    its = {}
    for solver in ("b200", "b200_twolevel"):
        ctx.set_poisson(solver, 0.0, 1e-6, 1000)
        bd, xd = torch_dev(b), torch_dev(np.zeros(m.n))
        rc, st = ctx.poisson_solve_dev(bd, xd)
        assert rc == 0 and st["status"] == 1, (solver, st)
        r_true = np.linalg.norm(bm - m.apply(xd.cpu().numpy())) / np.linalg.norm(bm)
        assert r_true <= 1e-6, (solver, r_true)
        its[solver] = st["iterations"]
        print(f"{solver}: {st['iterations']} iterations, {st['milliseconds']:.2f} ms, true residual {r_true:.2e}")
    print("iterations to 1e-6 on the sphere mesh", its)
    assert its["b200_twolevel"] * 3 <= its["b200"], its


def test_captured_twolevel_step_equals_launched_step():
    # the time step captured as a CUDA graph runs the two-level solver with
    # the coarse space built before the capture: the same steps as launched
    import cup3d_b200 as cup
    from cup3d_b200.workloads import SPHERE_FLAGS, SPHERE_MESH, SPHERE_BODY
    out = []
    for g in (1, 0):
        ctx = cup.Context(cup.config(SPHERE_FLAGS + f" -poissonSolver b200_twolevel -stepGraph {g}", device=0))
        ctx.set_mesh_sphere_wake(**SPHERE_MESH)
        ctx.obstacle_sphere(**SPHERE_BODY)
        its = []
        for step in range(4):
            dt, rc, st = ctx.step(step)
            assert rc == 0, st
            its.append(st["iterations"])
        out.append((ctx.download("vel"), ctx.download("pres"), its))
    (v1, p1, i1), (v0, p0, i0) = out
    print("two-level step iterations, captured / launched:", i1, i0)
    assert i1 == i0
    assert np.abs(v1 - v0).max() <= 1e-12 * np.abs(v0).max()
    assert np.abs(p1 - p0).max() <= 1e-12 * np.abs(p0).max()


@pytest.mark.parametrize("solver", ["b200", "b200_twolevel"])
def test_host_driven_form_matches_persistent_solver(solver):
    # -poissonPersistent 0: five kernels per iteration and a host check every
    # 8 iterations (the coarse correction by its own kernels); the same method
    # as the single cooperative launch, with other summation orders
    sols = {}
    for pers in (1, 0):
        ctx = make_ctx("amr3_mixed", device=0, extra=f"-poissonPersistent {pers}")
        m = oracle_mesh(ctx)
        b = np.random.default_rng(11).standard_normal(m.n)
        hh = np.repeat(m.h, 512)
        b -= np.sum(b * hh ** 3) / np.sum(hh ** 3)
        bd, xd = torch_dev(b), torch_dev(np.zeros(m.n))
        ctx.set_poisson(solver, 0.0, 1e-8, 1000)
        rc, st = ctx.poisson_solve_dev(bd, xd)
        assert rc == 0 and st["status"] == 1 and st["true_rel"] <= 1.5e-8, (pers, st)
        sols[pers] = (xd.cpu().numpy(), st["iterations"])
    print(solver, "iterations persistent / host-driven:", sols[1][1], sols[0][1])
    assert abs(sols[1][1] - sols[0][1]) <= max(2, sols[1][1] // 10)
    assert np.linalg.norm(sols[1][0] - sols[0][0]) <= 1e-6 * np.linalg.norm(sols[1][0])


def test_dense_inverse_blocked_on_sphere_coarse_matrix():
    # A_c of the benchmarked sphere mesh (2340 blocks, mean row of block mb
    # last in the pivot order): the blocked form, to the FP64 accuracy of a
    # dense inverse
    import torch
    from cup3d_b200.workloads import make_sphere_ctx
    ctx = make_sphere_ctx(0)
    Ac, _ = ctx.coarse_matrix()
    level, index, _ = ctx.blocks()
    mb = int(np.where((index == 0).all(axis=1))[0][0])
    a = torch.tensor(Ac, device="cuda")
    pivoted = ctx.dense_inverse(a, mb)
    X = a.cpu().numpy()
    ref = np.linalg.inv(Ac)
    err = np.abs(X - ref).max() / np.abs(ref).max()
    res = np.abs(X @ Ac - np.eye(len(Ac))).max()
    print(f"sphere A_c ({len(Ac)} blocks): blocked inverse vs numpy {err:.2e}, |X A - I| {res:.2e}, pivoted {pivoted}")
    assert not pivoted
    assert err <= 1e-10 and res <= 1e-9


@pytest.mark.parametrize("n", [1, 31, 33, 257])
def test_dense_inverse_sizes_and_pivoted_form(n):
    import torch
    ctx = make_ctx("amr2_free", device=0)
    rng = np.random.default_rng(n)
    # diagonally dominant: the blocked form
    A = rng.standard_normal((n, n)) + 2 * n * np.eye(n)
    a = torch.tensor(A, device="cuda")
    assert not ctx.dense_inverse(a, n // 2)
    assert np.abs(a.cpu().numpy() @ A - np.eye(n)).max() <= 1e-13
    if n < 2:
        return
    # a scaled cyclic shift (zero diagonal): one pivot block holds it all for
    # n <= 32 (partial pivoting inside the block); beyond, the first pivot
    # block has a zero row and the column-wise pivoted form runs
    B = np.roll(np.diag(1.0 + rng.random(n)), 1, axis=0)
    b = torch.tensor(B, device="cuda")
    assert ctx.dense_inverse(b) == (n > 32)
    assert np.abs(b.cpu().numpy() @ B - np.eye(n)).max() <= 1e-15


def test_dense_inverse_singular_matrix_is_an_error():
    import torch
    ctx = make_ctx("amr2_free", device=0)
    a = torch.zeros((40, 40), dtype=torch.float64, device="cuda")
    with pytest.raises(cup.CupError):
        ctx.dense_inverse(a)
    # the context stays usable
    A = np.eye(40) * 3.0
    a = torch.tensor(A, device="cuda")
    assert not ctx.dense_inverse(a)
    assert np.abs(a.cpu().numpy() - np.eye(40) / 3.0).max() <= 1e-15
