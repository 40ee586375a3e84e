"""Known-answer tests that pin the CPU oracle to the reference's formulas.

The reference ships no golden vectors for the hot path (its two C++ unit tests
cover ghost shifts on a periodic grid and a logger); these tests pin the oracle
with identities the reference's own formulas must satisfy.
"""
import numpy as np
import pytest

import oracle
from tests.meshes import cell_centres, make_ctx, oracle_mesh


def L_D():
    """8^3 Dirichlet 7-point matrix of PoissonSolverExp::getA_local (6 diag, -1 faces)."""
    n = 512
    A = np.zeros((n, n))
    for i in range(n):
        ix, iy, iz = i % 8, (i // 8) % 8, i // 64
        A[i, i] = 6
        for d, (lo) in enumerate((ix, iy, iz)):
            for s in (-1, 1):
                q = [ix, iy, iz]
                q[d] += s
                if 0 <= q[d] < 8:
                    A[i, q[0] + 8 * q[1] + 64 * q[2]] = -1
    return A


def test_pinv_is_minus_inverse_of_dirichlet_block():
    # PoissonSolverExp.cpp:17-111: P_inv = -(L_D)^-1
    P = oracle.pinv().reshape(512, 512)
    err = np.abs(P @ L_D() + np.eye(512)).max()
    assert err < 1e-12


def test_fast_diagonalization_equals_pinv():
    # The device preconditioner applies P_inv as S3 diag(-1/(li+lj+lk)) S3 with
    # S the DST-I eigenvectors of tridiag(-1,2,-1); restated here in numpy.
    k = np.arange(1, 9)
    S = np.sqrt(2 / 9) * np.sin(np.pi * np.outer(k, k) / 9)
    lam = 2 - 2 * np.cos(np.pi * k / 9)
    S3 = np.kron(np.kron(S, S), S)  # index order z,y,x matches i = x + 8y + 64z
    L3 = (lam[:, None, None] + lam[None, :, None] + lam[None, None, :]).reshape(-1)
    Pfd = -S3 @ np.diag(1 / L3) @ S3
    P = oracle.pinv().reshape(512, 512)
    assert np.abs(Pfd - P).max() < 1e-13


def test_block_cg_converges_to_exact_inverse():
    # getZImplParallel stops at 1e-7 relative: its output matches (1/h) P_inv r to that level
    ctx = make_ctx("amr2_free")
    m = oracle_mesh(ctx)
    r = np.random.default_rng(1).standard_normal(m.n)
    z_cg = m.precond_cg(r)
    z_ex = m.precond_pinv(r)
    rel = np.linalg.norm(z_cg - z_ex) / np.linalg.norm(z_ex)
    assert rel < 1e-5


def test_poisson_tgv_second_order():
    # KernelLHSPoisson: A x = h (sum6 - 6 c) ~ h^3 lap(x); for cos x cos y cos z, lap = -3 x
    ctx = make_ctx("tgv32")
    m = oracle_mesh(ctx)
    xyz, h = cell_centres(ctx)
    f = np.cos(xyz[:, 0]) * np.cos(xyz[:, 1]) * np.cos(xyz[:, 2])
    y = m.apply(f, mean_constraint=0)
    exact = -3 * h ** 3 * f
    err = np.abs(y - exact).max() / np.abs(exact).max()
    hh = h[0]
    assert err < 0.5 * hh ** 2  # 7-point truncation error ~ h^2/4


@pytest.mark.parametrize("name", ["amr2_free", "amr3_mixed"])
def test_poisson_amr_exact_for_quadratics(name):
    # The coarse-fine rows of PoissonSolverExp interpolate quadratically and take
    # second-order Taylor terms: A f = h^3 lap(f) exactly for quadratic f away
    # from the (zero-flux) domain boundary.
    ctx = make_ctx(name)
    m = oracle_mesh(ctx)
    xyz, h = cell_centres(ctx)
    x, y, z = xyz.T
    f = 0.3 * x * x - 0.7 * y * y + 0.2 * z * z + 0.5 * x * y - 0.1 * y * z + 0.4 * x - 0.2
    lap = 2 * (0.3 - 0.7 + 0.2)
    Af = m.apply(f, mean_constraint=0)
    kinds, _ = ctx.faces()
    cfg = ctx.cfg
    ext = [cfg.extent * b / max(cfg.bpd) for b in cfg.bpd]
    near = np.zeros(len(f), bool)
    for d in range(3):
        if cfg.bc[d] != 1:
            near |= (xyz[:, d] < 1.01 * h) | (xyz[:, d] > ext[d] - 1.01 * h)
        else:
            # periodic wrap breaks polynomials: exclude cells whose stencil wraps
            near |= (xyz[:, d] < 2.01 * h) | (xyz[:, d] > ext[d] - 2.01 * h)
    sel = ~near
    assert sel.sum() > 500
    got = Af[sel] / h[sel] ** 3
    assert np.abs(got - lap).max() < 1e-9 * max(1.0, abs(lap)) / min(h) ** 0


@pytest.mark.parametrize("name", ["amr3_periodic", "tgv32"])
def test_poisson_conservative(name):
    # Fully periodic: fluxes telescope, so the columns of A sum to zero.
    ctx = make_ctx(name)
    m = oracle_mesh(ctx)
    x = np.random.default_rng(5).standard_normal(m.n)
    y = m.apply(x, mean_constraint=0)
    assert abs(y.sum()) < 1e-12 * np.abs(y).sum()


def test_mean_constraint_row():
    ctx = make_ctx("amr2_free")
    m = oracle_mesh(ctx)
    level, index, h = ctx.blocks()
    x = np.random.default_rng(2).standard_normal(m.n)
    y0 = m.apply(x, mean_constraint=0)
    y1 = m.apply(x, mean_constraint=1)
    y2 = m.apply(x, mean_constraint=2)
    hh = np.repeat(h, 512)
    avg = np.sum(x * hh ** 3)
    mb = int(np.where((index == 0).all(axis=1))[0][0])
    diff = y1 - y0
    diff[mb * 512] = 0
    assert np.abs(diff).max() == 0
    assert abs(y1[mb * 512] - avg) < 1e-14 * np.abs(x).sum()
    assert np.allclose(y2, y0 + avg * hh ** 3, rtol=0, atol=1e-14)


@pytest.mark.parametrize("name", ["tgv32", "amr2_free"])
def test_solvers_converge_and_agree(name):
    ctx = make_ctx(name)
    m = oracle_mesh(ctx)
    rng = np.random.default_rng(3)
    b = rng.standard_normal(m.n)
    hh = np.repeat(m.h, 512)
    b -= np.sum(b * hh ** 3) / np.sum(hh ** 3)  # compatible RHS
    x1, s1 = m.bicgstab_gpu(b, tol=0.0, tol_rel=1e-12)
    x2, s2 = m.bicgstab_pipelined(b, tol=0.0, tol_rel=1e-12, precond=0)
    assert s1["converged"] and s2["converged"]
    bb = b.copy()
    for bvec in (bb,):
        mb = m.nb and int(np.where((np.asarray(ctx.blocks()[1]) == 0).all(axis=1))[0][0])
        bvec[mb * 512] = 0.0
    for x in (x1, x2):
        r = bb - m.apply(x, mean_constraint=1)
        assert np.linalg.norm(r) <= 2e-12 * np.linalg.norm(bb)
    assert np.linalg.norm(x1 - x2) <= 1e-9 * np.linalg.norm(x1)


def test_ghost_shift_periodic_exact():
    # Port of tests/cubismup3d/TestBoundaries.cpp:13-81: a periodic uniform grid
    # holding 0.1 + ix + 1000 iy + 1e6 iz; every ghost equals the shifted cell.
    ctx = make_ctx("tgv32")
    m = oracle_mesh(ctx)
    level, index, h = ctx.blocks()
    N = 32
    gi = np.zeros(m.n)
    for b in range(m.nb):
        for c in range(512):
            ix = index[b, 0] * 8 + c % 8
            iy = index[b, 1] * 8 + (c // 8) % 8
            iz = index[b, 2] * 8 + c // 64
            gi[b * 512 + c] = 0.1 + ix + 1000 * iy + 1e6 * iz
    for b in (0, 5, m.nb - 1):
        lab = m.lab(gi, 1, 3, b, False)[0]
        for z in range(-3, 11):
            for y in range(-3, 11):
                for x in range(-3, 11):
                    out = sum(1 for q in (x, y, z) if q < 0 or q > 7)
                    if out > 1:
                        continue  # star stencils: edges and corners unused
                    ix = (index[b, 0] * 8 + x) % N
                    iy = (index[b, 1] * 8 + y) % N
                    iz = (index[b, 2] * 8 + z) % N
                    assert lab[z + 3, y + 3, x + 3] == 0.1 + ix + 1000 * iy + 1e6 * iz


def test_upwind5_exact_on_quintics():
    # AdvectionDiffusion.cpp:97-102: the upwind-biased stencil is exact for
    # polynomials of degree <= 5 (in the cell index).
    for sgn in (1.0, -1.0):
        u = np.array([np.polyval([0.1, -0.3, 0.2, 1.0, -2.0, 0.5], i) for i in range(-3, 4)])
        if sgn > 0:
            d = (-2 * u[0] + 15 * u[1] - 60 * u[2] + 20 * u[3] + 30 * u[4] - 3 * u[5]) / 60.
        else:
            d = (2 * u[6] - 15 * u[5] + 60 * u[4] - 20 * u[3] - 30 * u[2] + 3 * u[1]) / 60.
        exact = np.polyval(np.polyder([0.1, -0.3, 0.2, 1.0, -2.0, 0.5]), 0)
        assert abs(d - exact) < 1e-12


def test_rk3_coefficients_third_order():
    # AdvectionDiffusion.cpp:289-290, Williamson low-storage RK3: integrating
    # du/dt = lambda u for one step reproduces exp(lambda dt) to O(dt^4).
    a = [1 / 3, 15 / 16, 8 / 15]
    b = [-5 / 9, -153 / 128, 0.0]
    for lam_dt in (1e-2, 2e-2):
        u, tmp = 1.0, 0.0
        for s in range(3):
            tmp += lam_dt * u
            u += a[s] * tmp
            tmp *= b[s]
        assert abs(u - np.exp(lam_dt)) < 0.1 * lam_dt ** 4


def test_dissipation_diagnostics_of_taylor_green():
    # ComputeDissipation on the Taylor-Green field u = sin x cos y cos z,
    # v = -cos x sin y cos z on a uniform periodic 32^3 grid: kinetic energy
    # (2 pi)^3 / 8 exactly (cell-centred means of sin^2 cos^2 cos^2), zero
    # linear momentum and zero circulation by symmetry
    from tests.meshes import make_ctx, oracle_mesh, cell_centres
    ctx = make_ctx("tgv32")
    m = oracle_mesh(ctx)
    xyz, _ = cell_centres(ctx)
    x, y, z = xyz.T
    vel = np.concatenate([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), 0 * x])
    q = m.dissipation(vel, np.zeros(m.n), None, 0.01)
    assert abs(q[18] - np.pi ** 3) <= 1e-12 * np.pi ** 3
    assert np.abs(q[0:3]).max() <= 1e-12 and np.abs(q[6:9]).max() <= 1e-12
