"""Local maps of the two-level preconditioner (lmap.cuh): the per-block
correction z_b += W lab_b / h_b that the persistent solver applies on the
tensor cores, with W either the exact one-cell-overlap local solve
("b200_schwarz") or the trained linear network folded into one matrix
("b200_learned").

* the Schwarz map equals the restricted additive Schwarz solve written out
  here in numpy (the 7-point Laplacian on the block and its six face layers,
  zero beyond, solved densely): z_b = [L_s^-1 lab_b]_interior / h_b, on a
  uniform periodic mesh, within the BF16 rounding of W and of the labs
  (relative error <= 1e-2 of the map's own part);
* the residual lab's coarse-fine and boundary rules (sums of finer cells,
  an eighth of coarser interpolations, zero beyond boundaries) through
  the solver test on AMR meshes;
* the folded network equals the network applied by its convolution layers
  (cup_cnn_precond_dev) within BF16 rounding;
* the solver with the Schwarz map converges to the FP64 tolerance (true
  residual) in no more iterations than the two-level method without it.
"""
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


def star_positions():
    """Cube positions (x, y, z in -1..8) of the 896 star-lab entries: the
    block's cells (x + 8 y + 64 z), then face f = 2 d + s (s = 1: the upper
    side) with tangential (a, b) at 512 + 64 f + a + 8 b; the tangential axes
    of d are (1, 2), (0, 2), (0, 1)."""
    pos = []
    for c in range(512):
        pos.append((c % 8, (c // 8) % 8, c // 64))
    tans = {0: (1, 2), 1: (0, 2), 2: (0, 1)}
    for f in range(6):
        d, s = f // 2, f % 2
        for b in range(8):
            for a in range(8):
                q = [0, 0, 0]
                q[d] = 8 if s else -1
                q[tans[d][0]] = a
                q[tans[d][1]] = b
                pos.append(tuple(q))
    return pos


def star_laplacian(pos):
    index = {p: j for j, p in enumerate(pos)}
    n = len(pos)
    L = np.zeros((n, n))
    for j, (x, y, z) in enumerate(pos):
        L[j, j] = -6.0
        for dx, dy, dz in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            k = index.get((x + dx, y + dy, z + dz))
            if k is not None:
                L[j, k] = 1.0
    return L


def test_schwarz_map_matches_dense_overlap_solve():
    import torch
    # no mean-constraint row (it enters no other block's lab)
    ctx = make_ctx("tgv32", device=0, extra="-bMeanConstraint 0")
    m = oracle_mesh(ctx)
    level, index, h = ctx.blocks()
    r = rhs(m, 4)
    z = torch.zeros(m.n, dtype=torch.float64, device="cuda")
    zb = torch.zeros_like(z)
    ctx.schwarz_apply(torch_dev(r), z)
    ctx.block_inverse(torch_dev(r), zb)
    z, zb = z.cpu().numpy(), zb.cpu().numpy()
    # the periodic 32^3 field of r, and each block's star lab from it
    nbk = 4
    g = np.zeros((32, 32, 32))
    for b in range(m.nb):
        ix, iy, iz = index[b]
        g[8 * iz:8 * iz + 8, 8 * iy:8 * iy + 8, 8 * ix:8 * ix + 8] = r[512 * b:512 * (b + 1)].reshape(8, 8, 8)
    pos = star_positions()
    Linv = np.linalg.inv(star_laplacian(pos))
    ref = np.zeros(m.n)
    for b in range(m.nb):
        ix, iy, iz = index[b]
        lab = np.array([g[(8 * iz + q[2]) % 32, (8 * iy + q[1]) % 32, (8 * ix + q[0]) % 32] for q in pos])
        ref[512 * b:512 * (b + 1)] = (Linv @ lab)[:512] / h[b]
    corr_ref, corr = ref - zb, z - zb
    err = np.linalg.norm(corr - corr_ref) / np.linalg.norm(corr_ref)
    print(f"Schwarz map: relative error of the correction {err:.2e}; correction / block inverse "
          f"{np.linalg.norm(corr_ref) / np.linalg.norm(zb):.3f}")
    assert err <= 1e-2, err
    assert np.linalg.norm(z - ref) <= 1e-2 * np.linalg.norm(ref)
    assert nbk ** 3 == m.nb


def test_folded_network_matches_convolution_path():
    import torch
    ctx = make_ctx("amr3_mixed", device=0)
    m = oracle_mesh(ctx)
    n = ctx.cnn_num_params()
    ctx.cnn_set_params((np.random.default_rng(5).standard_normal(n) * 0.15).astype(np.float32))
    r = torch_dev(rhs(m, 3))
    zc, zm, zb = torch.zeros_like(r), torch.zeros_like(r), torch.zeros_like(r)
    ctx.cnn_precond(r, zc)
    ctx.cnn_map_apply(r, zm)
    ctx.block_inverse(r, zb)
    zc, zm, zb = zc.cpu().numpy(), zm.cpu().numpy(), zb.cpu().numpy()
    err = np.linalg.norm(zm - zc) / np.linalg.norm(zc - zb)
    print(f"folded network vs convolution path: relative error {err:.2e}")
    assert err <= 2e-2, err


@pytest.mark.parametrize("name", ["amr3_mixed", "amr2_free"])
def test_schwarz_solver_converges_in_fewer_iterations(name):
    ctx = make_ctx(name, device=0)
    m = oracle_mesh(ctx)
    its = {}
    for solver in ("b200_twolevel", "b200_schwarz"):
        b = rhs(m, 90)
        bd, xd = torch_dev(b), torch_dev(np.zeros(m.n))
        ctx.set_poisson(solver, 0.0, 1e-8, 1000)
        rc, st = ctx.poisson_solve_dev(bd, xd)
        assert rc == 0 and st["status"] == 1 and st["true_rel"] <= 1.5e-8, (solver, st)
        its[solver] = st["iterations"]
    print(name, "iterations to 1e-8", its)
    # measured: 34 against 36 (amr3_mixed), 34 against 35 (amr2_free)
    assert its["b200_schwarz"] <= its["b200_twolevel"], its
