"""Mesh adaptation on the CPU: the oracle's leaf decision (refinement with
2:1 balance, merging of siblings) and field transfer (Simulation::adaptMesh,
Simulation.cpp:128-149; the rules stand in for Cubism's MeshAdaptation)."""
import numpy as np

import oracle


def _mesh(leaves, bpd=(2, 2, 2), level_max=4, bc=(0, 0, 0)):
    leaves = np.array(sorted(leaves), np.int32)
    return oracle.Mesh(leaves[:, 0], leaves[:, 1:], list(bpd), level_max, list(bc), 1.0), leaves


def _uniform(l, bpd=(2, 2, 2)):
    return [(l, i, j, k) for k in range(bpd[2] << l) for j in range(bpd[1] << l) for i in range(bpd[0] << l)]


def test_refining_one_block_keeps_2to1_balance():
    m, leaves = _mesh(_uniform(0))
    ind = np.zeros(m.nb)
    ind[0] = 5.0  # block (0, 0, 0, 0) above Rtol
    out = m.adapt_leaves(ind, 1.0, 0.0)
    assert len(out) == 8 + 7  # one block split, no balance needed
    # twice more on the same corner: the balance refines the neighbours
    for _ in range(2):
        m, leaves = _mesh([tuple(r) for r in out])
        ind = np.zeros(m.nb)
        ind[np.argmax(m.level * 1000 - m.index.reshape(-1, 3).sum(axis=1))] = 5.0
        out = m.adapt_leaves(ind, 1.0, 0.0)
    assert max(r[0] for r in out) == 3
    _assert_balanced(out, (2, 2, 2), periodic=(False, False, False))


def _assert_balanced(leaves, bpd, periodic):
    """Every leaf's 26 neighbours are covered by leaves at most one level coarser."""
    s = {tuple(int(v) for v in r) for r in leaves}

    def cover(l, p):
        for a in range(l, -1, -1):
            k = (a, p[0] >> (l - a), p[1] >> (l - a), p[2] >> (l - a))
            if k in s:
                return a
        return None

    for l, i, j, k in s:
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    p = [i + dx, j + dy, k + dz]
                    ok = True
                    for d in range(3):
                        N = bpd[d] << l
                        if not 0 <= p[d] < N:
                            if periodic[d]:
                                p[d] %= N
                            else:
                                ok = False
                    if not ok:
                        continue
                    a = cover(l, p)
                    assert a is None or a >= l - 1, ((l, i, j, k), p, a)


def test_merging_needs_all_siblings_and_balance():
    m, _ = _mesh(_uniform(1))
    ind = np.zeros(m.nb)
    out = m.adapt_leaves(ind, 1.0, 0.5)
    assert len(out) == 8 and (out[:, 0] == 0).all()  # every sibling group merges
    ind[0] = 0.7  # one sibling between Ctol and Rtol: its group stays
    out = m.adapt_leaves(ind, 1.0, 0.5)
    assert len(out) == 8 + 7


def test_transfer_is_exact_for_linear_fields_and_conservative():
    m0, _ = _mesh(_uniform(1), bc=(1, 1, 1))
    ind = np.zeros(m0.nb)
    ind[:4] = 2.0
    leaves = m0.adapt_leaves(ind, 1.0, -1.0)
    m1, _ = _mesh([tuple(r) for r in leaves], bc=(1, 1, 1))

    def centres(m):
        c = np.arange(512)
        cell = np.stack([c % 8, (c // 8) % 8, c // 64], axis=1)
        idx = m.index.reshape(-1, 3)
        return ((idx[:, None, :] * 8 + cell[None] + 0.5) * m.h[:, None, None]).reshape(-1, 3), np.repeat(m.h, 512)

    x0, h0 = centres(m0)
    x1, h1 = centres(m1)
    f = 0.3 + 2.0 * np.sin(2 * np.pi * x0[:, 0]) * np.cos(2 * np.pi * x0[:, 1])
    g = m0.adapt_transfer(m1, f, 1, False)
    # conservation: the h^3-weighted sum is unchanged
    assert abs(np.sum(g * h1 ** 3) - np.sum(f * h0 ** 3)) < 1e-13
    # blocks that stay are copied
    keep0 = {tuple(r): b for b, r in enumerate(zip(m0.level, *m0.index.reshape(-1, 3).T))}
    for b, r in enumerate(zip(m1.level, *m1.index.reshape(-1, 3).T)):
        if r in keep0:
            assert np.array_equal(g[b * 512:(b + 1) * 512], f[keep0[r] * 512:(keep0[r] + 1) * 512])
    # a linear field: refined values exact away from periodic wrap
    lin0 = 1.0 + 0.5 * x0[:, 0] - 0.25 * x0[:, 2]
    lin1 = m0.adapt_transfer(m1, lin0, 1, False)
    ref = 1.0 + 0.5 * x1[:, 0] - 0.25 * x1[:, 2]
    inner = (x1 > 0.1).all(axis=1) & (x1 < 0.9).all(axis=1)
    assert np.abs(lin1 - ref)[inner].max() < 1e-13
