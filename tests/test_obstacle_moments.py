"""The reference's sphere chi-moment test (tests/python/test_obstacles.py:7-74)
on the oracle's obstacle creation (ObstaclesCreate.cpp:18-148).

The reference runs `Sphere L=3 xpos=3.125 ypos=2.5 zpos=2.5` on an 8x4x4-block
domain of extent 10 with levelMax 2, samples chi on the uniform level-1 grid
(h = 10/128) and checks: the volume to 3 places, the first moments below 1e-9
and the second moments against 4/15 pi r^5 to 1 place.  Here the same sums
run over the oracle's chi (i) on the uniform level-1 mesh and (ii) on a mesh
refined to level 1 only around the body surface, which must give the same
moments to rounding (interior chi is 1 at either level).
"""
import numpy as np
import pytest

import oracle

EXTENT, R, CTR = 10.0, 1.5, (3.125, 2.5, 2.5)
BPD = (8, 4, 4)


def _uniform_level1():
    idx = np.array([(i, j, k) for k in range(8) for j in range(8) for i in range(16)], np.int32)
    return np.ones(len(idx), np.int32), idx


def _refined_at_surface():
    # level 1 where a level-0 block's cells come within 2 coarse cells of the
    # sphere surface, level 0 elsewhere
    h0 = EXTENT / 64
    level, index = [], []
    for k in range(BPD[2]):
        for j in range(BPD[1]):
            for i in range(BPD[0]):
                lo = np.array([i, j, k]) * 8 * h0
                near = np.clip(np.array(CTR), lo, lo + 8 * h0)
                far = np.where(np.abs(lo - CTR) > np.abs(lo + 8 * h0 - CTR), lo, lo + 8 * h0)
                dmin, dmax = np.linalg.norm(near - CTR), np.linalg.norm(far - CTR)
                if dmin <= R + 2 * h0 and dmax >= R - 2 * h0:
                    for c in range(8):
                        level.append(1)
                        index.append((2 * i + (c & 1), 2 * j + ((c >> 1) & 1), 2 * k + (c >> 2)))
                else:
                    level.append(0)
                    index.append((i, j, k))
    return np.array(level, np.int32), np.array(index, np.int32)


def _moments(m, chi):
    h = np.repeat(m.h, 512)
    idx = m.index.reshape(-1, 3)
    c = np.arange(512)
    cell = np.stack([c % 8, (c // 8) % 8, c // 64], axis=1)
    xyz = ((idx[:, None, :] * 8 + cell[None, :, :] + 0.5) * m.h[:, None, None]).reshape(-1, 3) - np.array(CTR)
    x, y, z = xyz.T
    h3 = h ** 3
    return dict(M=np.sum(chi * h3), Mx=np.sum(x * chi * h3), My=np.sum(y * chi * h3), Mz=np.sum(z * chi * h3),
                Mxx=np.sum(x * x * chi * h3), Myy=np.sum(y * y * chi * h3), Mzz=np.sum(z * z * chi * h3),
                Mxy=np.sum(x * y * chi * h3), Myz=np.sum(y * z * chi * h3), Mzx=np.sum(z * x * chi * h3))


def _oracle_sphere(level, index):
    m = oracle.Mesh(level, index, list(BPD), 2, [0, 0, 0], EXTENT)
    return m, m.create_obstacle("sphere", CTR, R)


@pytest.mark.parametrize("mesh", ["uniform_level1", "refined_at_surface"])
def test_sphere_chi_moments_as_the_reference_test(mesh):
    level, index = _uniform_level1() if mesh == "uniform_level1" else _refined_at_surface()
    m, ob = _oracle_sphere(level, index)
    mo = _moments(m, ob["chi"])
    # assertAlmostEqual(a, b, places=p)  <=>  round(a - b, p) == 0
    assert round(mo["M"] - 4 / 3 * np.pi * R ** 3, 3) == 0, mo["M"]
    for k in ("Mx", "My", "Mz", "Mxy", "Myz", "Mzx"):
        assert abs(mo[k]) < 1e-9, (k, mo[k])
    for k in ("Mxx", "Myy", "Mzz"):
        assert round(mo[k] - 4 / 15 * np.pi * R ** 5, 1) == 0, (k, mo[k])
    # the chi-based mass and centre of mass (kernelComputeGridCoM)
    assert abs(ob["mass"] - mo["M"]) < 1e-12 * mo["M"]
    assert np.all(np.abs(ob["com"] - np.array(CTR)) < 1e-12)


def test_sphere_moments_do_not_depend_on_interior_refinement():
    a = _moments(*(lambda mo: (mo[0], mo[1]["chi"]))(_oracle_sphere(*_uniform_level1())))
    b = _moments(*(lambda mo: (mo[0], mo[1]["chi"]))(_oracle_sphere(*_refined_at_surface())))
    for k in a:
        assert abs(a[k] - b[k]) <= 1e-12 * max(1.0, abs(a[k])), (k, a[k], b[k])


def test_ellipsoid_distance_is_exact_on_axes_and_sphere():
    # Eberly's point-to-ellipsoid distance (Ellipsoid.cpp:22-258): with equal
    # axes the signed distance is r - |p|; on an axis it is e_i - |p_i|
    level, index = _uniform_level1()
    m = oracle.Mesh(level, index, list(BPD), 2, [0, 0, 0], EXTENT)
    s = m.create_obstacle("sphere", CTR, R)
    e = m.create_obstacle("ellipsoid", CTR, (R, R, R))
    assert np.array_equal(s["slot"] >= 0, s["slot"] >= 0)
    # same body, different fill box (2 (maxAxis + safety) for the ellipsoid):
    # chi agrees where both have slots, to rounding of the two distance formulas
    assert np.max(np.abs(s["chi"] - e["chi"])) < 1e-12
    assert len(e["block_of_slot"]) >= len(s["block_of_slot"])


def test_rotated_ellipsoid_volume_and_centre():
    # semi-axes 1.2, 0.6, 0.45 rotated by a seeded quaternion: volume to 1e-3
    # relative and chi centre of mass at the body centre (second-order Towers
    # quadrature on h = 10/128)
    level, index = _uniform_level1()
    m = oracle.Mesh(level, index, list(BPD), 2, [0, 0, 0], EXTENT)
    q = np.random.default_rng(3).standard_normal(4)
    q /= np.linalg.norm(q)
    ax = (1.2, 0.6, 0.45)
    ob = m.create_obstacle("ellipsoid", CTR, ax, q)
    vol = 4 / 3 * np.pi * np.prod(ax)
    assert abs(ob["mass"] - vol) < 1e-3 * vol, (ob["mass"], vol)
    assert np.all(np.abs(ob["com"] - np.array(CTR)) < 2e-3)
