"""The oracle's surface forces (ComputeForces restated) against a known answer:
with the velocity at rest and a hydrostatic pressure P = g z, the pressure
force -sum P n dS over the surface points is the buoyancy -g V e_z of the
body (divergence theorem), and the viscous force is zero.  A sphere of 6.4
cells radius on a uniform 32^3 mesh (the sphere workload resolves its body
with 4 cells per radius): within 1% of -g V, with V the sphere's exact
volume (measured 0.2%; the reference's smoothed delta over-counts a curved
surface's area by a few per cent at 13-26 cells per radius, which this
restatement reproduces); the torque about the centre vanishes by symmetry."""
import numpy as np

import oracle


def test_hydrostatic_pressure_force_is_the_buoyancy():
    bpd = 4
    level = np.zeros(bpd ** 3, np.int32)
    index = np.array([(i, j, k) for k in range(bpd) for j in range(bpd) for i in range(bpd)], np.int32)
    m = oracle.Mesh(level, index, [bpd, bpd, bpd], 1, [0, 0, 0], 1.0)
    c, r, g = np.array([0.5, 0.5, 0.5]), 0.2, 3.0
    ob = m.create_obstacle("sphere", c, r)
    bos = ob["block_of_slot"]
    nrm = m.obstacle_surface("sphere", c, r, bos, ob["chi_o"])
    h = 1.0 / (8 * bpd)
    n = m.nb * 512
    z = np.zeros(n)
    for b in range(m.nb):
        iz = np.arange(512) // 64
        z[512 * b:512 * (b + 1)] = (index[b][2] * 8 + iz + 0.5) * h
    pres = g * z
    vel = np.zeros(3 * n)
    udef = np.zeros(3 * len(bos) * 512)
    kin = np.concatenate([c, np.zeros(6)])
    q, bad = m.compute_forces(vel, pres, ob["chi"], bos, nrm, udef, 1e-3, kin)
    assert bad == 0
    V = 4.0 / 3.0 * np.pi * r ** 3
    print("pressure force", q[3:6], "expected z", -g * V)
    assert abs(q[5] + g * V) <= 0.01 * g * V
    assert np.abs(q[3:5]).max() <= 1e-3 * g * V
    assert np.abs(q[6:9]).max() == 0.0          # no viscous force at rest
    assert np.abs(q[9:12]).max() <= 1e-3 * g * V * r
