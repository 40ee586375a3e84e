"""Named workloads of the time-step hot path, shared by bench.py and the
kernel profiling cases.

Sphere at Re=300: domain 4x2x2, 4x2x2 level-0 blocks of 8^3 cells,
levelMax 4 (mesh frozen after refinement around the sphere and its wake:
2340 blocks, 1.198M cells), sphere radius 0.0625 at (1,1,1) moving at +0.1
in x with the frame following it (uinf = -0.1), nu = 0.1*0.125/300, WENO5,
implicit penalization lambda=1e6, plain FP64 BiCGSTAB with the exact block
preconditioner, tolerances -poissonTol 1e-6, -poissonTolRel 1e-4.
"""
from __future__ import annotations

import numpy as np

SPHERE_FLAGS = ("-bpdx 4 -bpdy 2 -bpdz 2 -levelMax 4 -extent 4 -nu 4.1666666666666667e-05 -CFL 0.3 "
                "-lambda 1e6 -advection weno5 -uinfx -0.1 -poissonTol 1e-6 -poissonTolRel 1e-4 -rampup 100")
SPHERE_MESH = dict(center=(1.0, 1.0, 1.0), radius=0.0625, flow_dir=-1, near_radius=2.5, wake_len=1.0,
                   wake_radius=3.0)
SPHERE_BODY = dict(center=(1.0, 1.0, 1.0), radius=0.0625, vel=(0.1, 0.0, 0.0))
SPHERE_WORKLOAD = "sphere_re300_amr_levelmax4_weno5_fp64"


def sphere_wake_leaves(bpd=(4, 2, 2), level_max=4, extent=4.0, center=SPHERE_MESH["center"],
                       radius=SPHERE_BODY["radius"], flow_dir=SPHERE_MESH["flow_dir"],
                       near_radius=SPHERE_MESH["near_radius"], wake_len=SPHERE_MESH["wake_len"],
                       wake_radius=SPHERE_MESH["wake_radius"]):
    """Leaves (level, i, j, k) of the frozen sphere mesh, in pure Python: the
    same refinement rule and the same floating-point operations as the
    library's cup_set_mesh_sphere_wake (a block of level l is split when its
    box comes within (r + near_radius 2^-l) of the centre, or within
    wake_radius 2^-l of the wake segment; then 2:1 balance over the 26
    neighbours).  Used where the library must not be loaded (the CPU
    reference arm of bench.py); the two generators are compared in the tests."""
    import math
    aux = 1 << (level_max - 1)
    nfe = [float(b) * aux * 8 for b in bpd]
    ex0 = (nfe[0] / max(nfe)) * extent
    h0 = ex0 * aux / nfe[0]
    leaves = {(0, i, j, k) for k in range(bpd[2]) for j in range(bpd[1]) for i in range(bpd[0])}

    def split(b):
        leaves.discard(b)
        for c in range(8):
            leaves.add((b[0] + 1, 2 * b[1] + (c & 1), 2 * b[2] + ((c >> 1) & 1), 2 * b[3] + (c >> 2)))

    def covering(l, p):
        for l2 in range(l, -1, -1):
            k = (l2, p[0] >> (l - l2), p[1] >> (l - l2), p[2] >> (l - l2))
            if k in leaves:
                return k
        return None

    def balance():
        changed = True
        while changed:
            changed = False
            todo = set()
            for b in list(leaves):
                l = b[0]
                if l < 2:
                    continue
                for dz in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dx in (-1, 0, 1):
                            if dx == dy == dz == 0:
                                continue
                            p = [b[1] + dx, b[2] + dy, b[3] + dz]
                            if any(p[d] < 0 or p[d] >= (bpd[d] << l) for d in range(3)):
                                continue  # freespace: no wrap
                            c = covering(l, p)
                            if c is not None and c[0] < l - 1:
                                todo.add(c)
            for c in sorted(todo):
                if c in leaves:
                    split(c)
                    changed = True

    def tag(l, lo, hi):
        scale = math.ldexp(1.0, -l)
        s = 0.0
        for d in range(3):
            e = max(lo[d] - center[d], 0.0, center[d] - hi[d])
            s += e * e
        if math.sqrt(s) < radius + near_radius * scale:
            return True
        x0, x1 = center[0], center[0] + flow_dir * wake_len
        xa, xb = min(x0, x1), max(x0, x1)
        ex = max(xa - hi[0], 0.0, lo[0] - xb)
        s = ex * ex
        for d in (1, 2):
            e = max(lo[d] - center[d], 0.0, center[d] - hi[d])
            s += e * e
        return math.sqrt(s) < wake_radius * scale

    for l in range(level_max - 1):
        hb = math.ldexp(h0, -l) * 8
        for b in sorted(x for x in leaves if x[0] == l):
            lo = [b[1] * hb, b[2] * hb, b[3] * hb]
            hi = [lo[0] + hb, lo[1] + hb, lo[2] + hb]
            if tag(l, lo, hi):
                split(b)
        balance()
    balance()
    return np.array(sorted(leaves), np.int32)


def make_sphere_ctx(device, solver="b200"):
    """Context with the frozen sphere mesh and the sphere obstacle."""
    import cup3d_b200 as cup
    cfg = cup.config(SPHERE_FLAGS + f" -poissonSolver {solver}", device=device)
    ctx = cup.Context(cfg)
    ctx.set_mesh_sphere_wake(**SPHERE_MESH)
    ctx.obstacle_sphere(**SPHERE_BODY)
    return ctx


# The learned preconditioner's evaluation case: the same sphere at Re=1000
# (nu = 0.1*0.125/1000), levelMax 5, the mesh frozen after the same
# refinement rule (5000 blocks, 2.56M cells).
SPHERE_RE1000_FLAGS = (SPHERE_FLAGS.replace("-levelMax 4", "-levelMax 5")
                       .replace("-nu 4.1666666666666667e-05", "-nu 1.25e-05"))
SPHERE_RE1000_WORKLOAD = "sphere_re1000_amr_levelmax5_weno5_fp64"


def make_sphere_re1000_ctx(device, solver="b200"):
    """Context with the Re=1000, levelMax 5 sphere mesh and the sphere obstacle."""
    import cup3d_b200 as cup
    cfg = cup.config(SPHERE_RE1000_FLAGS + f" -poissonSolver {solver}", device=device)
    ctx = cup.Context(cfg)
    ctx.set_mesh_sphere_wake(**SPHERE_MESH)
    ctx.obstacle_sphere(**SPHERE_BODY)
    return ctx


def poisson_rhs(ctx):
    """Seeded Poisson right-hand side on the context's mesh: N(0,1) white
    noise per cell plus 8 Gaussian sources (centres uniform in the sphere's
    bounding box +-0.5, widths uniform in 2-8 local cells, amplitudes
    10 N(0,1)), made h^3-weighted zero-mean."""
    rng = np.random.Generator(np.random.PCG64(20261203))
    xyz, hh = ctx.cell_centres()
    b = rng.standard_normal(len(hh))
    c0, r = np.array(SPHERE_BODY["center"]), SPHERE_BODY["radius"]
    lo, hi = c0 - r - 0.5, c0 + r + 0.5
    for _ in range(8):
        c = rng.uniform(lo, hi)
        d2 = np.sum((xyz - c) ** 2, axis=1)
        sigma = rng.uniform(2.0, 8.0) * hh[np.argmin(d2)]
        b += 10.0 * rng.standard_normal() * np.exp(-d2 / (2.0 * sigma ** 2))
    w = hh ** 3
    return b - np.sum(b * w) / np.sum(w)


# Swarm of independent penalized ellipsoids (semi-axes 0.1 x 0.05 x 0.05),
# one per case: case i draws from PCG64(64 + i) a unit quaternion uniform on
# S^3, a speed uniform in [0.05, 0.2] along the body's long axis, 2 or 3
# level-0 blocks per side of the unit cube, 3 or 4 levels and a centre in
# [0.35, 0.65]^3; the mesh is refined around the body (near radius 0.6 of the
# domain at the coarsest level, no wake), which gives 372-2659 blocks per case
# over the first 64 cases (73,239 blocks, 37.5M cells in all).  The bodies
# are held in place (-StaticObstacles 1): the penalization imposes their
# velocity, but a batch does not move bodies, so neither do the cases stepped
# one by one against it.
SWARM_AXES = (0.1, 0.05, 0.05)
SWARM_FLAGS = ("-extent 1 -nu 1e-4 -CFL 0.3 -lambda 1e6 -advection weno5 -poissonTol 1e-6 "
               "-poissonTolRel 1e-4 -rampup 0 -StaticObstacles 1")
SWARM_WORKLOAD = "ellipsoid_swarm_64_cases_weno5_fp64"


def swarm_case(i):
    """Parameters of swarm case i (see above)."""
    rng = np.random.Generator(np.random.PCG64(64 + i))
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    speed = rng.uniform(0.05, 0.2)
    bpd = 2 + int(rng.integers(0, 2))
    level_max = 3 + int(rng.integers(0, 2))
    center = rng.uniform(0.35, 0.65, 3)
    w, x, y, z = q
    long_axis = np.array([1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)])
    return dict(quat=q, vel=speed * long_axis, bpd=bpd, level_max=level_max, center=center)


def make_swarm_ctx(i, device, extra=""):
    """Context of swarm case i with its mesh and its ellipsoid (extra: more flags)."""
    import cup3d_b200 as cup
    p = swarm_case(i)
    b = p["bpd"]
    cfg = cup.config(SWARM_FLAGS + f" -bpdx {b} -bpdy {b} -bpdz {b} -levelMax {p['level_max']} {extra}",
                     device=device)
    ctx = cup.Context(cfg)
    ctx.set_mesh_sphere_wake(p["center"], SWARM_AXES[0], 1, near_radius=0.6, wake_len=0.0, wake_radius=0.6)
    if device >= 0:
        ctx.obstacle_ellipsoid(p["center"], SWARM_AXES, p["quat"], vel=p["vel"], on_device=True)
    return ctx


def swarm_rhs(ctx, i):
    """Seeded Poisson right-hand side of swarm case i: N(0,1) white noise per
    cell from PCG64(1000 + i), made h^3-weighted zero-mean."""
    hh = np.repeat(ctx.blocks()[2], 512)
    b = np.random.Generator(np.random.PCG64(1000 + i)).standard_normal(len(hh))
    return b - np.sum(b * hh ** 3) / np.sum(hh ** 3)
