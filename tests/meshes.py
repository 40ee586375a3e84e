"""Shared mesh cases for the tests: host-only product contexts plus the oracle
mesh built from the same leaf list in the same block order."""
from __future__ import annotations

import numpy as np

import cup3d_b200 as cup
import oracle

# name -> (flags, generator)
CASES = {
    # Taylor-Green, 4x4x4 blocks of 8^3, triply periodic
    "tgv32": ("-bpdx 4 -bpdy 4 -bpdz 4 -levelMax 1 -extent 6.283185307179586 "
              "-BC_x periodic -BC_y periodic -BC_z periodic", ("uniform",)),
    # 2-level random AMR, free-space boundaries
    "amr2_free": ("-bpdx 2 -bpdy 2 -bpdz 2 -levelMax 2 -extent 1", ("random", 7, 0.35)),
    # 3-level random AMR, periodic in x and z, wall in y (80 blocks)
    "amr3_mixed": ("-bpdx 4 -bpdy 2 -bpdz 3 -levelMax 3 -extent 2 -BC_x periodic -BC_y wall "
                   "-BC_z periodic", ("random", 1, 0.1)),
    # 3-level random AMR, fully periodic (141 blocks)
    "amr3_periodic": ("-bpdx 4 -bpdy 4 -bpdz 4 -levelMax 3 -extent 1 -BC_x periodic -BC_y periodic "
                      "-BC_z periodic", ("random", 3, 0.05)),
}


def make_ctx(name, device=-1, extra=""):
    flags, gen = CASES[name]
    cfg = cup.config(flags + " " + extra, device=device)
    ctx = cup.Context(cfg)
    if gen[0] == "uniform":
        ctx.set_mesh_uniform()
    elif gen[0] == "random":
        ctx.set_mesh_random(gen[1], gen[2])
    return ctx


def oracle_mesh(ctx):
    level, index, _ = ctx.blocks()
    cfg = ctx.cfg
    return oracle.Mesh(level, index, list(cfg.bpd), cfg.level_max, list(cfg.bc), cfg.extent)


def cell_centres(ctx):
    """Physical cell centres (nb*512, 3) in device block order."""
    level, index, h = ctx.blocks()
    nb = len(level)
    ix = np.arange(512) % 8
    iy = (np.arange(512) // 8) % 8
    iz = np.arange(512) // 64
    xyz = np.zeros((nb, 512, 3))
    for d, i in enumerate((ix, iy, iz)):
        xyz[:, :, d] = (index[:, d:d + 1] * 8 + i[None, :] + 0.5) * h[:, None]
    return xyz.reshape(-1, 3), np.repeat(h, 512)
