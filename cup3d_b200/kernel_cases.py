"""Small single-GPU cases of the hot-path kernels, for profilers.

    python -m cup3d_b200.kernel_cases spmv    # one Poisson operator application (sphere mesh)
    python -m cup3d_b200.kernel_cases solve   # 16 BiCGSTAB iterations (sphere mesh, seeded RHS)
    python -m cup3d_b200.kernel_cases step    # 4 full time steps of the sphere workload
    python -m cup3d_b200.kernel_cases swarm   # 16 iterations of a batched solve over 8 swarm cases
    python -m cup3d_b200.kernel_cases swarm_step  # 3 batched two-level steps of 8 swarm cases, bodies moving
    python -m cup3d_b200.kernel_cases learned # 20 training steps, then 16 iterations of the learned solve
    python -m cup3d_b200.kernel_cases adapt   # 20 two-level steps, one mesh adaptation, the coarse rebuild, 1 step

A second argument names the Poisson solver of the sphere cases (default
b200; e.g. b200_twolevel, or b200_twolevel_mixed, whose FP32 inner solve is
the k_bicg_persistent<float> launch).

The sphere cases build the sphere mesh of cup3d_b200.workloads (2340
blocks, 1.198M cells, ~0.3 GB of device memory); the swarm case batches the
first 8 ellipsoid-swarm cases (10,879 blocks, 5.6M cells, ~2.5 GB).  Each exits
0 on success.
"""
from __future__ import annotations

import sys

import numpy as np


def main(argv):
    import torch

    from cup3d_b200.workloads import make_sphere_ctx, make_swarm_ctx, poisson_rhs, swarm_rhs
    case = argv[1] if len(argv) > 1 else "solve"
    if case == "swarm_step":
        import cup3d_b200 as cup
        cases = [make_swarm_ctx(i, 0, "-stepGraph 0 -poissonSolver b200_twolevel -StaticObstacles 0") for i in range(8)]
        batch = cup.Batch(cases)
        for step in range(3):
            rc, dts, forces, st = batch.step(step)
        torch.cuda.synchronize()
        print(f"swarm_step ok: rc {rc}, {batch.nb} blocks, iterations {[s['iterations'] for s in st]}")
        return
    if case == "swarm":
        import cup3d_b200 as cup
        cases = [make_swarm_ctx(i, 0) for i in range(8)]
        b = torch.tensor(np.concatenate([swarm_rhs(c, i) for i, c in enumerate(cases)]), device="cuda")
        batch = cup.Batch(cases)
        batch.set_poisson("b200", 0.0, 1e-30, 16)
        x = torch.zeros_like(b)
        rc, st = batch.poisson_solve_dev(b, x)
        print(f"swarm ok: rc {rc}, {batch.nb} blocks, iterations {[s['iterations'] for s in st]}")
        return
    solver = argv[2] if len(argv) > 2 else "b200"
    ctx = make_sphere_ctx(0, solver)
    n = ctx.nb * 512
    if case == "spmv":
        x = torch.tensor(np.random.default_rng(1).standard_normal(n), device="cuda")
        y = torch.empty_like(x)
        ctx.poisson_apply(x, y, 0)
        torch.cuda.synchronize()
        print(f"spmv ok: {ctx.nb} blocks")
    elif case == "solve":
        b = torch.tensor(poisson_rhs(ctx), device="cuda")
        x = torch.zeros_like(b)
        ctx.set_poisson(solver, 0.0, 1e-30, 16)
        rc, st = ctx.poisson_solve_dev(b, x)
        print(f"solve ok: rc {rc}, {st['iterations']} iterations")
    elif case == "step":
        for step in range(4):
            ctx.step(step)
        torch.cuda.synchronize()
        print(f"step ok: {ctx.nb} blocks")
    elif case == "learned":
        # samples from the residuals of plain iterates 0, 2, 4, 8 of the seeded
        # right-hand side; 20 Adam steps (k_cnn_train); the learned solve
        # (its map phases inside k_bicg_persistent), 16 iterations
        b = torch.tensor(poisson_rhs(ctx), device="cuda")
        level, index, _ = ctx.blocks()
        mb = int(np.where((index == 0).all(axis=1))[0][0])
        ctx.cnn_init(7)
        ctx.cnn_dataset_reserve(ctx.nb * 4)
        for k in (0, 2, 4, 8):
            xk = torch.zeros_like(b)
            if k:
                ctx.set_poisson("b200", 0.0, 1e-30, k)
                ctx.poisson_solve_dev(b, xk)
            ax = torch.zeros_like(b)
            ctx.poisson_apply(xk, ax)
            r = b - ax
            r[mb * 512] = -ax[mb * 512]
            ctx.cnn_dataset_add(r.contiguous())
        ctx.cnn_train(20, 128, 1e-3, 11)
        x = torch.zeros_like(b)
        ctx.set_poisson("b200_learned", 0.0, 1e-30, 16)
        rc, st = ctx.poisson_solve_dev(b, x)
        print(f"learned ok: rc {rc}, {st['iterations']} iterations, {ctx.cnn_dataset_size()} samples")
    elif case == "adapt":
        # the settled sphere flow adapted once (vorticity tagging), then the
        # two-level coarse space of the new mesh (A_c by colours, the blocked
        # inverse) built by the first coarse application, then one step
        for step in range(20):
            ctx.step(step)
        changed = ctx.adapt_mesh()
        r = torch.ones(ctx.nb * 512, dtype=torch.float64, device="cuda")
        z = torch.zeros_like(r)
        ctx.coarse_apply(r, z)
        ctx.step(20)
        torch.cuda.synchronize()
        print(f"adapt ok: changed {changed}, {ctx.nb} blocks")
    else:
        raise SystemExit(f"unknown case {case!r}: spmv | solve | step | learned | adapt | swarm")


if __name__ == "__main__":
    main(sys.argv)
