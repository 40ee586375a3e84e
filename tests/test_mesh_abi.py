"""Host-side tests (no GPU): mesh construction, face tables and the C ABI."""
import re
from pathlib import Path

import numpy as np
import pytest

import cup3d_b200 as cup
from cup3d_b200 import _lib
from tests.meshes import CASES, make_ctx, oracle_mesh

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_header_symbol():
    header = (ROOT / "include" / "cup3d_b200.h").read_text()
    declared = set(re.findall(r"\b(cup_[a-z0-9_]+)\s*\(", header))
    declared -= {"cup_ctx"}
    L = _lib.lib()
    missing = [s for s in sorted(declared) if not hasattr(L, s)]
    assert not missing, missing
    assert declared <= set(_lib.SIGNATURES), sorted(declared - set(_lib.SIGNATURES))


@pytest.mark.parametrize("name", sorted(CASES))
def test_face_tables_match_oracle(name):
    ctx = make_ctx(name)
    m = oracle_mesh(ctx)
    k1, n1 = ctx.faces()
    k2, n2 = m.faces()
    assert (k1 == k2).all()
    assert (n1 == n2).all()


def test_sfc_order_deterministic_and_permutation_invariant():
    ctx = make_ctx("amr3_mixed")
    level, index, _ = ctx.blocks()
    perm = np.random.default_rng(0).permutation(len(level))
    ctx2 = cup.Context(ctx.cfg)
    ctx2.set_mesh(level[perm], index[perm])
    l2, i2, _ = ctx2.blocks()
    assert (l2 == level).all() and (i2 == index).all()


def test_sfc_neighbours_are_local():
    # Hilbert order of the roots: consecutive level-0 blocks are face neighbours
    ctx = cup.Context(cup.config("-bpdx 8 -bpdy 8 -bpdz 8 -levelMax 1", device=-1))
    ctx.set_mesh_uniform()
    _, index, _ = ctx.blocks()
    steps = np.abs(np.diff(index, axis=0)).sum(axis=1)
    assert (steps == 1).all()


def test_rejects_invalid_meshes():
    ctx = cup.Context(cup.config("-bpdx 2 -bpdy 1 -bpdz 1 -levelMax 3", device=-1))
    with pytest.raises(cup.CupError):  # hole
        ctx.set_mesh([0], [[0, 0, 0]])
    with pytest.raises(cup.CupError):  # overlap
        ctx.set_mesh([0, 0, 1], [[0, 0, 0], [1, 0, 0], [0, 0, 0]])
    # 2:1 violation across a face: level 0 next to level 2
    lv = [0] + [2] * 64
    idx = [[0, 0, 0]] + [[4 + i % 4, (i // 4) % 4, i // 16] for i in range(64)]
    with pytest.raises(cup.CupError):
        ctx.set_mesh(lv, idx)


def test_sphere_wake_mesh_is_balanced_and_refined():
    cfg = cup.config("-bpdx 4 -bpdy 2 -bpdz 2 -levelMax 4 -extent 4", device=-1)
    ctx = cup.Context(cfg)
    ctx.set_mesh_sphere_wake([1.0, 1.0, 1.0], 0.0625, -1, 0.5, 1.0, 0.5)
    level, index, h = ctx.blocks()
    assert level.max() == 3 and level.min() >= 0
    kinds, nbrs = ctx.faces()
    # every coarser/finer face links to blocks one level away
    for b in range(len(level)):
        for f in range(6):
            if kinds[b, f] == 2:
                assert level[nbrs[b, f, 0]] == level[b] - 1
            if kinds[b, f] == 3:
                assert all(level[nbrs[b, f, q]] == level[b] + 1 for q in range(4))


def test_config_parse_flags():
    cfg = cup.config("-bpdx 4 -bpdy 2 -bpdz 2 -levelMax 4 -extent 4 -nu 4.1667e-5 -CFL 0.3 "
                     "-BC_x periodic -poissonTolRel 1e-8 -poissonSolver b200_mixed -advection weno5")
    assert list(cfg.bpd) == [4, 2, 2] and cfg.level_max == 4 and cfg.nu == 4.1667e-5
    assert cfg.bc[0] == 1 and cfg.poisson_solver == 1 and cfg.advection == 1
    with pytest.raises(cup.CupError):
        cup.config("-poissonSolver cuda_iterative_typo")
    assert cup.config("").poisson_block_cache == 4
    assert cup.config("-poissonBlockCache 0").poisson_block_cache == 0
    with pytest.raises(cup.CupError):
        cup.config("-poissonBlockCache 5")


def test_batch_needs_device_contexts():
    ctx = cup.Context(cup.config("-bpdx 2 -bpdy 2 -bpdz 2", device=-1))
    ctx.set_mesh_uniform()
    with pytest.raises(cup.CupError, match="device context"):
        cup.Batch([ctx])
    assert cup.lib().cup_batch_num_cases(ctx._p) == 1


def test_python_sphere_mesh_equals_the_library_mesh():
    # bench.py's CPU reference arm builds the frozen sphere mesh without the
    # library; its leaves must be the library's (cup_set_mesh_sphere_wake)
    from cup3d_b200.workloads import SPHERE_FLAGS, SPHERE_MESH, sphere_wake_leaves
    ctx = cup.Context(cup.config(SPHERE_FLAGS, device=-1))
    ctx.set_mesh_sphere_wake(**SPHERE_MESH)
    level, index, _ = ctx.blocks()
    lib_leaves = sorted(map(tuple, np.column_stack([level, index]).tolist()))
    py_leaves = sorted(map(tuple, sphere_wake_leaves().tolist()))
    assert len(py_leaves) == 2340 and py_leaves == lib_leaves
