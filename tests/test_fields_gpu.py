"""Field transfer in the reference's block storage (the drop-in adapter's
path): per-block pointers, GridBlock cells [iz][iy][ix] with interleaved
components, blocks in any order.  Exact round trips against the SoA path."""
import numpy as np
import pytest

import cup3d_b200 as cup
from tests.meshes import make_ctx

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,ncomp", [("vel", 3), ("pres", 1)])
def test_block_storage_round_trip(name, ncomp):
    ctx = make_ctx("amr3_mixed", device=0)
    level, index, _ = ctx.blocks()
    nb = ctx.nb
    rng = np.random.default_rng(5)
    soa = rng.standard_normal(ncomp * nb * 512)
    # the reference's storage of block b: 512 cells x ncomp interleaved
    ref_blocks = [soa.reshape(ncomp, nb, 512)[:, b, :].T.copy() for b in range(nb)]
    perm = rng.permutation(nb)
    ctx.upload_blocks(name, level[perm], index[perm], [ref_blocks[b] for b in perm])
    assert np.array_equal(ctx.download(name), soa)
    ctx.upload(name, 2.0 * soa)
    got = ctx.download_blocks(name, level[perm], index[perm])
    for k, b in enumerate(perm):
        assert np.array_equal(got[k], 2.0 * ref_blocks[b].reshape(-1))


def test_block_storage_rejects_a_missing_or_repeated_block():
    ctx = make_ctx("amr2_free", device=0)
    level, index, _ = ctx.blocks()
    blocks = [np.zeros(512) for _ in range(ctx.nb)]
    with pytest.raises(cup.CupError):
        ctx.upload_blocks("pres", level[:-1], index[:-1], blocks[:-1])
    lv, ix = level.copy(), index.copy()
    lv[1], ix[1] = lv[0], ix[0]
    with pytest.raises(cup.CupError):
        ctx.upload_blocks("pres", lv, ix, blocks)
