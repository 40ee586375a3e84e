"""cup_cnn_forward_host_noalloc: the network forward staged in a static device
array instead of per-call allocations.

* two calls in a row (a full batch of CUP_CNN_FORWARD_NOALLOC_MAX samples,
  then a smaller one) give bit-identical outputs to cup_cnn_forward_host on
  the same inputs: the same kernel runs on the same weights;
* a batch above the static capacity is rejected with CUP_ERR_ARG and a
  message naming the capacity, before any device work.

The file name sorts last so that the suite also runs these tests after every
other test has used the device in the same process.
"""
import numpy as np
import pytest

from cup3d_b200 import _lib
from tests.meshes import make_ctx

pytestmark = pytest.mark.gpu


def _ctx_with_weights(seed):
    ctx = make_ctx("tgv32", device=0)
    p = np.random.default_rng(seed).standard_normal(ctx.cnn_num_params()).astype(np.float32) * 0.15
    ctx.cnn_set_params(p)
    return ctx


def test_noalloc_forward_matches_allocating_forward_on_two_calls():
    ctx = _ctx_with_weights(21)
    rng = np.random.default_rng(22)
    n1, n2 = _lib.CNN_FORWARD_NOALLOC_MAX, 5
    x1 = rng.standard_normal(n1 * 1000).astype(np.float32)
    x2 = rng.standard_normal(n2 * 1000).astype(np.float32)
    got1 = ctx.cnn_forward_noalloc(x1, n1)
    got2 = ctx.cnn_forward_noalloc(x2, n2)
    ref1 = ctx.cnn_forward(x1, n1)
    ref2 = ctx.cnn_forward(x2, n2)
    assert np.abs(ref1).max() > 0 and np.abs(ref2).max() > 0
    assert np.array_equal(got1, ref1)
    assert np.array_equal(got2, ref2)


def test_noalloc_forward_rejects_batches_above_capacity():
    ctx = _ctx_with_weights(23)
    n = _lib.CNN_FORWARD_NOALLOC_MAX + 1
    with pytest.raises(_lib.CupError) as err:
        ctx.cnn_forward_noalloc(np.zeros(n * 1000, np.float32), n)
    assert err.value.code == _lib.CUP_ERR_ARG
    assert "static staging capacity of 64" in str(err.value)
