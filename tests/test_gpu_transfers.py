"""Block transfers through the C-ABI (w2d_put_blocks / w2d_get_blocks) that
span several chunks of the library's 64 MB device stage: every block comes
back as it went in (FP64 pools exactly, FP32 pools as the values rounded to
single precision), in the caller's order, for IDs in any order, from
pageable and from pinned host arrays.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W = 20


def _pool(precision, nblocks, neq=4):
    from walicxe2d_b200.api import Context
    from walicxe2d_b200.params import base_params
    p = base_params(nblocks=nblocks, neq=neq, npas=neq - 4)
    p.precision = precision
    return Context(p)


@pytest.mark.parametrize("precision", [64, 32])
def test_multi_chunk_round_trip(precision):
    n = 7000                      # 7000 x 4 x 400 x 8 B = 89.6 MB: two chunks
    ctx = _pool(precision, n + 16)
    rng = np.random.default_rng(precision)
    ids = rng.permutation(np.arange(1, n + 17, dtype=np.int32))[:n]
    u = rng.normal(0.0, 1.0, (n, 4, W, W))
    ctx.put_blocks(ids, u)
    back = ctx.get_blocks(ids)
    want = u if precision == 64 else u.astype(np.float32).astype(np.float64)
    assert np.array_equal(back, want)
    # a second order of the same IDs, into a pinned array
    import torch
    order = rng.permutation(n)
    out = torch.empty((n, 4, W, W), dtype=torch.float64, pin_memory=True).numpy()
    ctx.get_blocks(ids[order], out)
    assert np.array_equal(out, want[order])
    ctx.close()


def test_ids_outside_the_pool_are_refused():
    ctx = _pool(64, 100)
    u = np.zeros((2, 4, W, W))
    with pytest.raises(Exception):
        ctx.put_blocks(np.array([1, 101], np.int32), u)
    with pytest.raises(Exception):
        ctx.get_blocks(np.array([0], np.int32))
    ctx.close()
