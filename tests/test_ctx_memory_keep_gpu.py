"""rak_ctx_set_memory_keep: with a context pool, rak_lowmem_cuda allocates its graph copy and working
buffers stream-ordered from the pool and keeps them mapped between calls. Results must not change
(synchronous mode: identical labels), on calls in a row, on graphs of different sizes, and after
the pool is switched off again."""
import numpy as np
import pytest

import rak_lowmem as rl

pytestmark = pytest.mark.gpu


def test_memory_keep_same_results():
    gs = [rl.gen_rmat(12, 8, seed=1, w_lo=1.0, w_hi=4.0), rl.gen_rmat(10, 16, seed=2), rl.gen_sbm(5000, 20, 12.0, 50.0, seed=3)]
    with rl.Context(0) as ctx:
        want = [ctx.lowmem(g, mode=rl.MODE_SYNC)[0] for g in gs]
        ctx.set_memory_keep(256 << 20)
        for rep in range(2):
            for g, w in zip(gs, want):
                lab, res = ctx.lowmem(g, mode=rl.MODE_SYNC)
                np.testing.assert_array_equal(lab, w)
                assert res.peak_device_bytes > 0
        ctx.set_memory_keep(0)
        for g, w in zip(gs, want):
            np.testing.assert_array_equal(ctx.lowmem(g, mode=rl.MODE_SYNC)[0], w)
