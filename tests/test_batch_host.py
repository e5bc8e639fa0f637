"""Batch packing on the host: HostBatch.concat keeps every graph intact (local ids, offsets)."""
import numpy as np

import rak_lowmem as rl


def test_concat_round_trip():
    gs = [rl.gen_rmat(8, 4, seed=s, w_lo=1.0, w_hi=5.0) for s in range(3)] + \
         [rl.HostGraph(np.zeros(4, np.int64), np.zeros(0, np.uint32), np.zeros(0, np.float32))]
    b = rl.HostBatch.concat(gs)
    assert b.graphs == 4 and b.n == sum(g.n for g in gs) and b.m == sum(g.m for g in gs)
    assert b.offsets[0] == 0 and b.offsets[-1] == b.m and np.all(np.diff(b.offsets) >= 0)
    for i, g in enumerate(gs):
        h = b.graph(i)
        np.testing.assert_array_equal(h.offsets, g.offsets)
        np.testing.assert_array_equal(h.targets, g.targets)
        np.testing.assert_array_equal(h.weights, g.weights)
        assert h.targets.max(initial=0) < max(g.n, 1)
    assert rl.HostBatch.concat(gs, weighted=False).weights is None
