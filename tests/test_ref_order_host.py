"""The reference GPU path's vertex order (inc/rakLowmemCuda.hxx:505-519, 563: std::partition of the
vertex ids by degree < 4, then of the rest by degree < 128) as the device code restates it: per
graph of a batch, one exclusive prefix count of the match flags gives every hole (a non-matching
element left of the match count, ranked from the left) and every mover (a matching element from
the match count on, ranked from the right); the k-th hole swaps with the k-th mover. Checked here,
in numpy over a concatenation of graphs, against the reference's own std::partition calls compiled
into the oracle bridge."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.skipif(not orc.have_ref_cpu(), reason="oracle/_ref not built")


def segmented_order(offsets, vbase):
    """Global vertex indices in each segment's reference order (the device kernels' arithmetic)."""
    n = len(offsets) - 1
    deg = np.diff(offsets)
    gid = np.repeat(np.arange(len(vbase) - 1), np.diff(vbase))
    b = vbase[gid]
    ks = np.arange(n, dtype=np.int64)
    lo_cnt = np.zeros(len(vbase) - 1, np.int64)
    for limit in (4, 128):
        lo = b + lo_cnt[gid]
        idx = np.arange(n)
        f = ((idx >= lo) & (deg[ks] < limit)).astype(np.int64)
        P = np.concatenate([[0], np.cumsum(f)])                  # exclusive prefix, n + 1 entries
        cnt = P[vbase[1:]] - P[vbase[:-1]]
        c = cnt[gid]
        pp = P[idx] - P[b]
        mover = np.full(n, -1, np.int64)
        m = (f == 1) & (idx - lo >= c)
        mover[(lo + (c - pp - 1))[m]] = idx[m]
        h = (f == 0) & (idx >= lo) & (idx - lo < c)
        j = mover[(lo + (idx - lo - pp))[h]]
        assert (j >= 0).all()
        ks_h, ks_j = ks[idx[h]].copy(), ks[j].copy()
        ks[idx[h]], ks[j] = ks_j, ks_h
        lo_cnt = lo_cnt + cnt if limit == 4 else lo_cnt
    return ks - b


def test_segmented_order_equals_reference_partition():
    gs = [rl.gen_rmat(9, 8, seed=3), rl.gen_sbm(2000, 20, 12.0, 30.0, seed=4),
          rl.gen_lattice(30, 20, 0.05, 0.01, seed=5), rl.gen_lattice(1, 50, 0.0, 0.0, seed=6),
          rl.HostGraph(np.zeros(2, np.int64), np.zeros(0, np.uint32)), rl.gen_rmat(12, 16, seed=7)]
    rows = [np.array([v for v in range(150) if v != u], np.uint32) for u in range(150)]
    off = np.zeros(151, np.int64)
    off[1:] = np.cumsum([len(r) for r in rows])
    gs.append(rl.HostGraph(off, np.concatenate(rows)))                 # every degree >= 128
    hb = rl.HostBatch.concat(gs)
    ks = segmented_order(np.asarray(hb.offsets), np.asarray(hb.graph_offsets))
    for i, g in enumerate(gs):
        a, z = int(hb.graph_offsets[i]), int(hb.graph_offsets[i + 1])
        np.testing.assert_array_equal(ks[a:z], orc.ref_vertex_order(g), err_msg=f"graph {i}")


def test_segmented_order_on_random_degree_sequences():
    """Batches of random graphs whose degrees straddle both partition limits (< 4 and < 128)."""
    rng = np.random.default_rng(1234)
    for trial in range(20):
        gs = []
        for _ in range(int(rng.integers(1, 6))):
            n = int(rng.integers(1, 400))
            kind = rng.random(n)
            deg = np.where(kind < 0.4, rng.integers(0, 4, n), np.where(kind < 0.9, rng.integers(4, 128, n),
                                                                       rng.integers(128, 200, n)))
            off = np.zeros(n + 1, np.int64)
            off[1:] = np.cumsum(deg)
            tgt = rng.integers(0, n, int(off[-1])).astype(np.uint32)    # any targets: only degrees matter
            gs.append(rl.HostGraph(off, tgt))
        hb = rl.HostBatch.concat(gs)
        ks = segmented_order(np.asarray(hb.offsets), np.asarray(hb.graph_offsets))
        for i, g in enumerate(gs):
            a, z = int(hb.graph_offsets[i]), int(hb.graph_offsets[i + 1])
            np.testing.assert_array_equal(ks[a:z], orc.ref_vertex_order(g), err_msg=f"trial {trial} graph {i}")
