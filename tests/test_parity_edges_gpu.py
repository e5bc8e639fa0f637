"""Parity on inputs at the edges of the domain, bit for bit against the oracle:

- multigraph CSRs: duplicate edges, self-loops and zero-weight edges (nothing in the C ABI requires
  a simple graph; the reference's per-vertex loops take the CSR as it is);
- vertices whose degrees sit exactly on the region boundaries of the default split layout
  (lane_max, G*lane_max for every group size, hub_min) and on split-chunk boundaries above hub_min;
- the Boyer-Moore sketch (slots 1) and small sketches on the same inputs.

Synchronous exact mode is compared with the oracle's exact scan, synchronous split mode with its
restatement of the split layout (default layout, so the split-vertex path with its arrival counters
and partial sketches is exercised at the library's own thresholds)."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.gpu

LANE_MAX, HUB_MIN, HUB_CHUNK = orc.DEFAULT_LAYOUT


@pytest.fixture(scope="module")
def ctx():
    c = rl.Context(0)
    yield c
    c.close()


def symmetric_csr(n, pairs, weights=None, keep_duplicates=False):
    """CSR over n vertices from undirected (u, v) pairs, both directions stored, targets sorted per
    vertex; duplicates kept when asked (a multigraph), self-loops stored once."""
    u, v = pairs[:, 0].astype(np.int64), pairs[:, 1].astype(np.int64)
    w = np.ones(len(u), np.float32) if weights is None else weights.astype(np.float32)
    loop = u == v
    src = np.concatenate([u, v[~loop]])
    dst = np.concatenate([v, u[~loop]])
    ww = np.concatenate([w, w[~loop]])
    order = np.lexsort((dst, src))
    src, dst, ww = src[order], dst[order], ww[order]
    if not keep_duplicates:
        keep = np.ones(len(src), bool)
        keep[1:] = (src[1:] != src[:-1]) | (dst[1:] != dst[:-1])
        src, dst, ww = src[keep], dst[keep], ww[keep]
    off = np.zeros(n + 1, np.int64)
    np.add.at(off, src + 1, 1)
    off = np.cumsum(off)
    return rl.HostGraph(off, dst.astype(np.uint32), None if weights is None else ww)


def multigraph():
    rng = np.random.default_rng(11)
    n = 3000
    base = rng.integers(0, n, size=(12000, 2))
    blocks = rng.integers(0, 30, size=n)                       # a planted structure to move towards
    inside = rng.integers(0, n, size=(20000, 2))
    inside = inside[blocks[inside[:, 0]] == blocks[inside[:, 1]]]
    dup = base[rng.integers(0, len(base), size=3000)]          # repeated pairs
    loops = np.repeat(rng.integers(0, n, size=(400, 1)), 2, axis=1)
    pairs = np.concatenate([base, inside, dup, loops])
    w = rng.uniform(1.0, 5.0, size=len(pairs)).astype(np.float32)
    w[rng.random(len(pairs)) < 0.05] = 0.0                     # zero-weight edges
    return symmetric_csr(n, pairs, w, keep_duplicates=True)


def degree_ladder():
    """Centre vertices with degrees on every region boundary of the default layout, each joined to
    distinct leaves; leaves also link among themselves so that they carry labels worth moving to."""
    degs = [LANE_MAX - 1, LANE_MAX, LANE_MAX + 1]
    for G in (2, 4, 8, 16, 32):
        degs += [G * LANE_MAX, G * LANE_MAX + 1]
    degs += [HUB_MIN, HUB_MIN + 1, HUB_MIN + HUB_CHUNK, HUB_MIN + HUB_CHUNK + 1]
    degs = sorted(set(d for d in degs if d > 1))
    leaves = 2 * max(degs)
    n = len(degs) + leaves
    rng = np.random.default_rng(5)
    pairs = []
    for i, d in enumerate(degs):
        nb = len(degs) + rng.choice(leaves, size=d, replace=False)
        pairs.append(np.stack([np.full(d, i), nb], 1))
    ring = np.arange(leaves)
    pairs.append(np.stack([len(degs) + ring, len(degs) + (ring + 1) % leaves], 1))
    pairs.append(np.stack([len(degs) + ring, len(degs) + rng.integers(0, leaves, leaves)], 1))
    g = symmetric_csr(n, np.concatenate(pairs))
    d = np.diff(g.offsets)
    for i, want in enumerate(degs):                            # the boundaries are really hit
        assert d[i] >= want
    return g


def check_sync(ctx, g, slots, rescan, split, gpu_rule=0):
    o = orc.make_opts(slots=slots, rescan=rescan, split=split, layout=orc.DEFAULT_LAYOUT, gpu_rule=gpu_rule)
    ref, it, edges = orc.sync_run(orc.Graph.of(g), o)
    mode = rl.MODE_SYNC_SPLIT if split else rl.MODE_SYNC
    lab, res = ctx.lowmem(g, mode=mode, slots=slots, rescan=rescan, sketch_rule=2 if gpu_rule else 1)
    assert res.iterations == it
    np.testing.assert_array_equal(lab, ref)
    assert res.traversed_edges == edges


@pytest.mark.parametrize("slots,rescan", [(8, 1), (8, 0), (4, 0), (1, 0)])
def test_multigraph_sync_exact(ctx, slots, rescan):
    check_sync(ctx, multigraph(), slots, rescan, split=0)


@pytest.mark.parametrize("slots", [8, 2, 1])
@pytest.mark.parametrize("gpu_rule", [0, 1])
def test_multigraph_sync_split(ctx, slots, gpu_rule):
    check_sync(ctx, multigraph(), slots, 0, split=1, gpu_rule=gpu_rule)


@pytest.mark.parametrize("slots", [8, 1])
@pytest.mark.parametrize("gpu_rule", [0, 1])
def test_degree_boundaries_sync_split_default_layout(ctx, slots, gpu_rule):
    g = degree_ladder()
    summary = rl.plan_summary(g)
    assert summary[0][6] >= 2                                  # split vertices exist at the default layout
    check_sync(ctx, g, slots, 0, split=1, gpu_rule=gpu_rule)


def test_degree_boundaries_sync_exact(ctx):
    check_sync(ctx, degree_ladder(), 8, 1, split=0)


@pytest.mark.parametrize("slots", [8, 1])
def test_edge_inputs_async_valid(ctx, slots):
    for g in (multigraph(), degree_ladder()):
        lab, res = ctx.lowmem(g, slots=slots, compute_modularity=1)
        assert lab.max() < g.n and res.iterations >= 1
        q_oracle = orc.modularity(orc.Graph.of(g), lab)
        assert res.modularity == pytest.approx(q_oracle, rel=1e-9, abs=1e-12)


def _device_csr_at(g, shift):
    """g on the device with its targets (and weights) starting `shift` elements into a buffer, so
    the arrays are 4-byte but not 16-byte aligned when shift % 4 != 0."""
    import torch
    off = torch.from_numpy(np.ascontiguousarray(g.offsets)).cuda()
    tbuf = torch.zeros(g.m + shift, dtype=torch.int32, device="cuda")
    tbuf[shift:] = torch.from_numpy(g.targets.view(np.int32)).cuda()
    tgt = tbuf[shift:]
    wt = None
    if g.weights is not None:
        wbuf = torch.zeros(g.m + shift, dtype=torch.float32, device="cuda")
        wbuf[shift:] = torch.from_numpy(g.weights).cuda()
        wt = wbuf[shift:]
    return (off, tbuf, tgt, wt), rl.device_csr(off, tgt, wt)


@pytest.mark.parametrize("shift", [0, 1, 3])
@pytest.mark.parametrize("mode", [rl.MODE_SYNC, rl.MODE_SYNC_SPLIT])
def test_unaligned_edge_arrays(ctx, shift, mode):
    """One-lane vertices read their edge lists in 16-byte vectors when the target and weight arrays
    are 16-byte aligned, and element by element otherwise: the labels are the oracle's either way
    (weighted R-MAT, one-lane lists both shorter and longer than the vector threshold)."""
    import torch
    g = rl.gen_rmat(13, 16, seed=31, w_lo=1.0, w_hi=10.0)
    keep, csr = _device_csr_at(g, shift)
    assert (keep[2].data_ptr() % 16 == 0) == (shift % 4 == 0)
    for slots in (8, 1):
        o = orc.make_opts(slots=slots, rescan=1 if mode == rl.MODE_SYNC else 0,
                          split=1 if mode == rl.MODE_SYNC_SPLIT else 0, layout=orc.DEFAULT_LAYOUT)
        ref, it, edges = orc.sync_run(orc.Graph.of(g), o)
        out = torch.empty(g.n, dtype=torch.int32, device="cuda")
        res = ctx.lowmem_device(csr, out, mode=mode, slots=slots)
        np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), ref)
        assert res.iterations == it and res.traversed_edges == edges
