"""Batched persistent launch (rak_batch_*) on the GPU: every graph of a batch gets exactly what
running it alone gives (synchronous modes, against the oracle, per graph), capture/replay in a CUDA
graph reproduces the launch, per-graph modularity matches, and invalid batches are refused."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.gpu

LAYOUT = dict(lane_max=8, hub_min=64, hub_chunk=32)   # forces every work region on small graphs


def mixed_graphs(weighted):
    lo, hi = (1.0, 9.0) if weighted else (1.0, 1.0)
    gs = [rl.gen_rmat(s, 6, seed=100 + s, w_lo=lo, w_hi=hi) for s in (6, 9, 10, 7)]
    gs += [rl.gen_sbm(800, 8, 10.0, 20.0, seed=5), rl.gen_lattice(20, 15, 0.05, 0.02, seed=6)]
    gs += [rl.HostGraph(np.zeros(4, np.int64), np.zeros(0, np.uint32))]        # isolated vertices only
    if weighted:
        gs = [g if g.weights is not None else rl.HostGraph(g.offsets, g.targets, np.ones(g.m, np.float32))
              for g in gs]
    return gs


@pytest.fixture(scope="module")
def ctx():
    c = rl.Context(0)
    yield c
    c.close()


def run_batch(ctx, hb, **opts):
    import torch
    b = rl.Batch(ctx, hb, **{k: v for k, v in opts.items() if k in LAYOUT})
    out = torch.empty(hb.n, dtype=torch.int32, device="cuda")
    b.launch(out, **opts)
    it, tot = b.results()
    return b, out.cpu().numpy().view(np.uint32), it, tot


@pytest.mark.parametrize("weighted", [False, True])
@pytest.mark.parametrize("mode,slots,rescan", [(rl.MODE_SYNC, 8, 1), (rl.MODE_SYNC, 1, 0),
                                               (rl.MODE_SYNC_SPLIT, 8, 0), (rl.MODE_SYNC_SPLIT, 4, 0)])
def test_batch_equals_graphs_alone(ctx, weighted, mode, slots, rescan):
    gs = mixed_graphs(weighted)
    hb = rl.HostBatch.concat(gs)
    b, lab, it, tot = run_batch(ctx, hb, mode=mode, slots=slots, rescan=rescan, **LAYOUT)
    edges = 0
    for i, g in enumerate(gs):
        o = orc.make_opts(slots=slots, rescan=rescan, split=1 if mode == rl.MODE_SYNC_SPLIT else 0,
                          layout=(LAYOUT["lane_max"], LAYOUT["hub_min"], LAYOUT["hub_chunk"]))
        ref, rit, e = orc.sync_run(orc.Graph.of(g), o)
        a, z = int(hb.graph_offsets[i]), int(hb.graph_offsets[i + 1])
        np.testing.assert_array_equal(lab[a:z], ref, err_msg=f"graph {i}")
        assert it[i] == rit, (i, it[i], rit)
        edges += e
    assert tot.traversed_edges == edges
    assert tot.iterations == it.max()
    b.close()


def test_batch_async_valid_and_modularity(ctx):
    # well-separated planted partitions: asynchronous LPA recovers them alone and in the batch (the
    # asynchronous order varies from run to run, so the floor leaves room for one merged block)
    import torch
    gs = [rl.gen_sbm(2000 + 500 * k, 10 + k, 16.0, 1000.0, seed=k) for k in range(6)] + \
         [rl.gen_rmat(10, 8, seed=9)]
    hb = rl.HostBatch.concat(gs)
    b, lab, it, tot = run_batch(ctx, hb)
    q = b.modularity(torch.from_numpy(lab.view(np.int32)).cuda())
    for i, g in enumerate(gs):
        a, z = int(hb.graph_offsets[i]), int(hb.graph_offsets[i + 1])
        assert lab[a:z].max() < g.n and 1 <= it[i] <= 20
        assert q[i] == pytest.approx(orc.modularity(orc.Graph.of(g), lab[a:z]), rel=1e-9, abs=1e-12)
        if g.truth is not None:
            planted = orc.modularity(orc.Graph.of(g), g.truth)
            solo, res = ctx.lowmem(g, compute_modularity=1)
            assert res.modularity >= 0.85 * planted and q[i] >= 0.85 * planted, (i, q[i], res.modularity, planted)
    b.close()


def test_batch_capture_replay(ctx):
    import torch
    gs = mixed_graphs(False)
    hb = rl.HostBatch.concat(gs)
    b = rl.Batch(ctx, hb, **LAYOUT)
    ref = torch.empty(hb.n, dtype=torch.int32, device="cuda")
    b.launch(ref, mode=rl.MODE_SYNC_SPLIT, **LAYOUT)
    it_ref, _ = b.results()
    out = torch.full((hb.n,), -1, dtype=torch.int32, device="cuda")
    b.capture(out, mode=rl.MODE_SYNC_SPLIT, **LAYOUT)
    for _ in range(3):
        out.fill_(-1)
        torch.cuda.synchronize()
        b.replay()
        it, _ = b.results()
        assert torch.equal(out, ref)
        np.testing.assert_array_equal(it, it_ref)
    b.close()


def test_batch_rejects_bad_local_ids(ctx):
    gs = mixed_graphs(False)[:3]
    hb = rl.HostBatch.concat(gs)
    t = hb.targets.copy()
    t[0] = gs[0].n                       # a valid global id but beyond graph 0
    bad = rl.HostBatch(hb.graph_offsets, hb.offsets, t)
    with pytest.raises(rl.RakError) as e:
        rl.Batch(ctx, bad)
    assert e.value.status == 2


def test_batch_label_orders(ctx):
    """Asynchronous batches run with either label order (ids by default, the reference order on
    request) and captured launches replay with it; the synchronous modes label by id only."""
    import torch
    gs = mixed_graphs(False)[:3]
    hb = rl.HostBatch.concat(gs)
    b = rl.Batch(ctx, hb)
    out = torch.empty(hb.n, dtype=torch.int32, device="cuda")
    for order in (1, 2):
        b.launch(out, label_order=order)
        it, _ = b.results()
        lab = out.cpu().numpy().view(np.uint32)
        for i, g in enumerate(gs):
            a, z = int(hb.graph_offsets[i]), int(hb.graph_offsets[i + 1])
            assert lab[a:z].max() < g.n and it[i] >= 1
    b.capture(out, label_order=2)
    for _ in range(2):
        out.fill_(-1)
        b.replay()
        it, _ = b.results()
        assert int(out.min()) >= 0 and (it >= 1).all()
    with pytest.raises(rl.RakError) as e:
        b.launch(out, mode=rl.MODE_SYNC_SPLIT, label_order=2)
    assert e.value.status == 7
    b.close()
