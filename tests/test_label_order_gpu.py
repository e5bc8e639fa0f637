"""Label order of the asynchronous mode: labels are positions in the reference GPU path's vertex
order (inc/rakLowmemCuda.hxx:505-519, 563) -- the order its pickless rule compares -- and come
back as vertex ids. The device restatement of that order must equal the reference's own two
std::partition calls (oracle bridge), for one graph and for every graph of a batch (each graph
partitioned on its own), and lattice-like graphs, whose ids follow the grid, must not stall under
the pickless rule, alone or batched."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not orc.have_ref_cpu(), reason="oracle/_ref not built")]


@pytest.fixture(scope="module")
def ctx():
    c = rl.Context(0)
    yield c
    c.close()


def _dense(n):
    rows = [np.array([v for v in range(n) if v != u], np.uint32) for u in range(n)]
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum([len(r) for r in rows])
    return rl.HostGraph(off, np.concatenate(rows))


CASES = {
    "rmat14": lambda: rl.gen_rmat(14, 8, seed=3),
    "sbm": lambda: rl.gen_sbm(20000, 50, 12.0, 30.0, seed=4),
    "lattice": lambda: rl.gen_lattice(200, 150, 0.05, 0.01, seed=5),
    "dense200": lambda: _dense(200),                       # every degree >= 128
    "path": lambda: rl.gen_lattice(1, 500, 0.0, 0.0, seed=6),   # every degree < 4
    "single": lambda: rl.HostGraph(np.zeros(2, np.int64), np.zeros(0, np.uint32)),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("bits", [32, 64])
def test_order_equals_reference_partition(ctx, name, bits):
    import torch
    g = CASES[name]()
    off = torch.from_numpy(g.offsets.astype(np.int64 if bits == 64 else np.int32)).cuda()
    tgt = torch.from_numpy(g.targets.view(np.int32)).cuda()
    ks = torch.empty(g.n, dtype=torch.int32, device="cuda")
    ctx.reference_vertex_order(rl.device_csr(off, tgt, None), ks)
    np.testing.assert_array_equal(ks.cpu().numpy().view(np.uint32), orc.ref_vertex_order(g))


@pytest.mark.parametrize("slots", [8, 1])
def test_lattice_does_not_stall(ctx, slots):
    """Grid-ordered ids: with the reference's label order both sketches find the lattice's local
    structure (id labels let the pickless rule block most first moves for Boyer-Moore)."""
    g = rl.gen_lattice(512, 512, 0.05, 0.01, seed=7)
    lab, res = ctx.lowmem(g, slots=slots, compute_modularity=1)
    assert lab.max() < g.n and res.iterations >= 3
    assert res.modularity > 0.4, res


def test_label_order_options(ctx):
    g = rl.gen_rmat(11, 8, seed=8)
    for order in (1, 2):
        lab, res = ctx.lowmem(g, label_order=order, compute_modularity=1)
        assert lab.max() < g.n and res.modularity == pytest.approx(orc.modularity(orc.Graph.of(g), lab), rel=1e-9, abs=1e-12)
    with pytest.raises(rl.RakError) as e:
        ctx.lowmem(g, mode=rl.MODE_SYNC, label_order=2)
    assert e.value.status == 7


def test_batch_order_equals_reference_partition_per_graph(ctx):
    import torch
    gs = [CASES[k]() for k in sorted(CASES)] + [rl.gen_rmat(12, 16, seed=9), CASES["path"]()]
    hb = rl.HostBatch.concat(gs)
    b = rl.Batch(ctx, hb)
    ks = torch.full((hb.n,), -1, dtype=torch.int32, device="cuda")
    b.reference_vertex_order(ks)
    got = ks.cpu().numpy().view(np.uint32)
    for i, g in enumerate(gs):
        a, z = int(hb.graph_offsets[i]), int(hb.graph_offsets[i + 1])
        np.testing.assert_array_equal(got[a:z], orc.ref_vertex_order(g), err_msg=f"graph {i}")
    b.close()


@pytest.mark.parametrize("slots", [8, 1])
def test_batched_lattice_does_not_stall(ctx, slots):
    """With label_order 2 a batch runs each graph in its own reference order, like a single graph
    (batches default to id labels)."""
    import torch
    gs = [rl.gen_lattice(256, 256, 0.05, 0.01, seed=11), rl.gen_rmat(12, 16, seed=12),
          rl.gen_lattice(300, 200, 0.05, 0.01, seed=13)]
    hb = rl.HostBatch.concat(gs)
    b = rl.Batch(ctx, hb)
    out = torch.empty(hb.n, dtype=torch.int32, device="cuda")
    b.launch(out, slots=slots, label_order=2)
    b.results()
    q = b.modularity(out)
    lab = out.cpu().numpy().view(np.uint32)
    for i, g in enumerate(gs):
        a, z = int(hb.graph_offsets[i]), int(hb.graph_offsets[i + 1])
        assert lab[a:z].max() < g.n
        assert q[i] == pytest.approx(orc.modularity(orc.Graph.of(g), lab[a:z]), rel=1e-9, abs=1e-12)
    assert q[0] > 0.4 and q[2] > 0.4, q
    b.close()


@pytest.mark.parametrize("rule", [1, 2])
@pytest.mark.parametrize("name", ["rmat12", "lattice"])
def test_sync_split_from_reference_positions_matches_oracle(ctx, rule, name):
    """The reference label order run deterministically: the synchronous split mode started from the
    reference's positions as initial labels (q) -- the labels the pickless rule then compares --
    equals the oracle's synchronous run from the same labels, bit for bit, under either rule set."""
    g = rl.gen_rmat(12, 8, seed=21) if name == "rmat12" else rl.gen_lattice(120, 90, 0.05, 0.01, seed=22)
    ks = orc.ref_vertex_order(g)
    pos = np.empty_like(ks)
    pos[ks] = np.arange(len(ks), dtype=np.uint32)
    lab, res = ctx.lowmem(g, q=pos, mode=rl.MODE_SYNC_SPLIT, sketch_rule=rule)
    o = orc.make_opts(slots=8, rescan=0, split=1, layout=orc.DEFAULT_LAYOUT, gpu_rule=1 if rule == 2 else 0)
    ref, it, edges = orc.sync_run(orc.Graph.of(g), o, q=pos)
    assert res.iterations == it
    np.testing.assert_array_equal(lab, ref)
    assert res.traversed_edges == edges
