"""Bit-exact parity at the sizes of the benchmark configurations, not only on small graphs.

- Config 1 (R-MAT scale 16, edge factor 16, unit weights, int32 CSR): complete synchronous runs
  against the oracle -- the exact mode (the reference CPU rules, rescan on) for νMG8 and νBM, and
  the split mode under both of the reference's rule sets, with the default layout and with one
  that splits the largest vertices into chunks.
- Configs 2a (R-MAT scale 24, edge factor 32, weights U[1,10), int32 CSR; 1.0 G edges) and 2b (the
  2^25-vertex lattice): one split-mode step from the labels the asynchronous mode starts from --
  positions in the reference GPU path's vertex order -- on a pickless iteration, as the reference's
  first iteration is (inc/rakLowmemCuda.hxx:473-476), against the oracle's step from the same
  labels; labels and next flags compared in full.
- A graph with more than 2^31 edges and int64 offsets (config 3: R-MAT scale 27, edge factor 16,
  4.2 G edges): one split-mode step, so that edge indexes, chunk starts and offsets beyond 32 bits
  are exercised, against the oracle.

The oracle decides the vertices of a step on all host cores (OpenMP); each decision reads only the
snapshot, so the result is the one-thread result."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.gpu

FORCED_SPLIT = dict(lane_max=32, hub_min=1024, hub_chunk=256)   # every regime, split chunks included


@pytest.fixture(scope="module")
def ctx():
    c = rl.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def config1():
    return rl.gen_rmat(16, 16, seed=42).with_offsets32()


def _layout(lay):
    return (lay["lane_max"], lay["hub_min"], lay["hub_chunk"]) if lay else orc.DEFAULT_LAYOUT


@pytest.mark.parametrize("slots", [8, 1])
def test_config1_sync_exact_run(ctx, config1, slots):
    g = config1
    lab, res = ctx.lowmem(g, mode=rl.MODE_SYNC, slots=slots)
    ref, it, edges = orc.sync_run(orc.Graph.of(g), orc.make_opts(slots=slots, rescan=1))
    assert res.iterations == it
    assert res.traversed_edges == edges
    np.testing.assert_array_equal(lab, ref)


@pytest.mark.parametrize("rule", [1, 2])
@pytest.mark.parametrize("layout", [None, FORCED_SPLIT], ids=["default", "forced_split"])
def test_config1_sync_split_run(ctx, config1, rule, layout):
    g = config1
    lab, res = ctx.lowmem(g, mode=rl.MODE_SYNC_SPLIT, slots=8, sketch_rule=rule, **(layout or {}))
    ref, it, edges = orc.sync_run(orc.Graph.of(g), orc.make_opts(slots=8, split=1, layout=_layout(layout),
                                                                 gpu_rule=1 if rule == 2 else 0))
    assert res.iterations == it
    assert res.traversed_edges == edges
    np.testing.assert_array_equal(lab, ref)


def _step_from_positions(ctx, csr, host, rule):
    """One pickless split-mode step from reference-order positions on the GPU and in the oracle."""
    import torch
    n = host.n
    ks = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.reference_vertex_order(csr, ks)
    ks_h = ks.cpu().numpy().view(np.uint32)
    pos = np.empty(n, np.uint32)
    pos[ks_h] = np.arange(n, dtype=np.uint32)
    ones = np.ones(n, np.uint8)
    rg = rl.ResidentGraph(ctx, csr)
    vp = torch.from_numpy(pos.view(np.int32)).cuda()
    ap = torch.from_numpy(ones).cuda()
    vn, an = torch.empty_like(vp), torch.empty_like(ap)
    ch = rg.step(0, vp, ap, vn, an, mode=rl.MODE_SYNC_SPLIT, slots=8, pickless_step=8, sketch_rule=rule)
    got_v, got_a = vn.cpu().numpy().view(np.uint32), an.cpu().numpy()
    rg.close()
    del vp, ap, vn, an, ks
    og = orc.Graph.of(host)
    rv, ra, rch, edges, processed = orc.sync_step(og, orc.make_opts(slots=8, split=1, pickless_step=8,
                                                                    gpu_rule=1 if rule == 2 else 0), 0, pos, ones)
    assert ch == rch
    np.testing.assert_array_equal(got_v, rv)
    np.testing.assert_array_equal(got_a, ra)
    return rch


def test_config2a_split_step_from_reference_positions(ctx):
    dg = rl.gen_rmat_device(ctx, 24, 32, 0.57, 0.19, 0.19, 42, 1.0, 10.0, offset_bits=32)
    try:
        host = dg.to_host()
        for rule in (1, 2):
            assert _step_from_positions(ctx, dg.csr, host, rule) > 0
    finally:
        dg.close()


def test_config2b_split_step_from_reference_positions(ctx):
    import torch
    g = rl.gen_lattice(8192, 4096, 0.05, 0.01, seed=42).with_offsets32()
    off = torch.from_numpy(np.ascontiguousarray(g.offsets)).cuda()
    tgt = torch.from_numpy(g.targets.view(np.int32)).cuda()
    csr = rl.device_csr(off, tgt, None)
    assert _step_from_positions(ctx, csr, g, 1) > 0


def test_more_than_2_31_edges_split_step(ctx):
    """R-MAT scale 27 / edge factor 16 with int64 offsets: m > 2^31, split vertices whose edges start
    beyond index 2^31. One split-mode step from vertex-id labels, every vertex affected."""
    import torch
    dg = rl.gen_rmat_device(ctx, 27, 16, 0.57, 0.19, 0.19, 42, 1.0, 1.0, offset_bits=64)
    try:
        assert dg.m > 2 ** 31
        host = dg.to_host()
        n = host.n
        assert int(host.offsets[n - 1]) > 2 ** 31
        rg = rl.ResidentGraph(ctx, dg.csr)
        ids = np.arange(n, dtype=np.uint32)
        vp = torch.from_numpy(ids.view(np.int32)).cuda()
        ap = torch.ones(n, dtype=torch.uint8, device="cuda")
        vn, an = torch.empty_like(vp), torch.empty_like(ap)
        ch = rg.step(3, vp, ap, vn, an, mode=rl.MODE_SYNC_SPLIT, slots=8, pickless_step=0)
        got_v, got_a = vn.cpu().numpy().view(np.uint32), an.cpu().numpy()
        rg.close()
        del vp, ap, vn, an
        rv, ra, rch, edges, _ = orc.sync_step(orc.Graph.of(host), orc.make_opts(slots=8, split=1), 3, ids,
                                              np.ones(n, np.uint8))
        assert edges == dg.m
        assert ch == rch and rch > 0
        np.testing.assert_array_equal(got_v, rv)
        np.testing.assert_array_equal(got_a, ra)
    finally:
        dg.close()
