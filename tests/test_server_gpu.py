"""Serving loop (rak_server_*): continuous batching with admission by a device-memory budget and
overlapping launches. Each request's result must be the same in the mix as alone (synchronous
mode: identical labels and iterations; asynchronous mode: the planted partitions recovered to
the same quality), oversized requests are refused, and a full queue answers busy."""
import threading

import numpy as np
import pytest

import rak_lowmem as rl

pytestmark = pytest.mark.gpu

LAYOUT = dict(lane_max=8, hub_min=64, hub_chunk=32)


@pytest.fixture(scope="module")
def ctx():
    c = rl.Context(0)
    yield c
    c.close()


def request_graphs():
    gs = [rl.gen_rmat(s, 6, seed=200 + s) for s in (8, 11, 9, 12, 10)]
    gs += [rl.gen_rmat(10, 8, seed=7, w_lo=1.0, w_hi=5.0), rl.gen_sbm(3000, 20, 12.0, 20.0, seed=3),
           rl.gen_lattice(30, 20, 0.05, 0.02, seed=4), rl.HostGraph(np.zeros(3, np.int64), np.zeros(0, np.uint32))]
    return gs * 3


def test_results_same_alone_and_in_the_mix(ctx):
    gs = request_graphs()
    alone = [ctx.lowmem(g, mode=rl.MODE_SYNC, **LAYOUT) for g in gs]
    srv = rl.Server(ctx, budget_bytes=64 << 20, max_graphs_per_launch=5, slots=2, mode=rl.MODE_SYNC, **LAYOUT)
    tickets = [None] * len(gs)

    def client(idx):
        for i in idx:
            tickets[i] = srv.submit(gs[i])

    th = [threading.Thread(target=client, args=(range(k, len(gs), 2),)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i, g in enumerate(gs):
        lab, res = srv.wait(tickets[i])
        np.testing.assert_array_equal(lab, alone[i][0], err_msg=f"request {i}")
        assert res.iterations == alone[i][1].iterations
        assert res.time_ms >= res.plan_ms >= 0
    st = srv.stats()
    assert st["completed"] == st["submitted"] == len(gs) and st["rejected"] == 0
    assert st["launches"] >= len(gs) // 5 and st["device_bytes_in_use"] == 0
    srv.close()


@pytest.mark.parametrize("label_order", [0, 2])
def test_async_quality_in_the_mix(ctx, label_order):
    """Default labels (ids) and the reference label order, rebuilt for every packed set of graphs;
    a grid-numbered lattice in the mix finds its local structure with the reference order."""
    gs = [rl.gen_sbm(4000 + 1000 * k, 20, 16.0, 1000.0, seed=k) for k in range(8)]
    lat = rl.gen_lattice(200, 150, 0.05, 0.01, seed=5)
    srv = rl.Server(ctx, max_graphs_per_launch=3, slots=2, label_order=label_order)
    ts = [srv.submit(g) for g in gs]
    tl = srv.submit(lat)
    import oracle as orc
    for t, g in zip(ts, gs):
        lab, res = srv.wait(t)
        assert lab.max() < g.n and res.iterations >= 1
        planted = orc.modularity(orc.Graph.of(g), g.truth)
        assert orc.modularity(orc.Graph.of(g), lab) >= 0.85 * planted
    lab, res = srv.wait(tl)
    assert lab.max() < lat.n
    if label_order == 2:
        assert orc.modularity(orc.Graph.of(lat), lab) > 0.4
    srv.close()


def test_launches_overlap_under_load(ctx):
    gs = [rl.gen_rmat(14, 16, seed=300 + i) for i in range(6)]
    srv = rl.Server(ctx, max_graphs_per_launch=1, slots=2)
    ts = [srv.submit(g) for g in gs * 4]
    for t in ts:
        srv.wait(t)
    st = srv.stats()
    assert st["launches"] == len(ts) and st["max_concurrent_launches"] == 2
    srv.close()


def test_oversized_request_refused_others_served(ctx):
    big = rl.gen_rmat(14, 16, seed=1)
    small = rl.gen_rmat(7, 4, seed=2)
    srv = rl.Server(ctx, budget_bytes=1 << 20, slots=1)
    tb, ts = srv.submit(big), srv.submit(small)
    with pytest.raises(rl.RakError) as e:
        srv.wait(tb)
    assert e.value.status == 3
    lab, _ = srv.wait(ts)
    assert len(lab) == small.n
    assert srv.stats()["rejected"] == 1
    srv.close()


def test_full_queue_is_busy(ctx):
    first = rl.gen_rmat(16, 16, seed=5)
    small = rl.gen_rmat(6, 4, seed=6)
    srv = rl.Server(ctx, max_graphs_per_launch=1, slots=1, queue_capacity=2)
    tickets, busy = [srv.submit(first)], 0
    for _ in range(20):
        try:
            tickets.append(srv.submit(small))
        except rl.RakError as e:
            assert e.status == 8
            busy += 1
    assert busy > 0
    for t in tickets:
        srv.wait(t)
    srv.close()


def device_graph(g):
    import torch
    off = torch.from_numpy(np.ascontiguousarray(g.offsets)).cuda()
    tgt = torch.from_numpy(g.targets.view(np.int32)).cuda()
    wt = torch.from_numpy(g.weights).cuda() if g.weights is not None else None
    return (off, tgt, wt), rl.device_csr(off, tgt, wt)


def test_device_requests_same_as_host_requests(ctx):
    """Graphs kept in device memory (an arena) are packed by the gather kernel; their results
    equal those of the same graphs submitted from the host, and of each graph alone."""
    gs = request_graphs()
    alone = [ctx.lowmem(g, mode=rl.MODE_SYNC, **LAYOUT) for g in gs]
    arena = [device_graph(g) for g in gs]
    srv = rl.Server(ctx, max_graphs_per_launch=4, slots=2, mode=rl.MODE_SYNC, **LAYOUT)
    ts = []
    for i, g in enumerate(gs):          # host and device requests interleaved in the same launches
        keep, csr = arena[i]
        ts.append(srv.submit_device(csr, keep) if i % 3 else srv.submit(g))
    for i, t in enumerate(ts):
        lab, res = srv.wait(t)
        np.testing.assert_array_equal(lab, alone[i][0], err_msg=f"request {i}")
        assert res.iterations == alone[i][1].iterations
    st = srv.stats()
    assert st["completed"] == len(gs) and st["rejected"] == 0 and st["device_bytes_in_use"] == 0
    srv.close()


def test_invalid_device_graph_fails_others_served(ctx):
    import torch
    good = [rl.gen_rmat(9, 6, seed=40 + i) for i in range(3)]
    alone = [ctx.lowmem(g, mode=rl.MODE_SYNC, **LAYOUT)[0] for g in good]
    bad_tgt = good[0].targets.copy()
    bad_tgt[len(bad_tgt) // 2] = good[0].n          # one target out of range
    bad_off = good[1].offsets.copy()
    bad_off[5], bad_off[6] = bad_off[6], bad_off[5] - 1   # offsets decrease
    bads = []
    for off, tgt in ((good[0].offsets, bad_tgt), (bad_off, good[1].targets)):
        o = torch.from_numpy(np.ascontiguousarray(off)).cuda()
        t = torch.from_numpy(tgt.view(np.int32)).cuda()
        bads.append(((o, t), rl.device_csr(o, t, None)))
    srv = rl.Server(ctx, max_graphs_per_launch=8, slots=1, mode=rl.MODE_SYNC, **LAYOUT)
    ts_bad = [srv.submit_device(csr, keep) for keep, csr in bads]
    arena = [device_graph(g) for g in good]
    ts_good = [srv.submit_device(csr, keep) for keep, csr in arena]
    for t in ts_bad:
        with pytest.raises(rl.RakError) as e:
            srv.wait(t)
        assert e.value.status == 2
    for t, want in zip(ts_good, alone):
        lab, _ = srv.wait(t)
        np.testing.assert_array_equal(lab, want)
    st = srv.stats()
    assert st["rejected"] == 2 and st["completed"] == 3 and st["device_bytes_in_use"] == 0
    srv.close()
