"""The replica path of bench.py (--gpus N under torch.distributed.run), exercised on CPU with the
gloo backend and 2 ranks: the whole-job aggregation takes the slowest rank's time and the sum of
every rank's work, and the reference arm runs on rank 0 only (the other ranks exit without work)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        assert bench.dist_setup() == (world, rank, rank)
        seconds = 1.0 + rank            # rank 1 is the slowest
        units = 100 * (rank + 1)
        t, u = bench.whole_job(dist, seconds, units, "cpu")
        out.put((rank, t, u))
        # the reference arm: rank 0 alone does work; others return at once
        class A:
            steps, warmup, workload = 1, 3, "rmat16_ef16"
        if rank != 0:
            assert bench.run_reference(A, bench.WORKLOADS["rmat16_ef16"], world, rank) is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_whole_job_aggregation_two_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(out.get(timeout=5) for _ in range(2))
    for rank, t, u in got:
        assert t == pytest.approx(2.0) and u == pytest.approx(300.0)


def test_single_process_is_local():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.whole_job(None, 2.5, 7, "cpu") == (2.5, 7.0)


def test_batch_mix_shares_are_the_full_mix():
    """The batched leg deals graph i to rank i mod N: each rank's share, built on its own, is the
    same graphs as those positions of the full mix."""
    sys.path.insert(0, ROOT)
    import numpy as np
    import bench
    full = bench.batch_mix(6, 4, 4)
    for rank in range(2):
        part = bench.batch_mix(6, 4, 4, keep=lambda i: i % 2 == rank)
        assert len(part) == 3
        for j, g in enumerate(part):
            f = full[2 * j + rank]
            np.testing.assert_array_equal(g.offsets, f.offsets)
            np.testing.assert_array_equal(g.targets, f.targets)


def _serving_rank(rank, world, port, out):
    import datetime
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = bench.my_requests(101, world, rank)
        rng = np.random.default_rng(rank)
        part = {"lat": list(rng.random(len(mine)) * (rank + 1)), "queued": [0.5] * len(mine),
                "span": 1.0 + rank, "edges": 10 * len(mine), "q": {rank: 0.5 + rank}}
        parts = bench.gather_objects(dist, part)
        out.put((rank, mine, parts, bench.merge_serving(parts)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_serving_requests_dealt_and_merged_two_ranks():
    """Serving sharded by request: ranks take disjoint shares that cover the stream, every rank
    receives every rank's results, and the merge takes percentiles over all requests, the slowest
    rank's span and summed counts."""
    import numpy as np
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serving_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted((out.get(timeout=5) for _ in range(2)), key=lambda x: x[0])
    shares = [set(m) for _, m, _, _ in got]
    assert shares[0].isdisjoint(shares[1]) and shares[0] | shares[1] == set(range(101))
    parts0, merged0 = got[0][2], got[0][3]
    assert [len(p["lat"]) for p in parts0] == [51, 50] and merged0 == got[1][3]
    lat = np.concatenate([p["lat"] for p in parts0])
    assert merged0["requests"] == 101 and merged0["span_s"] == 2.0 and merged0["ranks"] == 2
    assert merged0["p99_ms"] == pytest.approx(float(np.percentile(lat, 99)))
    assert merged0["graphs_per_s"] == pytest.approx(101 / 2.0) and merged0["edges_per_s"] == pytest.approx(1010 / 2.0)
