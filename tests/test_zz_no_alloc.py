"""rak_lowmem_cuda_noalloc: the entry point for callers that cannot allocate device memory -- for
example a process whose device memory is already held by a framework's pooling allocator, or a
latency-critical loop that must not pay cudaMalloc/cudaFree's device synchronisation. It works in
the library's fixed device array instead of allocating.

Checked through the C ABI against the allocating entry point rak_lowmem_cuda on the same
device-located graphs, twice in a row (the array keeps the previous call's contents, so the second
call shows that everything that must start from zero is cleared). The synchronous modes are
deterministic, so the labels must be identical; the split mode exercises the split-vertex partial
sketches and arrival counters that live in the array. The default asynchronous mode is checked for
valid labels and modularity, and a repeated call for unchanged free device memory.
"""
import numpy as np
import pytest

import rak_lowmem as rl

pytestmark = pytest.mark.gpu

SPLIT_LAYOUT = dict(lane_max=8, hub_min=64, hub_chunk=32)


def device_graph(g):
    import torch
    off = torch.from_numpy(np.ascontiguousarray(g.offsets)).cuda()
    tgt = torch.from_numpy(g.targets.view(np.int32)).cuda()
    wt = torch.from_numpy(g.weights).cuda() if g.weights is not None else None
    return (off, tgt, wt), rl.device_csr(off, tgt, wt)


CASES = [
    ("rmat12_split8", lambda: rl.gen_rmat(12, 8, seed=21), dict(mode=rl.MODE_SYNC_SPLIT, slots=8, **SPLIT_LAYOUT)),
    ("rmat12w_split4", lambda: rl.gen_rmat(12, 8, seed=22, w_lo=1.0, w_hi=10.0),
     dict(mode=rl.MODE_SYNC_SPLIT, slots=4, **SPLIT_LAYOUT)),
    ("rmat13w_exact8", lambda: rl.gen_rmat(13, 8, seed=23, w_lo=1.0, w_hi=10.0), dict(mode=rl.MODE_SYNC, slots=8)),
    ("sbm_split_bm", lambda: rl.gen_sbm(20000, 40, 12.0, 20.0, seed=24), dict(mode=rl.MODE_SYNC_SPLIT, slots=1,
                                                                             **SPLIT_LAYOUT)),
]


@pytest.mark.parametrize("name,make,opts", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_allocating_entry_point(name, make, opts):
    import torch
    g = make()
    keep, csr = device_graph(g)
    with rl.Context(0) as ctx:
        want = torch.empty(g.n, dtype=torch.int32, device="cuda")
        ref = ctx.lowmem_device(csr, want, compute_modularity=1, **opts)
    stream = torch.cuda.Stream()
    for call in range(2):
        got = torch.full((g.n,), -1, dtype=torch.int32, device="cuda")
        res = rl.lowmem_noalloc(0, stream.cuda_stream, csr, got, compute_modularity=1, **opts)
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"{name}: call {call} differs from rak_lowmem_cuda"
        assert res.iterations == ref.iterations
        assert res.traversed_edges == ref.traversed_edges
        assert res.modularity == pytest.approx(ref.modularity, rel=1e-9, abs=1e-12)
        assert 0 < res.peak_device_bytes <= rl.NOALLOC_SCRATCH_BYTES


def test_noalloc_refuses_graphs_beyond_the_array():
    import torch
    n = 4 << 20                                   # ~20 bytes per vertex needed: more than 64 MiB
    off = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    tgt = torch.zeros(1, dtype=torch.int32, device="cuda")
    csr = rl.rak_csr(n, 0, 64, rl.DEVICE, off.data_ptr(), tgt.data_ptr(), None)
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    with pytest.raises(rl.RakError) as e:
        rl.lowmem_noalloc(0, None, csr, out)
    assert e.value.status == 3
    assert "bytes of scratch" in str(e.value)


def test_noalloc_async_default_is_valid_and_matches_quality():
    """The default asynchronous mode (id labels, in-place updates) is not deterministic:
    its labels must be valid vertex ids and its modularity close to the allocating entry point's."""
    import torch
    g = rl.gen_sbm(20000, 40, 12.0, 20.0, seed=26)
    keep, csr = device_graph(g)
    with rl.Context(0) as ctx:
        want = torch.empty(g.n, dtype=torch.int32, device="cuda")
        ref = ctx.lowmem_device(csr, want, compute_modularity=1)
    for call in range(2):
        got = torch.full((g.n,), -1, dtype=torch.int32, device="cuda")
        res = rl.lowmem_noalloc(0, None, csr, got, compute_modularity=1)
        torch.cuda.synchronize()
        lab = got.cpu().numpy()
        assert lab.min() >= 0 and lab.max() < g.n, f"call {call}: labels outside the vertex ids"
        assert res.iterations >= 1
        assert res.modularity == pytest.approx(ref.modularity, rel=0.02), (call, res.modularity, ref.modularity)


def test_noalloc_label_orders():
    import torch
    g = rl.gen_rmat(10, 8, seed=25)
    keep, csr = device_graph(g)
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    with pytest.raises(rl.RakError) as e:        # synchronous modes label by id, as rak_lowmem_cuda
        rl.lowmem_noalloc(0, None, csr, out, mode=rl.MODE_SYNC, label_order=2)
    assert e.value.status == 7
    for order in (1, 2):
        res = rl.lowmem_noalloc(0, None, csr, out, label_order=order, sketch_rule=2)
        torch.cuda.synchronize()
        assert res.iterations >= 1 and 0 <= int(out.min()) and int(out.max()) < g.n


def test_noalloc_second_call_takes_no_device_memory():
    """After a first call of a variant (which may load that variant's code onto the device), a
    second identical call leaves the device's free memory unchanged."""
    import torch
    g = rl.gen_rmat(12, 8, seed=27, w_lo=1.0, w_hi=10.0)
    keep, csr = device_graph(g)
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    opts = dict(mode=rl.MODE_SYNC_SPLIT, slots=8, compute_modularity=1, **SPLIT_LAYOUT)
    rl.lowmem_noalloc(0, None, csr, out, **opts)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    rl.lowmem_noalloc(0, None, csr, out, **opts)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
