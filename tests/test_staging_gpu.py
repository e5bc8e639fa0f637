"""Edge tiles staged in shared memory by bulk copies (rak_options.edge_staging 1: vertices scanned by
a whole warp -- lane groups of 32 and split-vertex chunks -- in the asynchronous and split modes).
Bulk copies need 16-byte aligned addresses, so a range's first and last few edges are read from
global memory directly, and a launch whose target and weight arrays differ in their 16-byte
alignment does not stage at all. Every case must leave the split mode bit-identical to the oracle:
here the CSR arrays are views that start 4, 8 or 12 bytes past a 16-byte boundary, under layouts
that put vertices of every size into lane groups and split chunks, with staging on and off."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.gpu

LAYOUTS = {"small": (8, 64, 32), "mid": (32, 1024, 256), "wide": (16, 20000, 1024),
           "default": orc.DEFAULT_LAYOUT}


def _view(arr, dtype, shift):
    """A device copy of arr whose data pointer is `shift` elements past a 256-byte boundary."""
    import torch
    buf = torch.zeros(len(arr) + 8, dtype=dtype, device="cuda")
    if len(arr):
        buf[shift:shift + len(arr)] = torch.from_numpy(np.ascontiguousarray(arr)).to(dtype).cuda()
    return buf, buf[shift:shift + len(arr)]


@pytest.mark.parametrize("shift_t,shift_w", [(0, 0), (1, 1), (2, 2), (3, 3), (1, 0), (0, 3)])
@pytest.mark.parametrize("layout", sorted(LAYOUTS))
def test_split_mode_with_offset_arrays(shift_t, shift_w, layout):
    import torch
    g = rl.gen_rmat(14, 24, seed=31, w_lo=1.0, w_hi=10.0)
    off = torch.from_numpy(np.ascontiguousarray(g.offsets)).cuda()
    tb, tgt = _view(g.targets.view(np.int32), torch.int32, shift_t)
    wb, wt = _view(g.weights, torch.float32, shift_w)
    csr = rl.device_csr(off, tgt, wt)
    lm, hm, hc = LAYOUTS[layout]
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    with rl.Context(0) as ctx:
        for rule in (1, 2):
            res = ctx.lowmem_device(csr, out, mode=rl.MODE_SYNC_SPLIT, slots=8, sketch_rule=rule, lane_max=lm,
                                    hub_min=hm, hub_chunk=hc, edge_staging=1)
            ref, it, edges = orc.sync_run(orc.Graph.of(g), orc.make_opts(slots=8, split=1, layout=(lm, hm, hc),
                                                                         gpu_rule=1 if rule == 2 else 0))
            assert res.iterations == it and res.traversed_edges == edges
            np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), ref)


@pytest.mark.parametrize("shift", [0, 1, 3])
def test_unit_weights_and_boyer_moore(shift):
    import torch
    g = rl.gen_rmat(13, 32, seed=32)
    off = torch.from_numpy(np.ascontiguousarray(g.offsets)).cuda()
    tb, tgt = _view(g.targets.view(np.int32), torch.int32, shift)
    csr = rl.device_csr(off, tgt, None)
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    with rl.Context(0) as ctx:
        for slots, staging in ((1, 1), (4, 1), (8, 1), (8, 2)):
            res = ctx.lowmem_device(csr, out, mode=rl.MODE_SYNC_SPLIT, slots=slots, lane_max=16, hub_min=512,
                                    hub_chunk=64, edge_staging=staging)
            ref, it, _ = orc.sync_run(orc.Graph.of(g), orc.make_opts(slots=slots, split=1, layout=(16, 512, 64)))
            assert res.iterations == it
            np.testing.assert_array_equal(out.cpu().numpy().view(np.uint32), ref)


def test_async_with_staging_valid():
    g = rl.gen_rmat(15, 32, seed=33, w_lo=1.0, w_hi=10.0)
    with rl.Context(0) as ctx:
        for staging in (1, 2):
            lab, res = ctx.lowmem(g, edge_staging=staging, lane_max=32, hub_min=2048, hub_chunk=512,
                                  compute_modularity=1)
            assert lab.max() < g.n and res.iterations >= 1 and res.modularity > 0.0
        with pytest.raises(rl.RakError) as e:
            ctx.lowmem(g, edge_staging=3)
        assert e.value.status == 1
