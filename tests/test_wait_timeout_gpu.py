"""Failure detection without a GPU fault. Every device-side wait of the persistent kernel -- the
grid barrier between iterations -- is bounded by rak_options.wait_timeout_ns. When the bound runs
out, the waiting block records RAK_ERR_TIMEOUT, raises the launch's abort flag, and every block
leaves the kernel; the call returns RAK_ERR_TIMEOUT and the context stays usable. (The reference has
no bound: its blocking read-back waits for ever, inc/rakLowmemCuda.hxx:486, and CUDA errors exit the
process, inc/_cuda.hxx:221-235.)

A 1 ns bound makes the first barrier that any block reaches before the last block run out: blocks
finish their share of an iteration's work items at different times. Nothing here hangs or faults the
GPU: the waits end by themselves, and the run that follows checks the context still computes."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.gpu


def _times_out(call):
    for _ in range(3):          # a wait that never had to wait cannot run out: try again
        try:
            call()
        except rl.RakError as e:
            return e
    return None


@pytest.mark.parametrize("mode", [rl.MODE_SYNC, rl.MODE_ASYNC])
def test_wait_runs_out_and_context_stays_usable(mode):
    g = rl.gen_rmat(16, 16, seed=42)
    og = orc.Graph.of(g)
    with rl.Context(0) as ctx:
        err = _times_out(lambda: ctx.lowmem(g, mode=mode, wait_timeout_ns=1))
        assert err is not None, "no wait ran out"
        assert err.status == 5, err            # RAK_ERR_TIMEOUT
        assert "wait" in str(err)
        # the same context, default bound: a complete, correct run
        lab, res = ctx.lowmem(g, mode=rl.MODE_SYNC)
        ref, it, _ = orc.sync_run(og, orc.make_opts(slots=8, rescan=1))
        assert res.iterations == it and np.array_equal(lab, ref)


def test_resident_graph_wait_runs_out_then_runs():
    import torch
    g = rl.gen_rmat(15, 16, seed=43, w_lo=1.0, w_hi=10.0)
    og = orc.Graph.of(g)
    with rl.Context(0) as ctx:
        rg = rl.ResidentGraph(ctx, g)
        out = torch.empty(g.n, dtype=torch.int32, device="cuda")
        opts = dict(mode=rl.MODE_SYNC_SPLIT, lane_max=8, hub_min=64, hub_chunk=32)
        err = _times_out(lambda: rg.run(out, wait_timeout_ns=1, **opts))
        assert err is not None and err.status == 5
        res = rg.run(out, **opts)
        ref, it, _ = orc.sync_run(og, orc.make_opts(slots=8, split=1, layout=(8, 64, 32)))
        assert res.iterations == it
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)
        rg.close()


def test_negative_bound_is_rejected():
    g = rl.gen_rmat(8, 8, seed=1)
    with rl.Context(0) as ctx:
        with pytest.raises(rl.RakError) as e:
            ctx.lowmem(g, wait_timeout_ns=-1)
        assert e.value.status == 1
