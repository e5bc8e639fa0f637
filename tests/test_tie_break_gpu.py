"""Hashed ties (rak_options.tie_break 2) on the GPU: in the synchronous modes, where runs are
deterministic, labels equal the oracle's bit for bit on every iteration count with the same tie
rule; asynchronous runs (whose default it is) give valid labels; option errors are statuses."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.gpu

SMALL = (8, 64, 32)
GRAPHS = {
    "lattice": lambda: rl.gen_lattice(60, 40, 0.05, 0.02, seed=8),          # degree <= 6: ties everywhere
    "rmat12": lambda: rl.gen_rmat(12, 8, seed=9),
    "rmat11_w": lambda: rl.gen_rmat(11, 8, seed=10, w_lo=1.0, w_hi=10.0),
    "sbm": lambda: rl.gen_sbm(4000, 40, 12.0, 20.0, seed=11),
}


@pytest.fixture(scope="module")
def ctx():
    c = rl.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", sorted(GRAPHS))
@pytest.mark.parametrize("mode", [rl.MODE_SYNC, rl.MODE_SYNC_SPLIT])
@pytest.mark.parametrize("tie_iters", [4, 20])
@pytest.mark.parametrize("layout", [None, SMALL], ids=["default", "small"])
def test_sync_hashed_ties_match_oracle(ctx, name, mode, tie_iters, layout):
    g = GRAPHS[name]()
    lay = dict(zip(("lane_max", "hub_min", "hub_chunk"), layout)) if layout else {}
    lab, res = ctx.lowmem(g, mode=mode, slots=8, tie_break=2, tie_iterations=tie_iters, **lay)
    o = orc.make_opts(slots=8, rescan=1 if mode == rl.MODE_SYNC else 0, split=1 if mode == rl.MODE_SYNC_SPLIT else 0,
                      layout=layout or orc.DEFAULT_LAYOUT, tie_until=tie_iters)
    ref, it, edges = orc.sync_run(orc.Graph.of(g), o)
    assert res.iterations == it and res.traversed_edges == edges
    np.testing.assert_array_equal(lab, ref)


def test_hashed_ties_change_lattice_result(ctx):
    """On a lattice most choices are ties: the hashed rule must actually be in effect."""
    g = GRAPHS["lattice"]()
    a, _ = ctx.lowmem(g, mode=rl.MODE_SYNC, slots=8, tie_break=1)
    b, _ = ctx.lowmem(g, mode=rl.MODE_SYNC, slots=8, tie_break=2)
    assert not np.array_equal(a, b)


def test_sync_steps_with_hashed_ties(ctx):
    import torch
    g = GRAPHS["rmat12"]()
    og = orc.Graph.of(g)
    rng = np.random.default_rng(3)
    rg = rl.ResidentGraph(ctx, g, lane_max=8, hub_min=64, hub_chunk=32)
    for it in (0, 3, 4, 9):
        vp = rng.integers(0, g.n // 5, g.n).astype(np.uint32)
        ap = (rng.random(g.n) < 0.8).astype(np.uint8)
        tv, ta = torch.from_numpy(vp.view(np.int32)).cuda(), torch.from_numpy(ap).cuda()
        vn, an = torch.empty_like(tv), torch.empty_like(ta)
        ch = rg.step(it, tv, ta, vn, an, mode=rl.MODE_SYNC_SPLIT, slots=8, tie_break=2, tie_iterations=5,
                     lane_max=8, hub_min=64, hub_chunk=32)
        rv, ra, rch, _, _ = orc.sync_step(og, orc.make_opts(slots=8, split=1, layout=SMALL, tie_until=5), it, vp, ap)
        np.testing.assert_array_equal(vn.cpu().numpy().view(np.uint32), rv)
        np.testing.assert_array_equal(an.cpu().numpy(), ra)
        assert ch == rch
    rg.close()


@pytest.mark.parametrize("slots,q_min", [(2, 0.3), (8, 0.6), (16, 0.6)])
def test_async_default_valid(ctx, slots, q_min):
    """Two slots cannot hold a degree-4 neighbourhood, so its bound is lower."""
    g = rl.gen_lattice(300, 200, 0.05, 0.01, seed=12)
    lab, res = ctx.lowmem(g, slots=slots, compute_modularity=1)
    assert lab.max() < g.n and res.iterations >= 1 and res.modularity > q_min


def test_option_errors(ctx):
    g = rl.gen_rmat(8, 8, seed=1)
    for bad in (dict(tie_break=3), dict(tie_iterations=-1)):
        with pytest.raises(rl.RakError) as e:
            ctx.lowmem(g, **bad)
        assert e.value.status == 1
    with pytest.raises(rl.RakError) as e:
        ctx.lowmem(g, sketch_rule=2, tie_break=2)
    assert e.value.status == 7
