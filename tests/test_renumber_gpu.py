"""Renumbered runs (rak_options.renumber): the graph copied on the device in the library's work order
(heaviest vertices first), labels kept at their original values, results gathered back into the
graph's own numbering. The reference runs on a copy in its degree-partition order too
(inc/rakLowmemCuda.hxx:505-519, 563-568).

The synchronous split mode takes the option on request, and its results must not depend on it: the
split layout depends on degrees only, every row keeps its edge order, and labels keep their values,
so a renumbered run equals the run on the graph as given bit for bit -- offsets, targets, weights,
initial labels and flags, and the final gather all checked at once, in every work regime. The
asynchronous mode renumbers large dense resident graphs by default; here a renumbered run is
compared with the run on the graph as given."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.gpu

FORCED_SPLIT = dict(lane_max=32, hub_min=1024, hub_chunk=256)   # every regime, split chunks included

GRAPHS = {
    "rmat14_w": lambda: rl.gen_rmat(14, 16, seed=5, w_lo=1.0, w_hi=10.0),
    "rmat15_unit_off32": lambda: rl.gen_rmat(15, 16, seed=6).with_offsets32(),
    "sbm": lambda: rl.gen_sbm(20000, 40, 16.0, 20.0, seed=7),
    "lattice": lambda: rl.gen_lattice(160, 120, 0.05, 0.01, seed=8),
}


@pytest.fixture(scope="module")
def ctx():
    with rl.Context(0) as c:
        yield c


@pytest.mark.parametrize("layout", ["default", "forced"])
@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_split_mode_renumbered_equals_as_given(ctx, name, layout):
    g = GRAPHS[name]()
    ly = FORCED_SPLIT if layout == "forced" else {}
    lab0, r0 = ctx.lowmem(g, mode=rl.MODE_SYNC_SPLIT, renumber=2, **ly)
    lab1, r1 = ctx.lowmem(g, mode=rl.MODE_SYNC_SPLIT, renumber=1, **ly)
    assert r1.iterations == r0.iterations
    assert np.array_equal(lab1, lab0)
    assert r1.traversed_edges == r0.traversed_edges and r1.moved_vertices == r0.moved_vertices


def test_split_mode_renumbered_matches_oracle(ctx):
    g = rl.gen_rmat(13, 12, seed=9, w_lo=1.0, w_hi=10.0)
    lab, res = ctx.lowmem(g, mode=rl.MODE_SYNC_SPLIT, renumber=1, **FORCED_SPLIT)
    ref, it, _ = orc.sync_run(orc.Graph.of(g), orc.make_opts(slots=8, split=1, layout=(32, 1024, 256)))
    assert res.iterations == it
    assert np.array_equal(lab, ref)


def test_renumbered_initial_labels_and_flags(ctx):
    g = rl.gen_rmat(14, 16, seed=10, w_lo=1.0, w_hi=10.0)
    rng = np.random.default_rng(3)
    q = rng.integers(0, g.n, g.n).astype(np.uint32)
    flags = (rng.random(g.n) < 0.6).astype(np.uint8)
    kw = dict(mode=rl.MODE_SYNC_SPLIT, max_iterations=3, **FORCED_SPLIT)
    lab0, r0 = ctx.lowmem(g, q=q, flags=flags, renumber=2, **kw)
    lab1, r1 = ctx.lowmem(g, q=q, flags=flags, renumber=1, **kw)
    assert r1.iterations == r0.iterations and r1.processed_vertices == r0.processed_vertices
    assert np.array_equal(lab1, lab0)


def test_resident_graph_keeps_one_copy_across_layouts(ctx):
    import torch
    g = rl.gen_rmat(14, 16, seed=11, w_lo=1.0, w_hi=10.0)
    rg = rl.ResidentGraph(ctx, g)
    out0 = torch.empty(g.n, dtype=torch.int32, device="cuda")
    out1 = torch.empty(g.n, dtype=torch.int32, device="cuda")
    for ly in ({}, FORCED_SPLIT, {}):     # the copy follows the plan when the layout changes
        rg.run(out0, mode=rl.MODE_SYNC_SPLIT, renumber=2, **ly)
        rg.run(out1, mode=rl.MODE_SYNC_SPLIT, renumber=1, **ly)
        assert torch.equal(out0, out1)
    rg.close()


@pytest.mark.parametrize("slots", [8, 1])   # 1: labels are positions in the reference order by default
def test_async_renumbered_quality(ctx, slots):
    g = rl.gen_rmat(18, 16, seed=42)
    og = orc.Graph.of(g)
    lab1, r1 = ctx.lowmem(g, slots=slots, renumber=1, compute_modularity=1)
    lab0, r0 = ctx.lowmem(g, slots=slots, renumber=2, compute_modularity=1)
    assert lab1.max() < g.n and lab0.max() < g.n
    assert r1.modularity == pytest.approx(orc.modularity(og, lab1), rel=1e-9, abs=1e-12)
    # the same algorithm on the same graph: the asynchronous order differs, the quality does not
    assert r1.modularity >= r0.modularity * 0.97 - 1e-4, (r1.modularity, r0.modularity)


def test_exact_mode_is_not_renumbered(ctx):
    g = rl.gen_rmat(12, 8, seed=12)
    lab0, r0 = ctx.lowmem(g, mode=rl.MODE_SYNC, renumber=2)
    lab1, r1 = ctx.lowmem(g, mode=rl.MODE_SYNC, renumber=1)
    assert np.array_equal(lab0, lab1)
    with pytest.raises(rl.RakError) as e:
        ctx.lowmem(g, renumber=3)
    assert e.value.status == 1


def test_default_copy_only_when_it_fits(ctx):
    """The default makes the renumbered copy of a large dense resident graph only when it fits beside
    what the device already holds (with 1 GiB to spare); otherwise the run works on the graph as
    given. Device memory is filled with one tensor to leave too little room, then released."""
    import torch
    g = rl.gen_rmat(22, 16, seed=13)            # 2^22 vertices, average degree above 8: copied by default
    rg = rl.ResidentGraph(ctx, g)
    out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    copy_gb = (g.m * 4 + (g.n + 1) * 8 + g.n * 8) / 2**30   # targets, offsets, inverse map, work order
    free, _ = torch.cuda.mem_get_info(0)
    filler = torch.empty(max(0, free - (1 << 30) - (256 << 20)), dtype=torch.uint8, device="cuda")
    r0 = rg.run(out)                            # about 1.25 GiB free: below the copy plus its margin
    del filler
    torch.cuda.empty_cache()
    assert r0.memory_gb < copy_gb, (r0.memory_gb, copy_gb)
    lab0 = out.cpu().numpy().view(np.uint32)
    assert lab0.max() < g.n
    r1 = rg.run(out)                            # room again: the copy is made and used
    assert r1.memory_gb - r0.memory_gb >= 0.9 * copy_gb, (r1.memory_gb, r0.memory_gb, copy_gb)
    assert out.cpu().numpy().view(np.uint32).max() < g.n
    rg.close()
