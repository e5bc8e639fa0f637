"""Dense iterations (rak_options.dense_pct) of asynchronous single-graph runs: after an iteration whose
moved vertices hold at least dense_pct% of the edges, the next iteration's moves mark no neighbours
and the iteration after it processes every vertex. The default keeps the reference's pruning, in
which every move marks the mover's neighbours (inc/rakCuda.hxx:96-103, called from the move kernels
at inc/rakLowmemCuda.hxx:155,225,313,413).

Checked here: the default marks after every move; with the option the runs stay valid labellings,
the counters account for the iterations that marked nothing (and the one after each, which
processes every vertex), and the synchronous modes ignore it."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    with rl.Context(0) as c:
        yield c


@pytest.fixture(scope="module")
def g16():
    # the reference's CPU-runnable case: R-MAT scale 16, edge factor 16, unit weights
    return rl.gen_rmat(16, 16, seed=42)


def test_default_marks_after_every_move(ctx, g16):
    lab, res = ctx.lowmem(g16, slots=8)
    assert res.dense_iterations == 0
    assert res.marked_edges == res.moved_edges > 0


@pytest.mark.parametrize("slots", [8, 1])
def test_dense_iterations_are_counted_and_valid(ctx, g16, slots):
    n = g16.n
    lab, res = ctx.lowmem(g16, slots=slots, dense_pct=1, tolerance=0.0, max_iterations=6, compute_modularity=1)
    assert lab.max() < n
    # iteration 0 always marks (no iteration before it); on this graph the moves of the later ones
    # hold more than 1% of the edges, so they mark nothing
    assert 3 <= res.iterations <= 6
    assert 1 <= res.dense_iterations < res.iterations
    assert res.marked_edges < res.moved_edges
    # every dense iteration but the last is followed by one that processes every vertex with edges
    # (iteration 0 processes them all too: every flag starts set)
    nz = int(np.count_nonzero(g16.degrees()))
    assert res.processed_vertices >= nz * res.dense_iterations
    q = orc.modularity(orc.Graph.of(g16), lab)
    assert res.modularity == pytest.approx(q, rel=1e-9, abs=1e-12)
    assert q > 0.0


def test_dense_quality_on_a_full_run(ctx, g16):
    _, ref = ctx.lowmem(g16, slots=8, compute_modularity=1)
    lab, res = ctx.lowmem(g16, slots=8, dense_pct=20, compute_modularity=1)
    assert lab.max() < g16.n and res.iterations >= 1
    # a frontier of every vertex instead of the pruned one: the same kind of partition
    assert res.modularity >= 0.8 * ref.modularity, (res.modularity, ref.modularity)


@pytest.mark.parametrize("mode", [rl.MODE_SYNC, rl.MODE_SYNC_SPLIT])
def test_synchronous_modes_ignore_it(ctx, g16, mode):
    lab0, res0 = ctx.lowmem(g16, mode=mode, slots=8)
    lab1, res1 = ctx.lowmem(g16, mode=mode, slots=8, dense_pct=1)
    assert res1.dense_iterations == 0 and res1.marked_edges == res1.moved_edges
    assert res0.iterations == res1.iterations and np.array_equal(lab0, lab1)


def test_dense_pct_out_of_range(ctx, g16):
    with pytest.raises(rl.RakError) as e:
        ctx.lowmem(g16, dense_pct=101)
    assert e.value.status == 1
