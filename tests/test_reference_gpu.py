"""Head-to-head with the reference's own GPU path, rakLowmemStaticCuda<8> / <1>
(inc/rakLowmemCuda.hxx:624-632), compiled from its sources into oracle/_ref/ref_lpa_cuda and run
as a separate process on the same graph.

Checks that the default asynchronous νMG8-LPA reaches a modularity no more than 0.5% below the
reference's (the stated target), νBM-LPA no more than 5% below (no stated target; single
asynchronous BM runs vary by a few percent, most on near-degenerate graphs such as R-MAT, where
both land in one giant community), and prints both runs (time, iterations, traversed-edge rate)
for the record.
The graphs are R-MAT scale RAK_REF_SCALE (default 18, edge factor 16, unit weights), a planted
partition SBM and a road-like lattice (4-neighbour grid, 5% of edges deleted, 1% shortcuts). On the
lattice most choices are ties between equally weighted labels; the asynchronous default breaks them
by hash in its first iterations (rak_options.tie_break 2) and ends above the reference (0.687 vs
0.628 at 2^25 vertices), where the reference's rule -- the most recently inserted key -- made it end
5.8% below. `RAK_REF_SCALE=24 RAK_REF_EF=32 RAK_REF_WEIGHTED=1 pytest tests/test_reference_gpu.py
-m gpu -s` runs the benchmark graph.
"""
import json
import os

import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not orc.have_ref_cuda(), reason="oracle/_ref/ref_lpa_cuda not built")]

SCALE = int(os.environ.get("RAK_REF_SCALE", "18"))
EF = int(os.environ.get("RAK_REF_EF", "16"))
WEIGHTED = os.environ.get("RAK_REF_WEIGHTED", "0") == "1"


def graphs():
    out = {f"rmat{SCALE}_ef{EF}" + ("_w" if WEIGHTED else ""):
           rl.gen_rmat(SCALE, EF, seed=42, w_lo=1.0, w_hi=10.0 if WEIGHTED else 1.0)}
    out["sbm100k_k200"] = rl.gen_sbm(100000, 200, 16.0, 20.0, seed=7)
    out["lattice1024"] = rl.gen_lattice(1024, 1024, 0.05, 0.01, seed=42)
    return out


@pytest.fixture(scope="module")
def ctx():
    c = rl.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("slots", [8, 1])
def test_against_reference_gpu(ctx, slots):
    for name, g in graphs().items():
        og = orc.Graph.of(g)
        ref_lab, info = orc.ref_lowmem_cuda(og, slots=slots, timeout=1800)
        q_ref = ctx.modularity(g, ref_lab)
        lab, res = ctx.lowmem(g, slots=slots, compute_modularity=1, repeat=3)
        q = res.modularity
        # the reference's time covers its iterations (with one blocking read-back each);
        # traversed edges of the reference are not counted, so compare times per run
        rec = {"graph": name, "n": g.n, "m": g.m, "slots": slots,
               "reference": {"time_ms": info["time_ms"], "iterations": info["iterations"], "modularity": q_ref,
                             "memory_gb": info["memory_gb"]},
               "ours": {"time_ms": res.time_ms, "loop_ms": res.loop_ms, "iterations": res.iterations,
                        "modularity": q, "traversed_edges": res.traversed_edges,
                        "edges_per_s": res.traversed_edges / (res.loop_ms / 1e3)},
               "speedup_time": info["time_ms"] / res.time_ms}
        print("REFGPU " + json.dumps(rec))
        assert lab.max() < g.n
        tol = 0.005 if slots > 1 else 0.05
        # plus 1e-3 absolute: on unpermuted R-MAT both implementations can end in one giant
        # community (Q ~ 1e-5), where a relative tolerance compares noise
        assert q >= q_ref - tol * abs(q_ref) - 1e-3, rec


def test_repeated_runs_never_below_reference(ctx):
    """Asynchronous runs differ from run to run (the interleaving of updates is the GPU's). Every one
    of 6 runs of the default νMG8 must end no more than 0.5% below the reference's νMG8 (its median
    over 3 runs) on the same graph, plus 1e-3 absolute for graphs where both end in one community:
    R-MAT scale 20 / edge factor 32 / weights U[1,10), and the first 24 graphs of the serving pool
    (the batched-launch mix: small R-MAT and planted-partition graphs)."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    gs = [("rmat20_ef32_w", rl.gen_rmat(20, 32, seed=42, w_lo=1.0, w_hi=10.0))]
    gs += [(f"pool{i}", g) for i, g in enumerate(bench.batch_mix(64, 11, os.cpu_count())[:24])]
    worst = []
    for name, g in gs:
        og = orc.Graph.of(g)
        q_ref = float(np.median([ctx.modularity(g, orc.ref_lowmem_cuda(og, slots=8)[0]) for _ in range(3)]))
        qs = [ctx.modularity(g, ctx.lowmem(g)[0]) for _ in range(6)]
        floor = q_ref - 0.005 * abs(q_ref) - 1e-3
        worst.append((name, min(qs), q_ref))
        assert min(qs) >= floor, (name, qs, q_ref)
    print("REPEAT " + json.dumps(worst))
