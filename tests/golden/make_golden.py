"""Generates tests/golden/golden.npz: golden vectors produced by the reference's own CPU code.

The reference has no tests or fixtures of its own, so these vectors are made by running its
functions, compiled from its sources into oracle/_ref/libref_cpu.so by oracle/Makefile:
  - rakLowmemStaticOmp<MULTI,RESCAN,SLOTS> with one thread (labels, iterations)
        inc/rakLowmem.hxx:277-284
  - one synchronous iteration built from its per-vertex functions on a seeded snapshot
        inc/rakLowmem.hxx:100-172
  - modularityBy                                                       inc/properties.hxx:177-192
  - Misra-Gries / Boyer-Moore accumulation of hand-made (community, weight) streams
        inc/rakLowmem.hxx:63-89, 115-128
Inputs are stored with the outputs, so the fixtures do not depend on any generator.
Run where the reference sources are available:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "rak-lowmem-communities-cuda_b200"))
import oracle as orc  # noqa: E402
import rak_lowmem as rl  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")

RUNS = [(8, 1), (8, 0), (4, 1), (16, 0), (2, 1), (1, 0)]   # (slots, rescan); slots 1 = Boyer-Moore
STEPS = [(8, 1), (8, 0), (4, 1), (1, 0)]


def csr_from_edges(n, edges, weights=None):
    """Symmetric CSR (both directions) from undirected (u, v[, w]) pairs; keeps self-loops once."""
    adj = [[] for _ in range(n)]
    for i, (u, v) in enumerate(edges):
        w = 1.0 if weights is None else weights[i]
        adj[u].append((v, w))
        if u != v:
            adj[v].append((u, w))
    off = np.zeros(n + 1, np.int64)
    tgt, wt = [], []
    for u in range(n):
        for v, w in sorted(adj[u]):
            tgt.append(v)
            wt.append(w)
        off[u + 1] = len(tgt)
    return off, np.array(tgt, np.uint32), (None if weights is None else np.array(wt, np.float32))


def hand_graphs():
    g = {}
    g["path10"] = csr_from_edges(10, [(i, i + 1) for i in range(9)])
    cl = [(a, b) for blk in (range(0, 5), range(5, 10)) for a in blk for b in blk if a < b]
    g["bridge"] = csr_from_edges(10, cl + [(4, 5)])
    g["star"] = csr_from_edges(10, [(0, i) for i in range(1, 10)])
    g["selfloops"] = csr_from_edges(8, [(0, 1), (1, 2), (0, 2), (3, 4), (4, 5), (3, 5), (2, 3), (1, 1), (4, 4)])
    g["noedges"] = (np.zeros(6, np.int64), np.zeros(0, np.uint32), None)
    g["cycle4_w"] = csr_from_edges(4, [(0, 1), (1, 2), (2, 3), (3, 0)], [1.5, 2.5, 1.5, 2.5])
    return g


def generated_graphs():
    g = {}
    a = rl.gen_rmat(9, 8, seed=11)
    g["rmat9"] = (a.offsets.copy(), a.targets.copy(), None)
    b = rl.gen_rmat(8, 8, seed=5, w_lo=1.0, w_hi=10.0)
    g["rmat8_w"] = (b.offsets.copy(), b.targets.copy(), b.weights.copy())
    c = rl.gen_sbm(600, 6, 12.0, 20.0, seed=3)
    g["sbm600"] = (c.offsets.copy(), c.targets.copy(), None)
    d = rl.gen_lattice(16, 12, 0.1, 0.05, seed=9)
    g["lattice16x12"] = (d.offsets.copy(), d.targets.copy(), None)
    return g


def main():
    if not orc.have_ref_cpu():
        sys.exit("oracle/_ref/libref_cpu.so missing: run `make -C oracle` where the reference sources exist")
    out = {}
    graphs = {**hand_graphs(), **generated_graphs()}
    out["graphs"] = np.array(sorted(graphs))
    rng = np.random.default_rng(2024)
    for name, (off, tgt, wt) in sorted(graphs.items()):
        g = orc.Graph(off, tgt, wt)
        out[f"{name}/offsets"] = off
        out[f"{name}/targets"] = tgt
        if wt is not None:
            out[f"{name}/weights"] = wt
        for slots, rescan in RUNS:
            lab, it, _ = orc.ref_lowmem_omp(g, slots, rescan, threads=1)
            out[f"{name}/run_{slots}_{rescan}/labels"] = lab
            out[f"{name}/run_{slots}_{rescan}/iterations"] = np.array(it)
            out[f"{name}/run_{slots}_{rescan}/modularity"] = np.array(orc.ref_modularity(g, lab))
        n = g.n
        vp = rng.integers(0, max(n // 3, 1), n).astype(np.uint32) if n else np.zeros(0, np.uint32)
        ap = (rng.random(n) < 0.6).astype(np.uint8)
        out[f"{name}/snap/labels"] = vp
        out[f"{name}/snap/flags"] = ap
        for slots, rescan in STEPS:
            for pickless in (0, 1):
                vn, an, ch = orc.ref_sync_step(g, slots, rescan, pickless, vp, ap)
                key = f"{name}/step_{slots}_{rescan}_{pickless}"
                out[key + "/labels"] = vn
                out[key + "/flags"] = an
                out[key + "/changed"] = np.array(ch)
    for slots in (1, 2, 4, 8, 16):
        for i in range(12):
            L = int(rng.integers(1, 48))
            c = rng.integers(0, 10, L).astype(np.uint32)
            w = rng.choice(np.array([1.0, 2.0, 0.5, 3.25, 0.75], np.float32), L)
            k, ww = orc.ref_sketch_stream(slots, c, w)
            key = f"stream/{slots}/{i}"
            out[key + "/comm"] = c
            out[key + "/wts"] = w
            out[key + "/keys"] = k
            out[key + "/weights"] = ww
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
