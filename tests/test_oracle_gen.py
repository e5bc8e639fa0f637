"""The oracle's C restatement of the library's synthetic graphs (oracle/rmat_gen.c) equals the
library's own generators bit for bit: offsets, targets and weights. bench.py's reference arm builds
its workload graph with the restatement, so that arm never loads the library."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl


def same(a, b):
    assert a.n == b.n and a.m == b.m
    assert np.array_equal(a.offsets, np.asarray(b.offsets, dtype=np.int64))
    assert np.array_equal(a.targets, b.targets)
    if b.weights is None:
        assert a.weights is None
    else:
        assert a.weights is not None
        assert np.array_equal(a.weights.view(np.uint32), b.weights.view(np.uint32))


@pytest.mark.parametrize("scale,ef,w,seed", [
    (1, 4, (1.0, 1.0), 42),          # two vertices: only self-loops or one edge
    (8, 1.5, (1.0, 1.0), 7),         # fractional edge factor
    (10, 8, (1.0, 1.0), 42),
    (12, 16, (1.0, 10.0), 42),       # weights in [1, 10), symmetric per undirected pair
    (15, 32, (0.5, 2.0), 3),
    (17, 16, (1.0, 1.0), 42),        # config-1 family, 2^17 vertices
])
def test_rmat_equals_library(scale, ef, w, seed):
    a = orc.gen_rmat(scale, ef, seed=seed, w_lo=w[0], w_hi=w[1], threads=3)
    b = rl.gen_rmat(scale, ef, 0.57, 0.19, 0.19, seed, w[0], w[1])
    same(a, b)


def test_rmat_other_quadrant_probabilities():
    a = orc.gen_rmat(11, 8, 0.45, 0.15, 0.15, seed=9)
    b = rl.gen_rmat(11, 8, 0.45, 0.15, 0.15, 9)
    same(a, b)


def test_rmat_independent_of_thread_count():
    a = orc.gen_rmat(13, 16, seed=5, w_lo=1.0, w_hi=10.0, threads=1)
    b = orc.gen_rmat(13, 16, seed=5, w_lo=1.0, w_hi=10.0, threads=4)
    same(a, b)


@pytest.mark.parametrize("wh,pd,sc", [((1, 1), 0.05, 0.01), ((37, 23), 0.05, 0.01), ((200, 150), 0.2, 0.05),
                                      ((64, 1), 0.0, 0.0)])
def test_lattice_equals_library(wh, pd, sc):
    a = orc.gen_lattice(wh[0], wh[1], pd, sc, seed=42, threads=2)
    b = rl.gen_lattice(wh[0], wh[1], pd, sc, 42)
    same(a, b)


def test_bad_arguments_rejected():
    with pytest.raises(RuntimeError):
        orc.gen_rmat(0, 8)
    with pytest.raises(RuntimeError):
        orc.gen_lattice(0, 5)
