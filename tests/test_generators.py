"""Synthetic graph generators (host): deterministic, symmetric, simple (no self-loops or
duplicates), sorted adjacency, and independent of the thread count."""
import numpy as np

import rak_lowmem as rl


def check_simple_symmetric(g, weighted):
    deg = g.degrees()
    src = np.repeat(np.arange(g.n, dtype=np.int64), deg)
    dst = g.targets.astype(np.int64)
    assert not np.any(src == dst)
    key = src * g.n + dst
    assert np.all(np.diff(key) > 0)                     # sorted, duplicate-free per row
    rev = np.sort(dst * g.n + src)
    np.testing.assert_array_equal(np.sort(key), rev)     # symmetric
    if weighted:
        order = np.argsort(dst * g.n + src)
        np.testing.assert_array_equal(g.weights, g.weights[order][np.argsort(np.argsort(key))])


def test_rmat_properties_and_determinism():
    a = rl.gen_rmat(11, 8, seed=3, threads=1)
    b = rl.gen_rmat(11, 8, seed=3, threads=4)
    np.testing.assert_array_equal(a.offsets, b.offsets)
    np.testing.assert_array_equal(a.targets, b.targets)
    assert a.weights is None
    check_simple_symmetric(a, False)
    c = rl.gen_rmat(11, 8, seed=4)
    assert not np.array_equal(a.targets[:1000], c.targets[:1000])
    # skew of the (0.57, 0.19, 0.19, 0.05) quadrants: low ids carry most edges
    deg = a.degrees()
    assert deg[: a.n // 8].sum() > deg[-a.n // 8:].sum() * 4


def test_rmat_weights_symmetric_and_in_range():
    g = rl.gen_rmat(10, 8, seed=5, w_lo=1.0, w_hi=10.0)
    assert g.weights.dtype == np.float32 and g.weights.min() >= 1.0 and g.weights.max() < 10.0
    check_simple_symmetric(g, True)


def test_sbm_truth_and_structure():
    g = rl.gen_sbm(2000, 20, 16.0, 20.0, seed=1)
    check_simple_symmetric(g, False)
    assert g.truth is not None and g.truth.max() == 19
    src = np.repeat(np.arange(g.n), g.degrees())
    inside = np.mean(g.truth[src] == g.truth[g.targets])
    # p_in/p_out = 20 with 20 blocks of 100: expected internal share 20*99 / (20*99 + 1900)
    assert abs(inside - 1980 / 3880) < 0.03
    assert abs(g.m / g.n - 16.0) < 1.0


def test_lattice_degrees():
    g = rl.gen_lattice(40, 30, 0.05, 0.0, seed=2)
    check_simple_symmetric(g, False)
    assert g.degrees().max() <= 4
    full = 2 * (39 * 30 + 40 * 29)
    assert 0.9 * full < g.m < full
    h = rl.gen_lattice(40, 30, 0.05, 0.01, seed=2)
    assert h.m >= g.m
