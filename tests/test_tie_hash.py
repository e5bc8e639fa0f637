"""Hashed ties (rak_options.tie_break 2): the oracle's tie order is the SplitMix64 finaliser of
(key << 32 | u) ^ l * 0xD6E8FEB86659FD93, and its argmax takes the largest weight, then among equal
maximum weights the key with the largest hash. Checked here against a plain-Python statement of the
same formula on random streams; the GPU kernels are checked against the oracle in
tests/test_tie_break_gpu.py."""
import numpy as np

import oracle as orc

M64 = (1 << 64) - 1


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & M64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & M64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & M64
    return x ^ (x >> 31)


def tie_hash(u, key, l):
    return splitmix64(((key << 32) | u) ^ ((l * 0xD6E8FEB86659FD93) & M64))


def test_hash_formula():
    rng = np.random.default_rng(5)
    for _ in range(2000):
        u, key, l = (int(x) for x in rng.integers(0, 2 ** 32, 3))
        assert orc._o.orc_tie_hash(u, key, l) == tie_hash(u, key, l)


def test_hashed_argmax():
    rng = np.random.default_rng(6)
    for _ in range(3000):
        slots = int(rng.choice([2, 4, 8, 16]))
        s = orc.orc_sketch()
        keys = rng.choice(1 << 20, slots, replace=False)
        wts = rng.integers(0, 4, slots).astype(np.float32)      # many equal weights, some zero
        for i in range(slots):
            s.k[i], s.w[i] = int(keys[i]), float(wts[i])
        u, l = int(rng.integers(0, 1 << 20)), int(rng.integers(0, 20))
        c, w = orc.C.c_uint32(0), orc.C.c_float(0)
        orc._o.orc_sketch_choose_hashed(orc.C.byref(s), slots, u, l, orc.C.byref(c), orc.C.byref(w))
        wm = float(wts.max())
        if wm <= 0:
            assert c.value == orc.NONE and w.value == 0.0
            continue
        tied = [i for i in range(slots) if wts[i] == wm]
        best = max(tied, key=lambda i: (tie_hash(u, int(keys[i]), l), -i))
        assert (c.value, w.value) == (int(keys[best]), wm)
