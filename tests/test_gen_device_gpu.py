"""Device R-MAT generator (rak_gen_rmat_device): bit-identical to the host generator -- same offsets,
targets and weights -- for weighted and unit graphs, 32- and 64-bit offsets, and skewed or uniform
quadrant probabilities."""
import numpy as np
import pytest

import rak_lowmem as rl

pytestmark = pytest.mark.gpu

CASES = [
    dict(scale=8, edge_factor=4, seed=1, offset_bits=64),
    dict(scale=12, edge_factor=16, seed=2, w_lo=1.0, w_hi=10.0, offset_bits=32),
    dict(scale=14, edge_factor=8, a=0.25, b=0.25, c=0.25, seed=3, offset_bits=64),
    dict(scale=16, edge_factor=32, seed=42, w_lo=0.5, w_hi=2.0, offset_bits=64),
]


@pytest.mark.parametrize("kw", CASES, ids=[f"s{c['scale']}_ef{c['edge_factor']}_{c['offset_bits']}" for c in CASES])
def test_device_rmat_equals_host(kw):
    kw = dict(kw)
    bits = kw.pop("offset_bits")
    want = rl.gen_rmat(**kw)
    with rl.Context(0) as ctx:
        dg = rl.gen_rmat_device(ctx, offset_bits=bits, **kw)
        assert dg.n == want.n and dg.m == want.m
        assert int(dg.csr.offset_bits) == bits
        got = dg.to_host()
        np.testing.assert_array_equal(got.offsets, want.offsets)
        np.testing.assert_array_equal(got.targets, want.targets)
        if want.weights is None:
            assert got.weights is None and not dg.weighted
        else:
            np.testing.assert_array_equal(got.weights.view(np.uint32), want.weights.view(np.uint32))
        # runs on the device graph directly
        import torch
        out = torch.empty(dg.n, dtype=torch.int32, device="cuda")
        res = ctx.lowmem_device(dg.csr, out, mode=rl.MODE_SYNC)
        assert res.iterations >= 1
        dg.close()
