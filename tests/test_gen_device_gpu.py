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


SBM_CASES = [(2, 1, 4.0), (1000, 8, 16.0), (5000, 1000, 16.0), (100000, 200, 16.0), (262144, 37, 12.0), (7, 7, 3.0)]


@pytest.mark.parametrize("n,k,deg", SBM_CASES, ids=[f"n{c[0]}_k{c[1]}" for c in SBM_CASES])
@pytest.mark.parametrize("bits", [32, 64])
def test_device_sbm_equals_host(n, k, deg, bits):
    want = rl.gen_sbm(n, k, deg, 20.0, seed=17)
    with rl.Context(0) as ctx:
        dg = rl.gen_sbm_device(ctx, n, k, deg, 20.0, seed=17, offset_bits=bits)
        assert dg.n == want.n and dg.m == want.m and not dg.weighted
        got = dg.to_host()
        np.testing.assert_array_equal(got.offsets, want.offsets)
        np.testing.assert_array_equal(got.targets, want.targets)
        dg.close()


def test_device_batch_concat_runs_like_host_batch():
    """DeviceBatch.concat of device-built graphs equals HostBatch.concat of the host-built ones: the
    synchronous batch run gives the same labels."""
    import torch
    specs = [("rmat", 10, 8.0, 3), ("sbm", 3000, 30, 4), ("rmat", 12, 16.0, 5), ("sbm", 1500, 8, 6)]
    with rl.Context(0) as ctx:
        dev, host = [], []
        for kind, a, b, seed in specs:
            if kind == "rmat":
                dev.append(rl.gen_rmat_device(ctx, a, b, seed=seed, offset_bits=64 if seed % 2 else 32))
                host.append(rl.gen_rmat(a, b, seed=seed))
            else:
                dev.append(rl.gen_sbm_device(ctx, a, b, 16.0, 20.0, seed=seed))
                host.append(rl.gen_sbm(a, b, 16.0, 20.0, seed=seed))
        db = rl.DeviceBatch.concat([d.csr for d in dev])
        hb = rl.HostBatch.concat(host, weighted=False)
        assert db.n == hb.n and db.m == hb.m
        np.testing.assert_array_equal(db.offsets.cpu().numpy(), hb.offsets)
        np.testing.assert_array_equal(db.targets.cpu().numpy().view(np.uint32), hb.targets)
        outs = []
        for batch in (db, hb):
            b = rl.Batch(ctx, batch)
            out = torch.empty(hb.n, dtype=torch.int32, device="cuda")
            b.launch(out, mode=rl.MODE_SYNC)
            b.results()
            outs.append(out.cpu().numpy())
            b.close()
        np.testing.assert_array_equal(outs[0], outs[1])
        for d in dev:
            d.close()
