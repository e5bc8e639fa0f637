"""The C restatement against the live reference build (oracle/_ref, compiled from the reference's
sources) on seeded random graphs. Skipped where the reference build is absent."""
import numpy as np
import pytest

import oracle as orc
import rak_lowmem as rl

pytestmark = pytest.mark.skipif(not orc.have_ref_cpu(), reason="oracle/_ref not built (reference sources absent)")


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("weighted", [False, True])
def test_serial_and_steps_vs_reference(seed, weighted):
    g = rl.gen_rmat(10, 6, seed=seed, w_lo=1.0, w_hi=(9.0 if weighted else 1.0))
    og = orc.Graph.of(g)
    for slots, rescan in [(8, 1), (8, 0), (4, 0), (16, 1), (1, 0)]:
        a, ia = orc.serial_run(og, slots, rescan)
        b, ib, _ = orc.ref_lowmem_omp(og, slots, rescan, threads=1)
        assert ia == ib
        np.testing.assert_array_equal(a, b)
    rng = np.random.default_rng(seed)
    for slots, rescan in [(8, 1), (8, 0), (2, 1), (1, 0)]:
        vp = rng.integers(0, og.n // 5, og.n).astype(np.uint32)
        ap = (rng.random(og.n) < 0.8).astype(np.uint8)
        vn, an, ch, _, _ = orc.sync_step(og, orc.make_opts(slots=slots, rescan=rescan), 3, vp, ap)
        rn, ra, rch = orc.ref_sync_step(og, slots, rescan, 0, vp, ap)
        np.testing.assert_array_equal(vn, rn)
        np.testing.assert_array_equal(an, ra)
        assert ch == rch


def test_modularity_vs_reference():
    g = rl.gen_sbm(3000, 30, 10.0, 20.0, seed=4)
    og = orc.Graph.of(g)
    lab, _ = orc.serial_run(og, 8, 1)
    assert orc.modularity(og, lab) == pytest.approx(orc.ref_modularity(og, lab), rel=1e-12)
    assert orc.modularity(og, g.truth) == pytest.approx(orc.ref_modularity(og, g.truth), rel=1e-12)
    assert orc.modularity(og, g.truth) > 0.3   # internal share ~0.41 minus 1/30
