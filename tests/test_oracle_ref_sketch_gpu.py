"""The oracle's restatement of the reference GPU sketch rules (a new key takes the first free slot,
a full sketch decrements without clamping, the argmax is a tournament; Boyer-Moore starts from the
vertex's own label) against the reference's own device functions (inc/sketchCuda.hxx:
sketchAccumulateWarpCudU, sketchMaxGroupReduceCudU; inc/rakLowmemCuda.hxx:
rakLowmemBmScanCommunitiesCud),
compiled from its sources into oracle/_ref and run on the GPU on the same streams: every slot and
the chosen (key, weight) must be identical. Weights are multiples of 0.5, so sums and differences
are exact, and include zero weights, exact decrements to zero and ties."""
import numpy as np
import pytest

import oracle as orc

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not orc.have_ref_sketch_cuda(), reason="oracle/_ref/ref_sketch_cuda not built")]


def streams(slots, count, seed):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        length = int(rng.integers(0, 6 * slots + 1))
        alphabet = int(rng.integers(2, 3 * slots + 1))
        c = rng.integers(0, alphabet, length)
        w = rng.choice([0.0, 0.5, 1.0, 1.5, 2.0, 3.0], length)
        out.append(list(zip(c.tolist(), w.tolist())))
    return out


@pytest.mark.parametrize("slots", [2, 4, 8, 16])
def test_gpu_rule_sketch_matches_reference_device_code(slots):
    sts = streams(slots, 2000, 100 + slots)
    got = orc.ref_sketch_streams_gpu(slots, sts)
    for i, (st, (ref_slots, ref_best)) in enumerate(zip(sts, got)):
        s = orc.Sketch(slots, gpu_rule=True)
        for c, w in st:
            s.add(c, w)
        assert s.slots_list() == ref_slots, (i, st)
        assert s.choose() == ref_best, (i, st)


def test_gpu_rule_boyer_moore_matches_reference_device_code():
    sts = streams(1, 3000, 7)
    rng = np.random.default_rng(8)
    own = rng.integers(0, 4, len(sts)).tolist()
    got = orc.ref_sketch_streams_gpu(1, sts, own=own)
    for i, (st, d, (ref_slots, ref_best)) in enumerate(zip(sts, own, got)):
        s = orc.Sketch(1, gpu_rule=True)
        s.s.k[0], s.s.w[0] = d, 0.0                   # the GPU rules start from the own label
        for c, w in st:
            s.add(c, w)
        assert s.slots_list()[0] == ref_best == ref_slots[0], (i, d, st)
