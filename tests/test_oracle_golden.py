"""The C restatement (oracle/rak_oracle.c) against golden vectors made by the reference's own CPU
code (tests/golden/make_golden.py): serial runs, synchronous steps, modularity, sketch streams."""
import numpy as np
import pytest

import oracle as orc
from conftest import golden_graph

RUNS = [(8, 1), (8, 0), (4, 1), (16, 0), (2, 1), (1, 0)]
STEPS = [(8, 1), (8, 0), (4, 1), (1, 0)]


def names(z):
    return [str(x) for x in z["graphs"]]


def test_golden_has_graphs(golden):
    assert len(names(golden)) >= 10


@pytest.mark.parametrize("slots,rescan", RUNS)
def test_serial_runs_match_reference(golden, slots, rescan):
    for name in names(golden):
        g = golden_graph(golden, name)
        lab, it = orc.serial_run(g, slots, rescan)
        key = f"{name}/run_{slots}_{rescan}"
        assert it == int(golden[key + "/iterations"]), name
        np.testing.assert_array_equal(lab, golden[key + "/labels"], err_msg=name)
        q = golden[key + "/modularity"]
        assert orc.modularity(g, lab) == pytest.approx(float(q), rel=1e-12, abs=1e-15), name


@pytest.mark.parametrize("slots,rescan", STEPS)
@pytest.mark.parametrize("pickless", [0, 1])
def test_sync_steps_match_reference(golden, slots, rescan, pickless):
    for name in names(golden):
        g = golden_graph(golden, name)
        o = orc.make_opts(slots=slots, rescan=rescan, pickless_step=1 if pickless else 0)
        vn, an, ch, _, _ = orc.sync_step(g, o, 0, golden[f"{name}/snap/labels"], golden[f"{name}/snap/flags"])
        key = f"{name}/step_{slots}_{rescan}_{pickless}"
        np.testing.assert_array_equal(vn, golden[key + "/labels"], err_msg=name)
        np.testing.assert_array_equal(an, golden[key + "/flags"], err_msg=name)
        assert ch == int(golden[key + "/changed"]), name


@pytest.mark.parametrize("slots", [1, 2, 4, 8, 16])
def test_sketch_streams_match_reference(golden, slots):
    i = 0
    while f"stream/{slots}/{i}/comm" in golden:
        key = f"stream/{slots}/{i}"
        s = orc.Sketch(slots)
        for c, w in zip(golden[key + "/comm"], golden[key + "/wts"]):
            s.add(int(c), float(w))
        got = s.slots_list()
        assert [k for k, _ in got] == [int(x) for x in golden[key + "/keys"]], key
        np.testing.assert_array_equal(np.array([w for _, w in got], np.float32), golden[key + "/weights"])
        i += 1
    assert i > 0


def test_known_answer_streams():
    # Misra-Gries, 2 slots, CPU rule: last free slot, clamp at zero, stale keys reused by matching.
    s = orc.Sketch(2).add(5, 1.0)
    assert s.slots_list() == [(orc.NONE, 0.0), (5, 1.0)]           # last free slot first
    s.add(6, 2.0)
    assert s.slots_list() == [(6, 2.0), (5, 1.0)]
    s.add(7, 1.5)                                                     # full: all drop by 1.5, clamped
    assert s.slots_list() == [(6, 0.5), (5, 0.0)]
    s.add(5, 1.0)                                                     # stale key 5 matches its slot
    assert s.slots_list() == [(6, 0.5), (5, 1.0)]
    assert s.choose() == (5, 1.0)
    t = orc.Sketch(2).add(1, 2.0).add(2, 2.0)                         # tie: first maximum wins
    assert t.choose() == (2, 2.0)
    # Boyer-Moore: replaced when the candidate's weight is not above the new edge's.
    b = orc.Sketch(1).add(3, 1.0).add(4, 1.0)
    assert b.choose() == (4, 1.0)
    b.add(4, 2.0).add(9, 1.0)
    assert b.choose() == (4, 2.0)


def test_gpu_rule_known_answers():
    """The reference GPU sketch rules (inc/sketchCuda.hxx): a new key takes the FIRST free slot,
    a full sketch decrements without clamping (negative slots are not free), and the argmax is a
    tournament whose winner may weigh <= 0."""
    s = orc.Sketch(4, gpu_rule=True).add(7, 1.0).add(8, 1.0)
    assert s.slots_list()[:2] == [(7, 1.0), (8, 1.0)]              # slots 0, 1 (CPU rule: 3, 2)
    c = orc.Sketch(4).add(7, 1.0).add(8, 1.0)
    assert c.slots_list()[2:] == [(8, 1.0), (7, 1.0)]
    s = orc.Sketch(2, gpu_rule=True).add(1, 1.0).add(2, 3.0).add(3, 2.0)   # full: both drop by 2
    assert s.slots_list() == [(1, -1.0), (2, 1.0)]
    s.add(4, 5.0)                                                   # still no free slot: drop again
    assert s.slots_list() == [(1, -6.0), (2, -4.0)]
    assert s.choose() == (2, -4.0)                                  # winner may be negative
    t = orc.Sketch(4, gpu_rule=True).add(1, 1.0).add(2, 2.0).add(3, 2.0).add(4, 1.0)
    assert t.choose() == (3, 2.0)                                   # tournament: slot 2 beats slot 0,
    u = orc.Sketch(4).add(1, 1.0).add(2, 2.0).add(3, 2.0).add(4, 1.0)   # slot 1 never beats it
    assert u.choose()[1] == 2.0
    z = orc.Sketch(2, gpu_rule=True).add(5, 2.0).add(6, 2.0).add(7, 2.0)   # exact zero frees a slot
    assert z.slots_list() == [(5, 0.0), (6, 0.0)]
    z.add(8, 1.0)
    assert z.slots_list() == [(8, 1.0), (6, 0.0)]
