"""The golden vectors discriminate: an oracle with a planted mistake fails them. The mistakes are
planted in the oracle on the CPU, through switches the restatement already has -- the other
reference rule set (first free slot, unclamped decrement, tournament argmax) in place of the CPU
rules the golden vectors were made with, and a stale snapshot -- so a passing golden test says
something about the rules, not only about the plumbing."""
import numpy as np

import oracle as orc
from conftest import golden_graph


def names(z):
    return [str(x) for x in z["graphs"]]


def test_wrong_rule_set_fails_the_golden_steps(golden):
    """Synchronous steps under the GPU rules differ from the reference CPU steps on some graph."""
    differs = 0
    for name in names(golden):
        g = golden_graph(golden, name)
        o = orc.make_opts(slots=8, rescan=0, pickless_step=0, gpu_rule=1)
        vn, _, _, _, _ = orc.sync_step(g, o, 0, golden[f"{name}/snap/labels"], golden[f"{name}/snap/flags"])
        differs += int(not np.array_equal(vn, golden[f"{name}/step_8_0_0/labels"]))
    assert differs > 0


def test_wrong_rule_set_fails_the_golden_streams(golden):
    """Sketch streams under the GPU rules leave other slots than the reference CPU sketch."""
    differs, i = 0, 0
    while f"stream/8/{i}/comm" in golden:
        key = f"stream/8/{i}"
        s = orc.Sketch(8, gpu_rule=True)
        for c, w in zip(golden[key + "/comm"], golden[key + "/wts"]):
            s.add(int(c), float(w))
        differs += int([k for k, _ in s.slots_list()] != [int(x) for x in golden[key + "/keys"]])
        i += 1
    assert i > 0 and differs > 0


def test_stale_snapshot_fails_the_golden_steps(golden):
    """A step from the initial labels instead of the recorded snapshot differs on some graph."""
    differs = 0
    for name in names(golden):
        g = golden_graph(golden, name)
        o = orc.make_opts(slots=8, rescan=1, pickless_step=0)
        snap = golden[f"{name}/snap/labels"]
        ids = np.arange(len(snap), dtype=np.uint32)
        if np.array_equal(ids, snap):
            continue
        vn, _, _, _, _ = orc.sync_step(g, o, 0, ids, golden[f"{name}/snap/flags"])
        differs += int(not np.array_equal(vn, golden[f"{name}/step_8_1_0/labels"]))
    assert differs > 0
