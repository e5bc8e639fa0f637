"""bench.py --impl reference: the reference's own CPU MG8-LPA (built from its sources into
oracle/_ref) timed on the host cores, printing one JSON line with the same metric, unit and config
fields as the GPU arm, a cpu_baseline describing the run and an e2e object."""
import json
import os
import subprocess
import sys

import pytest

import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not orc.have_ref_cpu(), reason="reference CPU build (oracle/_ref) not present")
def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "rmat16_ef16", "--steps", "2", "--warmup", "3"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "edges/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 3 and line["n_gpus"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["workload"] == "rmat16_ef16" and line["config"]["n"] == 65536
