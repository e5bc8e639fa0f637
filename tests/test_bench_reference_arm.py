"""bench.py --impl reference: the reference's own CPU MG8-LPA (built from its sources into
oracle/_ref) timed on the host cores, printing one JSON line with the same metric, unit and config
fields as the GPU arm, a cpu_baseline describing the run and an e2e object. The arm builds its graph
with the oracle's generator and must not load this repository's library."""
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
    assert line["config"]["m"] == 1819320      # the library's generator gives the same graph


@pytest.mark.skipif(not orc.have_ref_cpu(), reason="reference CPU build (oracle/_ref) not present")
def test_reference_arm_loads_nothing_of_the_library():
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'rmat16_ef16', "
            "'--steps', '1', '--warmup', '3']; runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('LIBS', int('librak_lowmem' in maps), int('rak_lowmem' in sys.modules), int('libref_cpu' in maps))")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    libs = [l for l in out.stdout.splitlines() if l.startswith("LIBS")][-1].split()[1:]
    assert libs == ["0", "0", "1"], libs
