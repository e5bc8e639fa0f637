"""The C++ drop-in header (include/rak_lowmem.hpp) compiles against a reference-style graph type,
links against librak_lowmem.so, reports a missing GPU as an exception rather than exiting, and on
a GPU finds the two planted cliques."""
import os
import subprocess

import pytest

from conftest import PKG, ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp")


def build(tmp_path):
    exe = str(tmp_path / "dropin")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), SRC, "-L", PKG,
                    "-lrak_lowmem", f"-Wl,-rpath,{PKG}", "-o", exe], check=True)
    return exe


def test_dropin_builds_and_reports_no_device(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = subprocess.run([build(tmp_path)], capture_output=True, text=True)
    assert p.returncode == 3 and "error 6" in p.stdout, p.stdout + p.stderr


@pytest.mark.gpu
def test_dropin_runs_on_gpu(tmp_path):
    import numpy as np
    import oracle as orc
    p = subprocess.run([build(tmp_path)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout + p.stderr
    rows = [[int(v) for v in line.split()] for line in p.stdout.splitlines()[:3]]
    for m in rows:
        assert len(m) == 11 and m[0] == 0                    # vertex 0 does not exist
        assert all(1 <= c <= 10 for c in m[1:])              # community names are vertex keys
    # the synchronous run equals the oracle on the same graph with ids shifted to 0-based
    edges = [(i, j) for b in (0, 5) for i in range(b, b + 5) for j in range(i + 1, b + 5)] + [(4, 5)]
    adj = [[] for _ in range(10)]
    for i, j in edges:
        adj[i].append(j)
        adj[j].append(i)
    off = np.cumsum([0] + [len(a) for a in adj]).astype(np.int64)
    tgt = np.concatenate([np.array(a, np.uint32) for a in adj])
    ref, _, _ = orc.sync_run(orc.Graph(off, tgt), orc.make_opts(slots=8, rescan=1))
    assert [c - 1 for c in rows[2][1:]] == [int(v) for v in ref]
