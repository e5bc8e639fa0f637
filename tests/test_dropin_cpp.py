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
def test_dropin_finds_planted_cliques(tmp_path):
    p = subprocess.run([build(tmp_path)], capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout + p.stderr
    lines = p.stdout.splitlines()
    for line in lines[:2]:
        m = [int(v) for v in line.split()]
        assert len(m) == 11 and m[0] == 0                   # vertex 0 does not exist
        assert len(set(m[1:6])) == 1 and len(set(m[6:11])) == 1 and m[1] != m[6]
        assert 1 <= m[1] <= 10 and 1 <= m[6] <= 10          # names are vertex keys
