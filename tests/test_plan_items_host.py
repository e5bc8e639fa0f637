"""The plan's arithmetic, checked on the host by compiling the library's own header
(rak_internal.hpp) into tests/cpp/plan_items.cpp: the one-lane work items (lane_item_for,
region_items) and the kernel's loop over an item's batches visit every one-lane vertex exactly
once, for region sizes 0..20000 and grids of 1 to 100000 warps; and plan_key maps every degree into
the key histogram's range and to its region (one lane, the smallest sufficient lane group, or
split) for five layouts."""
import os
import subprocess

from conftest import ROOT


def test_every_one_lane_vertex_in_exactly_one_item(tmp_path):
    exe = str(tmp_path / "plan_items")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "rak-lowmem-communities-cuda_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "cpp", "plan_items.cpp"), "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
