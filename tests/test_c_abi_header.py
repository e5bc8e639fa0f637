"""The boundary is a C ABI: include/rak_lowmem.h compiles as strict C11 (no C++ in the
signatures or structs), links against librak_lowmem.so, and every public struct has the same size
and field offsets in C as in the ctypes binding the tests and bench use (so the two cannot drift
apart unnoticed). Runs without a GPU: only option defaults are called."""
import ctypes
import os
import subprocess

import pytest

import rak_lowmem as rl
from conftest import PKG, ROOT

STRUCTS = ["rak_csr", "rak_options", "rak_result", "rak_batch_csr", "rak_server_options", "rak_server_stats",
           "rak_tune_space", "rak_tune_entry", "rak_host_csr"]


def c_program():
    lines = ['#include "rak_lowmem.h"', "#include <stddef.h>", "#include <stdio.h>", "int main(void) {",
             "  rak_options o; rak_options_default(&o);",
             "  rak_tune_space sp; rak_tune_space_default(&sp);",
             '  printf("defaults %d %d %d %d\\n", o.slots, o.sketch_rule, o.label_order, sp.label_orders);']
    for s in STRUCTS:
        lines.append(f'  printf("size {s} %zu\\n", sizeof({s}));')
        for f in getattr(rl, s)._fields_:
            lines.append(f'  printf("off {s} {f[0]} %zu\\n", offsetof({s}, {f[0]}));')
    lines += ["  return 0;", "}"]
    return "\n".join(lines) + "\n"


def test_header_is_c11_and_layouts_match_the_binding(tmp_path):
    src, exe = tmp_path / "abi.c", str(tmp_path / "abi")
    src.write_text(c_program())
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-std=c11", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", PKG, "-lrak_lowmem", f"-Wl,-rpath,{PKG}", "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines()
    assert out[0] == "defaults 8 -1 -1 1"
    for line in out[1:]:
        kind, name, *rest = line.split()
        cls = getattr(rl, name)
        if kind == "size":
            assert int(rest[0]) == ctypes.sizeof(cls), name
        else:
            field, off = rest
            assert int(off) == getattr(cls, field).offset, (name, field)
