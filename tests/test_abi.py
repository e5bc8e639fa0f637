"""The C-ABI library without a GPU: it loads, exports every symbol include/rak_lowmem.h declares,
and its host-side logic (options, status strings, CSR validation, plan summary) behaves."""
import ctypes
import os
import re

import numpy as np
import pytest

import rak_lowmem as rl
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rak_lowmem.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rak_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(rl.LIB_PATH)
    syms = declared_symbols()
    assert "rak_lowmem_cuda" in syms and "rak_graph_step" in syms and len(syms) >= 15
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_version_and_status_strings():
    assert rl.abi_version() == 1
    for s in range(9):
        assert rl._lib.rak_status_string(s)


def test_option_defaults_follow_reference():
    o = rl.options()
    # RakOptions defaults (inc/rak.hxx:37-38) and the reference's νMG8 choice (main.cxx:90).
    assert (o.repeat, o.tolerance, o.max_iterations, o.slots) == (1, 0.05, 20, 8)
    assert o.mode == rl.MODE_ASYNC and o.rescan == -1 and o.pickless_step == -1 and o.validate == 1
    # rule set and label order resolve per mode and entry point (-1: the library's default)
    assert o.sketch_rule == -1 and o.label_order == -1


def test_no_device_reported_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    c = ctypes.c_void_p()
    assert rl._lib.rak_ctx_create(0, ctypes.byref(c)) == 6


def small():
    off = np.array([0, 2, 3, 4, 4], np.int64)
    tgt = np.array([1, 2, 0, 0], np.uint32)
    return rl.HostGraph(off, tgt)


def test_host_validation():
    assert rl.validate_host(small()) == 0
    g = small()
    bad = rl.HostGraph(g.offsets.copy(), np.array([1, 2, 0, 9], np.uint32))
    assert rl.validate_host(bad) == 2                                   # target out of range
    off = g.offsets.copy(); off[2] = 1; off[1] = 3
    assert rl.validate_host(rl.HostGraph(off, g.targets)) == 2           # offsets not monotone
    off = g.offsets.copy(); off[0] = 1
    assert rl.validate_host(rl.HostGraph(off, g.targets)) == 2           # offsets[0] != 0
    assert rl.validate_host(g.with_offsets32()) == 0


def test_plan_summary_partitions_vertices():
    g = rl.gen_rmat(12, 16, seed=1)
    counts, chunks = rl.plan_summary(g, lane_max=16, hub_min=512, hub_chunk=256)
    deg = g.degrees()
    assert sum(counts) == g.n
    assert counts[7] == int((deg == 0).sum())
    assert counts[0] == int(((deg >= 1) & (deg <= 16)).sum())
    assert counts[6] == int((deg > 512).sum())
    assert chunks == int(((deg[deg > 512] + 255) // 256).sum())
    with pytest.raises(rl.RakError):
        rl.plan_summary(g, lane_max=4096)                               # above MAX_LANE_MAX


def test_tune_space_defaults():
    sp = rl.tune_space()
    assert list(sp.lane_max)[:sp.n_lane_max] == [32, 64, 128, 256]
    assert list(sp.hub_min)[:sp.n_hub_min] == [4096, 8192, 16384, 32768, 65536]
    assert list(sp.hub_chunk)[:sp.n_hub_chunk] == [2048, 4096, 8192, 16384]
    assert list(sp.slots)[:sp.n_slots] == [4, 8, 16]
    assert sp.repeats == 2 and sp.quality_rel == 0.005 and sp.quality_abs == 0.001
    assert sp.label_orders == 1
    import ctypes
    assert ctypes.sizeof(rl.rak_tune_entry) == 8 * 4 + 3 * 8      # label_order + reserved keep alignment
    sp = rl.tune_space(slots=[8], hub_chunk=[4096, 8192], repeats=1)
    assert sp.n_slots == 1 and sp.n_hub_chunk == 2 and sp.repeats == 1
    with pytest.raises(ValueError):
        rl.tune_space(slots=[1, 2, 4, 8, 16, 32])
