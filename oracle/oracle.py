"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU checkers.

- liboracle.so: the plain-C restatement of the reference's sketch-based LPA (rak_oracle.c).
- _ref/libref_cpu.so: the reference's own CPU code compiled from its sources (ref_bridge.cpp);
  present only where the reference sources were available at build time.
- _ref/ref_lpa_cuda: the reference's own GPU path as a separate program (ref_main_cuda.cu).
- _ref/ref_sketch_cuda: the reference's own GPU sketch device functions on given streams, as a
  separate program (ref_sketch_cuda.cu), the pin of the GPU-rule restatement.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and only as
the checker or the CPU baseline; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_CPU_SO = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_CUDA_BIN = os.path.join(HERE, "_ref", "ref_lpa_cuda")
REF_SKETCH_BIN = os.path.join(HERE, "_ref", "ref_sketch_cuda")
GEN_SO = os.path.join(HERE, "liborcgen.so")
NONE = 0xFFFFFFFF
MAX_SLOTS = 32


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


if not os.path.exists(ORACLE_SO) or not os.path.exists(GEN_SO):
    build()
_o = C.CDLL(ORACLE_SO)


class orc_csr(C.Structure):
    _fields_ = [("n", C.c_int64), ("off", C.c_void_p), ("tgt", C.c_void_p), ("wt", C.c_void_p)]


class orc_layout(C.Structure):
    _fields_ = [("lane_max", C.c_int64), ("hub_min", C.c_int64), ("hub_chunk", C.c_int64)]


class orc_opts(C.Structure):
    _fields_ = [("slots", C.c_int), ("rescan", C.c_int), ("split", C.c_int), ("layout", orc_layout),
                ("tolerance", C.c_double), ("max_iterations", C.c_int), ("pickless_step", C.c_int),
                ("check_on_pickless", C.c_int), ("gpu_rule", C.c_int), ("tie_until", C.c_int)]


class orc_sketch(C.Structure):
    _fields_ = [("k", C.c_uint32 * MAX_SLOTS), ("w", C.c_float * MAX_SLOTS)]


def _sig(lib, name, res, *args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


P = C.c_void_p
_sig(_o, "orc_sketch_clear", None, C.POINTER(orc_sketch), C.c_int)
_sig(_o, "orc_mg_accumulate", None, C.POINTER(orc_sketch), C.c_int, C.c_uint32, C.c_float)
_sig(_o, "orc_bm_accumulate", None, C.POINTER(orc_sketch), C.c_uint32, C.c_float)
_sig(_o, "orc_sketch_merge", None, C.POINTER(orc_sketch), C.POINTER(orc_sketch), C.c_int)
_sig(_o, "orc_sketch_choose", None, C.POINTER(orc_sketch), C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_float))
_sig(_o, "orc_tie_hash", C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32)
_sig(_o, "orc_sketch_choose_hashed", None, C.POINTER(orc_sketch), C.c_int, C.c_uint32, C.c_uint32,
     C.POINTER(C.c_uint32), C.POINTER(C.c_float))
_sig(_o, "orc_mg_accumulate_gpu", None, C.POINTER(orc_sketch), C.c_int, C.c_uint32, C.c_float)
_sig(_o, "orc_sketch_choose_gpu", None, C.POINTER(orc_sketch), C.c_int, C.POINTER(C.c_uint32), C.POINTER(C.c_float))
_sig(_o, "orc_choose", None, C.POINTER(orc_csr), C.POINTER(orc_opts), C.c_uint32, P, C.POINTER(C.c_uint32),
     C.POINTER(C.c_float))
_sig(_o, "orc_sync_step", C.c_uint64, C.POINTER(orc_csr), C.POINTER(orc_opts), C.c_int, P, P, P, P,
     C.POINTER(C.c_uint64), C.POINTER(C.c_uint64))
_sig(_o, "orc_sync_run", C.c_int, C.POINTER(orc_csr), C.POINTER(orc_opts), P, P, C.POINTER(C.c_uint64))
_sig(_o, "orc_serial_run", C.c_int, C.POINTER(orc_csr), C.c_int, C.c_int, C.c_double, C.c_int, P)
_sig(_o, "orc_modularity", C.c_double, C.POINTER(orc_csr), P)

# Layout defaults of the product (rak_internal.hpp DEFAULT_LANE_MAX / HUB_MIN / HUB_CHUNK).
DEFAULT_LAYOUT = (256, 65536, 8192)   # the library's defaults (lane_max, hub_min, hub_chunk)


class Graph:
    """Host CSR view: int64 offsets, uint32 targets, float32 weights or None."""

    def __init__(self, offsets, targets, weights=None):
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        self.targets = np.ascontiguousarray(targets, dtype=np.uint32)
        self.weights = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        self.n = len(self.offsets) - 1
        self.m = len(self.targets)
        self.c = orc_csr(self.n, self.offsets.ctypes.data, self.targets.ctypes.data if len(self.targets) else None,
                         self.weights.ctypes.data if self.weights is not None else None)

    @staticmethod
    def of(g) -> "Graph":
        return g if isinstance(g, Graph) else Graph(g.offsets, g.targets, g.weights)


def make_opts(slots=8, rescan=0, split=0, layout=DEFAULT_LAYOUT, tolerance=0.05, max_iterations=20,
              pickless_step=0, check_on_pickless=1, gpu_rule=0, tie_until=0) -> orc_opts:
    return orc_opts(slots, rescan, split, orc_layout(*layout), tolerance, max_iterations, pickless_step,
                    check_on_pickless, gpu_rule, tie_until)


def sync_step(g, o: orc_opts, iteration, vcom_prev, aff_prev):
    g = Graph.of(g)
    vp = np.ascontiguousarray(vcom_prev, dtype=np.uint32)
    ap = np.ascontiguousarray(aff_prev, dtype=np.uint8)
    vn = np.empty_like(vp)
    an = np.empty_like(ap)
    e, p = C.c_uint64(0), C.c_uint64(0)
    ch = _o.orc_sync_step(C.byref(g.c), C.byref(o), iteration, vp.ctypes.data, ap.ctypes.data, vn.ctypes.data,
                          an.ctypes.data, C.byref(e), C.byref(p))
    return vn, an, int(ch), int(e.value), int(p.value)


def sync_run(g, o: orc_opts, q=None):
    g = Graph.of(g)
    out = np.empty(g.n, dtype=np.uint32)
    qq = None if q is None else np.ascontiguousarray(q, dtype=np.uint32)
    e = C.c_uint64(0)
    it = _o.orc_sync_run(C.byref(g.c), C.byref(o), None if qq is None else qq.ctypes.data, out.ctypes.data,
                         C.byref(e))
    return out, int(it), int(e.value)


def serial_run(g, slots=8, rescan=1, tolerance=0.05, max_iterations=20):
    g = Graph.of(g)
    out = np.empty(g.n, dtype=np.uint32)
    it = _o.orc_serial_run(C.byref(g.c), slots, rescan, tolerance, max_iterations, out.ctypes.data)
    return out, int(it)


def modularity(g, labels) -> float:
    g = Graph.of(g)
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    return float(_o.orc_modularity(C.byref(g.c), lab.ctypes.data))


def choose(g, o: orc_opts, u, vcom):
    g = Graph.of(g)
    v = np.ascontiguousarray(vcom, dtype=np.uint32)
    c, w = C.c_uint32(0), C.c_float(0)
    _o.orc_choose(C.byref(g.c), C.byref(o), u, v.ctypes.data, C.byref(c), C.byref(w))
    return int(c.value), float(w.value)


class Sketch:
    """A Misra-Gries (slots >= 2) or Boyer-Moore (slots == 1) sketch, for stream-level tests."""

    def __init__(self, slots, gpu_rule=False):
        self.slots = slots
        self.gpu = gpu_rule
        self.s = orc_sketch()
        _o.orc_sketch_clear(C.byref(self.s), slots)

    def add(self, c, w):
        if self.slots == 1:
            _o.orc_bm_accumulate(C.byref(self.s), c, w)
        elif self.gpu:
            _o.orc_mg_accumulate_gpu(C.byref(self.s), self.slots, c, w)
        else:
            _o.orc_mg_accumulate(C.byref(self.s), self.slots, c, w)
        return self

    def merge(self, other: "Sketch"):
        _o.orc_sketch_merge(C.byref(self.s), C.byref(other.s), self.slots)
        return self

    def choose(self):
        c, w = C.c_uint32(0), C.c_float(0)
        f = _o.orc_sketch_choose_gpu if self.gpu else _o.orc_sketch_choose
        f(C.byref(self.s), self.slots, C.byref(c), C.byref(w))
        return int(c.value), float(w.value)

    def slots_list(self):
        return [(int(self.s.k[i]), float(self.s.w[i])) for i in range(self.slots)]


# ---- the library's synthetic graphs, restated (rmat_gen.c) -----------------------------------
class og_graph(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("off", P), ("tgt", P), ("wt", P)]


_gen = C.CDLL(GEN_SO)
_sig(_gen, "og_gen_rmat", C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_float,
     C.c_float, C.c_int, C.POINTER(og_graph))
_sig(_gen, "og_gen_lattice", C.c_int, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_uint64, C.c_int,
     C.POINTER(og_graph))
_sig(_gen, "og_free", None, C.POINTER(og_graph))


def _take(og: og_graph) -> Graph:
    """A Graph whose arrays view the generated C arrays (no copy: a scale-27 graph is ~17 GB); the
    C arrays are freed when the Graph is collected, so keep the Graph while its arrays are used."""
    n, m = int(og.n), int(og.m)
    off = np.ctypeslib.as_array(C.cast(og.off, C.POINTER(C.c_int64)), shape=(n + 1,))
    tgt = np.ctypeslib.as_array(C.cast(og.tgt, C.POINTER(C.c_uint32)), shape=(max(m, 1),))[:m]
    wt = np.ctypeslib.as_array(C.cast(og.wt, C.POINTER(C.c_float)), shape=(max(m, 1),))[:m] if og.wt else None
    g = Graph(off, tgt, wt)
    g._owner = og
    weakref.finalize(g, _gen.og_free, C.byref(og))
    return g


def gen_rmat(scale, edge_factor, a=0.57, b=0.19, c=0.19, seed=42, w_lo=1.0, w_hi=1.0, threads=0) -> Graph:
    """The library's symmetric R-MAT (rak_gen_rmat), restated in C: bit-identical arrays."""
    og = og_graph()
    st = _gen.og_gen_rmat(scale, edge_factor, a, b, c, seed, w_lo, w_hi, threads, C.byref(og))
    if st:
        raise RuntimeError(f"og_gen_rmat failed ({st})")
    return _take(og)


def gen_lattice(width, height, p_delete=0.05, shortcut=0.01, seed=42, threads=0) -> Graph:
    """The library's perturbed 2D lattice (rak_gen_lattice), restated in C: bit-identical arrays."""
    og = og_graph()
    st = _gen.og_gen_lattice(width, height, p_delete, shortcut, seed, threads, C.byref(og))
    if st:
        raise RuntimeError(f"og_gen_lattice failed ({st})")
    return _take(og)


# ---- the reference itself, compiled from its sources ------------------------------------------
_ref = None


def have_ref_cpu() -> bool:
    return os.path.exists(REF_CPU_SO)


def ref_cpu():
    global _ref
    if _ref is None:
        if not have_ref_cpu():
            raise FileNotFoundError(REF_CPU_SO)
        _ref = C.CDLL(REF_CPU_SO)
        _sig(_ref, "ref_lowmem_omp", C.c_int, C.c_int64, P, P, P, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
             C.c_int, P, C.POINTER(C.c_float))
        _sig(_ref, "ref_lowmem_omp_sample", C.c_int64, C.c_int64, P, P, P, C.c_int, C.c_int, C.c_int64, C.c_int,
             C.POINTER(C.c_float))
        _sig(_ref, "ref_gve_omp_sample", C.c_int64, C.c_int64, P, P, P, C.c_int64, C.c_int, C.POINTER(C.c_float))
        _sig(_ref, "ref_gve_omp", C.c_int, C.c_int64, P, P, P, C.c_double, C.c_int, C.c_int, C.c_int, P,
             C.POINTER(C.c_float))
        _sig(_ref, "ref_modularity", C.c_double, C.c_int64, P, P, P, P)
        _sig(_ref, "ref_sync_step", C.c_int64, C.c_int64, P, P, P, C.c_int, C.c_int, C.c_int, P, P, P, P)
        _sig(_ref, "ref_sketch_stream", C.c_int, C.c_int, C.c_int64, P, P, P, P)
        _sig(_ref, "ref_vertex_order", None, C.c_int64, P, P)
        _sig(_ref, "ref_read_mtx", C.c_int, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int64),
             C.POINTER(C.c_int64), P, P, P)
    return _ref


def ref_read_mtx(path, weighted=False, symmetrize=True):
    """The reference driver's loading of an MTX file (readMtxOmpW + symmetrizeOmpU), 0-based:
    (offsets int64, targets uint32, weights float32 or None)."""
    n, m = C.c_int64(0), C.c_int64(0)
    ref_cpu().ref_read_mtx(str(path).encode(), int(weighted), int(symmetrize), C.byref(n), C.byref(m), None, None, None)
    off = np.empty(n.value + 1, np.int64)
    tgt = np.empty(max(m.value, 1), np.uint32)
    wt = np.empty(max(m.value, 1), np.float32)
    ref_cpu().ref_read_mtx(str(path).encode(), int(weighted), int(symmetrize), C.byref(n), C.byref(m),
                           off.ctypes.data, tgt.ctypes.data, wt.ctypes.data)
    return off, tgt[:m.value], (wt[:m.value] if weighted else None)


def ref_vertex_order(g):
    """The reference GPU entry's vertex order (std::partition by degree < 4, then < 128)."""
    g = Graph.of(g)
    ks = np.empty(g.n, np.uint32)
    ref_cpu().ref_vertex_order(g.n, g.offsets.ctypes.data, ks.ctypes.data)
    return ks


def ref_sketch_stream(slots, comm, wts):
    """Final (key, weight) slots after the reference accumulates the stream."""
    c = np.ascontiguousarray(comm, dtype=np.uint32)
    w = np.ascontiguousarray(wts, dtype=np.float32)
    k = np.empty(slots, dtype=np.uint32)
    ww = np.empty(slots, dtype=np.float32)
    if ref_cpu().ref_sketch_stream(slots, len(c), c.ctypes.data, w.ctypes.data, k.ctypes.data, ww.ctypes.data):
        raise ValueError(f"unsupported slots {slots}")
    return k, ww


def _gp(g: Graph):
    return g.n, g.offsets.ctypes.data, g.targets.ctypes.data if len(g.targets) else None, \
        g.weights.ctypes.data if g.weights is not None else None


def ref_lowmem_omp(g, slots=8, rescan=1, tolerance=0.05, max_iterations=20, threads=1, repeat=1):
    """rakLowmemStaticOmp<MULTI,RESCAN,SLOTS> (reference, inc/rakLowmem.hxx:277-284)."""
    g = Graph.of(g)
    out = np.empty(g.n, dtype=np.uint32)
    t = C.c_float(0)
    it = ref_cpu().ref_lowmem_omp(*_gp(g), slots, rescan, tolerance, max_iterations, threads, repeat,
                                  out.ctypes.data, C.byref(t))
    if it < 0:
        raise ValueError(f"unsupported slots {slots}")
    return out, int(it), float(t.value)


def ref_lowmem_omp_sample(g, slots=8, rescan=1, stride=1, threads=1):
    """One first iteration of the reference's rakLowmemInvokeOmp<MULTI,RESCAN,SLOTS> with
    rakLowmemStaticOmp's hooks, restricted to every stride-th vertex (inc/rakLowmem.hxx:226-284).
    Returns (traversed edges, the reference's own time in ms)."""
    g = Graph.of(g)
    t = C.c_float(0)
    e = ref_cpu().ref_lowmem_omp_sample(*_gp(g), slots, rescan, stride, threads, C.byref(t))
    if e < 0:
        raise ValueError(f"unsupported slots {slots}")
    return int(e), float(t.value)


def ref_gve_omp_sample(g, stride=1, threads=1):
    """The same sample of GVE-LPA's first iteration (rakInvokeOmp with rakStaticOmp's hooks,
    inc/rak.hxx:272-327). Returns (traversed edges, time in ms)."""
    g = Graph.of(g)
    t = C.c_float(0)
    e = ref_cpu().ref_gve_omp_sample(*_gp(g), stride, threads, C.byref(t))
    return int(e), float(t.value)


def ref_gve_omp(g, tolerance=0.05, max_iterations=20, threads=1, repeat=1):
    """rakStaticOmp (reference GVE-LPA, inc/rak.hxx:320-327)."""
    g = Graph.of(g)
    out = np.empty(g.n, dtype=np.uint32)
    t = C.c_float(0)
    it = ref_cpu().ref_gve_omp(*_gp(g), tolerance, max_iterations, threads, repeat, out.ctypes.data, C.byref(t))
    return out, int(it), float(t.value)


def ref_modularity(g, labels) -> float:
    g = Graph.of(g)
    lab = np.ascontiguousarray(labels, dtype=np.uint32)
    return float(ref_cpu().ref_modularity(*_gp(g), lab.ctypes.data))


def ref_sync_step(g, slots, rescan, pickless, vcom_prev, aff_prev):
    g = Graph.of(g)
    vp = np.ascontiguousarray(vcom_prev, dtype=np.uint32)
    ap = np.ascontiguousarray(aff_prev, dtype=np.uint8)
    vn = np.empty_like(vp)
    an = np.empty_like(ap)
    ch = ref_cpu().ref_sync_step(*_gp(g), slots, rescan, pickless, vp.ctypes.data, ap.ctypes.data,
                                 vn.ctypes.data, an.ctypes.data)
    if ch < 0:
        raise ValueError(f"unsupported slots {slots}")
    return vn, an, int(ch)


def have_ref_cuda() -> bool:
    return os.path.exists(REF_CUDA_BIN)


def ref_lowmem_cuda(g, slots=8, repeat=1, tolerance=0.05, max_iterations=20, timeout=600):
    """The reference's own GPU path rakLowmemStaticCuda<slots> run as a separate process (slots 0:
    the reference's ν-LPA, rakStaticCuda, with per-vertex hashtables)."""
    g = Graph.of(g)
    with tempfile.TemporaryDirectory() as d:
        gp, lp = os.path.join(d, "g.rakcsr"), os.path.join(d, "labels.bin")
        with open(gp, "wb") as f:
            f.write(b"RAKCSR01")
            f.write(np.array([g.n, len(g.targets)], dtype=np.int64).tobytes())
            f.write(np.array([1 if g.weights is not None else 0], dtype=np.int32).tobytes())
            f.write(g.offsets.tobytes())
            f.write(g.targets.tobytes())
            if g.weights is not None:
                f.write(g.weights.tobytes())
        p = subprocess.run([REF_CUDA_BIN, gp, str(slots), lp, str(repeat), str(tolerance), str(max_iterations)],
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"ref_lpa_cuda failed ({p.returncode}): {p.stderr[-2000:]}")
        info = json.loads(p.stdout.strip().splitlines()[-1])
        labels = np.fromfile(lp, dtype=np.uint32)
    return labels, info


def have_ref_sketch_cuda() -> bool:
    return os.path.exists(REF_SKETCH_BIN)


def ref_sketch_streams_gpu(slots, streams, own=None, timeout=120):
    """The reference's own GPU Misra-Gries accumulate and tournament argmax (inc/sketchCuda.hxx,
    sketchAccumulateWarpCudU and sketchMaxGroupReduceCudU) on each stream of (community, weight)
    pairs, from cleared keys: per stream the slots [(key, weight)] before the argmax and the
    (key, weight) it picks. slots 1: the reference's Boyer-Moore scan
    (rakLowmemBmScanCommunitiesCud) from own[i], the own label of stream i's vertex. Runs
    oracle/_ref/ref_sketch_cuda as a separate process."""
    off = np.zeros(len(streams) + 1, np.int64)
    off[1:] = np.cumsum([len(st) for st in streams])
    comm = np.array([c for st in streams for c, _ in st], np.uint32)
    wts = np.array([w for st in streams for _, w in st], np.float32)
    ns, total = len(streams), int(off[-1])
    with tempfile.TemporaryDirectory() as d:
        ip, op = os.path.join(d, "s.in"), os.path.join(d, "s.out")
        with open(ip, "wb") as f:
            f.write(b"RAKSKT01")
            f.write(np.array([slots], np.int32).tobytes())
            f.write(np.array([ns, total], np.int64).tobytes())
            f.write(off.tobytes())
            f.write(comm.tobytes())
            f.write(wts.tobytes())
            if slots == 1:
                f.write(np.asarray(own, np.uint32).tobytes())
        p = subprocess.run([REF_SKETCH_BIN, ip, op], capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"ref_sketch_cuda failed ({p.returncode}): {p.stderr[-2000:]}")
        raw = open(op, "rb").read()
    nk = ns * slots
    keys = np.frombuffer(raw, np.uint32, nk, 0).reshape(ns, slots)
    ws = np.frombuffer(raw, np.float32, nk, 4 * nk).reshape(ns, slots)
    bk = np.frombuffer(raw, np.uint32, ns, 8 * nk)
    bw = np.frombuffer(raw, np.float32, ns, 8 * nk + 4 * ns)
    return [([(int(keys[i, j]), float(ws[i, j])) for j in range(slots)], (int(bk[i]), float(bw[i])))
            for i in range(ns)]
