"""Python binding (ctypes) of librak_lowmem.so, the B200 memory-efficient label propagation library.

Mirrors the reference's call shape: ``rakLowmemStaticCuda<SLOTS>(x, o) -> RakResult`` becomes
``Context.lowmem(graph, q=None, options) -> (membership, result)`` with the same option names
(repeat, tolerance, max_iterations) and result fields (iterations, time_ms, marking_time_ms,
initialization_time_ms, memory_gb). The native library is required: importing this module raises
if ``librak_lowmem.so`` is missing; there is no CPU fallback.

Host graphs are numpy arrays; device graphs are torch CUDA tensors (torch only provides device
memory and streams here).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librak_lowmem.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {_HERE}` (or __graft_entry__.build())")
_lib = C.CDLL(LIB_PATH)

HOST, DEVICE = 0, 1
MODE_ASYNC, MODE_SYNC, MODE_SYNC_SPLIT = 0, 1, 2
STATUS = {0: "ok", 1: "invalid argument", 2: "invalid CSR", 3: "out of memory", 4: "CUDA error",
          5: "timeout", 6: "no device", 7: "unsupported", 8: "busy"}


class rak_csr(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("offset_bits", C.c_int32), ("location", C.c_int32),
                ("offsets", C.c_void_p), ("targets", C.c_void_p), ("weights", C.c_void_p)]


class rak_options(C.Structure):
    _fields_ = [("repeat", C.c_int32), ("tolerance", C.c_double), ("max_iterations", C.c_int32),
                ("slots", C.c_int32), ("mode", C.c_int32), ("rescan", C.c_int32),
                ("pickless_step", C.c_int32), ("check_on_pickless", C.c_int32), ("lane_max", C.c_int32),
                ("hub_min", C.c_int32), ("hub_chunk", C.c_int32), ("validate", C.c_int32),
                ("compute_modularity", C.c_int32), ("start_iteration", C.c_int32),
                ("initial_flags", C.c_void_p), ("sketch_rule", C.c_int32), ("label_order", C.c_int32),
                ("wait_timeout_ns", C.c_int64), ("tie_break", C.c_int32), ("tie_iterations", C.c_int32),
                ("edge_staging", C.c_int32), ("max_blocks", C.c_int32), ("dense_pct", C.c_int32),
                ("renumber", C.c_int32), ("reserved", C.c_int64 * 3)]


class rak_result(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("time_ms", C.c_float), ("marking_time_ms", C.c_float),
                ("initialization_time_ms", C.c_float), ("memory_gb", C.c_float), ("plan_ms", C.c_float),
                ("h2d_ms", C.c_float), ("d2h_ms", C.c_float), ("peak_device_bytes", C.c_uint64),
                ("traversed_edges", C.c_uint64), ("processed_vertices", C.c_uint64),
                ("changed_last", C.c_uint64), ("moved_vertices", C.c_uint64), ("moved_edges", C.c_uint64),
                ("loop_ms", C.c_float), ("reserved_f", C.c_float), ("modularity", C.c_double),
                ("marked_edges", C.c_uint64), ("dense_iterations", C.c_int32), ("reserved_r", C.c_int32)]


class rak_batch_csr(C.Structure):
    _fields_ = [("graphs", C.c_int64), ("n", C.c_int64), ("m", C.c_int64), ("location", C.c_int32),
                ("reserved", C.c_int32), ("graph_offsets", C.c_void_p), ("offsets", C.c_void_p),
                ("targets", C.c_void_p), ("weights", C.c_void_p)]


class rak_server_options(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("max_graphs_per_launch", C.c_int32), ("slots", C.c_int32),
                ("queue_capacity", C.c_int32), ("reserved", C.c_int32), ("run", rak_options)]


class rak_server_stats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("rejected", C.c_uint64),
                ("launches", C.c_uint64), ("graphs_launched", C.c_uint64), ("edges_completed", C.c_uint64),
                ("device_bytes_in_use", C.c_uint64), ("max_concurrent_launches", C.c_int32),
                ("pending", C.c_int32), ("load_ms", C.c_double), ("plan_ms", C.c_double), ("run_ms", C.c_double),
                ("pack_ms", C.c_double), ("plan_host_ms", C.c_double), ("enqueue_ms", C.c_double)]


class rak_tune_space(C.Structure):
    _fields_ = [("lane_max", C.c_int32 * 8), ("n_lane_max", C.c_int32), ("hub_min", C.c_int32 * 8),
                ("n_hub_min", C.c_int32), ("hub_chunk", C.c_int32 * 8), ("n_hub_chunk", C.c_int32),
                ("slots", C.c_int32 * 5), ("n_slots", C.c_int32), ("repeats", C.c_int32), ("label_orders", C.c_int32),
                ("quality_rel", C.c_double), ("quality_abs", C.c_double)]


class rak_tune_entry(C.Structure):
    _fields_ = [("lane_max", C.c_int32), ("hub_min", C.c_int32), ("hub_chunk", C.c_int32), ("slots", C.c_int32),
                ("iterations", C.c_int32), ("accepted", C.c_int32), ("label_order", C.c_int32),
                ("reserved", C.c_int32), ("ms", C.c_double), ("modularity", C.c_double),
                ("edges_per_s", C.c_double)]


class rak_host_csr(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("offsets", C.c_void_p), ("targets", C.c_void_p),
                ("weights", C.c_void_p), ("truth", C.c_void_p)]


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


P = C.c_void_p
_sig("rak_abi_version", C.c_int)
_sig("rak_status_string", C.c_char_p, C.c_int)
_sig("rak_options_default", None, C.POINTER(rak_options))
_sig("rak_ctx_create", C.c_int, C.c_int, C.POINTER(P))
_sig("rak_ctx_destroy", C.c_int, P)
_sig("rak_ctx_set_stream", C.c_int, P, P)
_sig("rak_ctx_set_memory_keep", C.c_int, P, C.c_uint64)
_sig("rak_ctx_last_error", C.c_char_p, P)
_sig("rak_lowmem_cuda", C.c_int, P, C.POINTER(rak_csr), P, C.POINTER(rak_options), P, C.POINTER(rak_result))
_sig("rak_graph_create", C.c_int, P, C.POINTER(rak_csr), C.POINTER(rak_options), C.POINTER(P))
_sig("rak_graph_destroy", C.c_int, P)
_sig("rak_graph_device_bytes", C.c_uint64, P)
_sig("rak_graph_run", C.c_int, P, P, P, C.POINTER(rak_options), P, C.POINTER(rak_result))
_sig("rak_graph_step", C.c_int, P, P, C.POINTER(rak_options), C.c_int, P, P, P, P, C.POINTER(C.c_uint64))
_sig("rak_modularity_f64", C.c_int, P, C.POINTER(rak_csr), P, C.POINTER(C.c_double))
_sig("rak_batch_create", C.c_int, P, C.POINTER(rak_batch_csr), C.POINTER(rak_options), C.POINTER(P))
_sig("rak_batch_destroy", C.c_int, P)
_sig("rak_batch_launch", C.c_int, P, P, P, C.POINTER(rak_options), P)
_sig("rak_batch_results", C.c_int, P, P, P, C.POINTER(rak_result))
_sig("rak_batch_capture", C.c_int, P, P, P, C.POINTER(rak_options), P)
_sig("rak_batch_replay", C.c_int, P, P)
_sig("rak_batch_modularity_f64", C.c_int, P, P, P, P)
_sig("rak_server_options_default", None, C.POINTER(rak_server_options))
_sig("rak_tune_space_default", None, C.POINTER(rak_tune_space))
_sig("rak_graph_autotune", C.c_int, P, P, C.POINTER(rak_options), C.POINTER(rak_tune_space), P,
     C.POINTER(rak_options), C.POINTER(rak_tune_entry), C.c_int32, C.POINTER(C.c_int32))
_sig("rak_batch_autotune", C.c_int, P, P, C.c_int64, C.POINTER(rak_options), C.POINTER(rak_tune_space), P,
     C.POINTER(rak_options), C.POINTER(rak_tune_entry), C.c_int32, C.POINTER(C.c_int32))
_sig("rak_server_create", C.c_int, P, C.POINTER(rak_server_options), C.POINTER(P))
_sig("rak_server_submit", C.c_int, P, C.POINTER(rak_csr), C.POINTER(C.c_uint64))
_sig("rak_server_wait", C.c_int, P, C.c_uint64, C.c_double, P, C.POINTER(rak_result))
_sig("rak_server_stats_get", C.c_int, P, C.POINTER(rak_server_stats))
_sig("rak_server_destroy", C.c_int, P)
_sig("rak_lowmem_cuda_noalloc", C.c_int, C.c_int, P, C.POINTER(rak_csr), P, C.POINTER(rak_options), P,
     C.POINTER(rak_result))
NOALLOC_SCRATCH_BYTES = 64 << 20
_sig("rak_gen_rmat", C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64,
     C.c_float, C.c_float, C.c_int, C.POINTER(rak_host_csr))
_sig("rak_gen_sbm", C.c_int, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_uint64, C.c_int,
     C.POINTER(rak_host_csr))
_sig("rak_gen_lattice", C.c_int, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_uint64, C.c_int,
     C.POINTER(rak_host_csr))
_sig("rak_host_csr_free", None, C.POINTER(rak_host_csr))
_sig("rak_gen_rmat_device", C.c_int, P, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64,
     C.c_float, C.c_float, C.c_int32, C.POINTER(rak_csr))
_sig("rak_gen_sbm_device", C.c_int, P, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_uint64, C.c_int32,
     C.POINTER(rak_csr))
_sig("rak_device_csr_free", C.c_int, C.POINTER(rak_csr))
_sig("rak_reference_vertex_order", C.c_int, P, C.POINTER(rak_csr), P)
_sig("rak_batch_reference_vertex_order", C.c_int, P, P, P)
_sig("rak_read_mtx", C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(rak_host_csr))
_sig("rak_device_csr_to_host", C.c_int, C.POINTER(rak_csr), C.POINTER(rak_host_csr))
_sig("rak_csr_validate_host", C.c_int, C.POINTER(rak_csr))
_sig("rak_plan_summary_host", C.c_int, C.POINTER(rak_csr), C.POINTER(rak_options), C.POINTER(C.c_int64),
     C.POINTER(C.c_int64))


class RakError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{STATUS.get(status, status)}: {msg}" if msg else STATUS.get(status, str(status)))


def abi_version() -> int:
    return _lib.rak_abi_version()


def options(**kw) -> rak_options:
    """Defaults of rak_options_default, overridden by keyword (field names of rak_options)."""
    o = rak_options()
    _lib.rak_options_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


def tune_space(**kw) -> rak_tune_space:
    """rak_tune_space_default, overridden by keyword: lane_max / hub_min / hub_chunk / slots take a
    list of values, the other fields a number."""
    sp = rak_tune_space()
    _lib.rak_tune_space_default(C.byref(sp))
    for k, v in kw.items():
        if k in ("lane_max", "hub_min", "hub_chunk", "slots"):
            arr = getattr(sp, k)
            if len(v) > len(arr):
                raise ValueError(f"at most {len(arr)} values for {k}")
            for i, x in enumerate(v):
                arr[i] = int(x)
            setattr(sp, "n_" + k, len(v))
        elif hasattr(sp, k):
            setattr(sp, k, v)
        else:
            raise TypeError(f"unknown tuning field {k}")
    return sp


_OPTION_KEYS = ("lane_max", "hub_min", "hub_chunk", "slots", "label_order")


def _tune_out(best, log, n):
    return ({k: getattr(best, k) for k in _OPTION_KEYS},
            [{f[0]: getattr(log[i], f[0]) for f in rak_tune_entry._fields_} for i in range(min(n, len(log)))])


@dataclass
class Result:
    """RakResult<K> fields plus this library's counters."""
    iterations: int
    time_ms: float
    marking_time_ms: float
    initialization_time_ms: float
    memory_gb: float
    plan_ms: float
    h2d_ms: float
    d2h_ms: float
    peak_device_bytes: int
    traversed_edges: int
    processed_vertices: int
    changed_last: int
    moved_vertices: int
    moved_edges: int
    loop_ms: float
    reserved_f: float
    modularity: float
    marked_edges: int
    dense_iterations: int
    reserved_r: int

    @staticmethod
    def of(r: rak_result) -> "Result":
        return Result(*[getattr(r, f[0]) for f in rak_result._fields_])


class HostGraph:
    """A host CSR: offsets (int32 or int64, n+1), targets (uint32, m), weights (float32 or None)."""

    def __init__(self, offsets, targets, weights=None, truth=None, _owner=None):
        self.offsets = offsets
        self.targets = targets
        self.weights = weights
        self.truth = truth
        self._owner = _owner
        self.n = len(offsets) - 1
        self.m = int(offsets[-1]) if self.n >= 0 else 0

    def csr(self) -> rak_csr:
        return rak_csr(self.n, self.m, 64 if self.offsets.dtype == np.int64 else 32, HOST,
                       self.offsets.ctypes.data, self.targets.ctypes.data if self.m else None,
                       self.weights.ctypes.data if self.weights is not None else None)

    def with_offsets32(self) -> "HostGraph":
        return HostGraph(self.offsets.astype(np.int32), self.targets, self.weights, self.truth, self._owner)

    def degrees(self) -> np.ndarray:
        return np.diff(self.offsets.astype(np.int64))


class _Owned:
    def __init__(self, h: rak_host_csr):
        self.h = h

    def __del__(self):
        if _lib is not None:
            _lib.rak_host_csr_free(C.byref(self.h))


class _View:
    """Array interface over library-owned memory that keeps the owner alive: every numpy array
    (and slice) made from it references this object, so the memory outlives all of them."""

    def __init__(self, ptr, count, dtype, owner):
        self.__array_interface__ = {"data": (ptr, False), "shape": (count,), "typestr": np.dtype(dtype).str,
                                    "version": 3}
        self._owner = owner


def _wrap_host(h: rak_host_csr) -> HostGraph:
    owner = _Owned(h)
    n, m = h.n, h.m

    def arr(ptr, count, dtype):
        if not ptr or count == 0:
            return np.zeros(count, dtype=dtype)
        return np.asarray(_View(ptr, count, dtype, owner))

    off = arr(h.offsets, n + 1, np.int64)
    tgt = arr(h.targets, m, np.uint32)
    wt = arr(h.weights, m, np.float32) if h.weights else None
    truth = arr(h.truth, n, np.uint32) if h.truth else None
    return HostGraph(off, tgt, wt, truth, owner)


def _check(st: int, ctx=None):
    if st != 0:
        msg = _lib.rak_ctx_last_error(ctx).decode() if ctx else ""
        raise RakError(st, msg)


def gen_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=42, w_lo=1.0, w_hi=1.0, threads=0) -> HostGraph:
    h = rak_host_csr()
    _check(_lib.rak_gen_rmat(scale, edge_factor, a, b, c, seed, w_lo, w_hi, threads, C.byref(h)))
    return _wrap_host(h)


def read_mtx(path, weighted=False, symmetrize=True, threads=0) -> HostGraph:
    """rak_read_mtx: a Matrix Market coordinate file as the reference's driver reads it."""
    h = rak_host_csr()
    _check(_lib.rak_read_mtx(str(path).encode(), int(weighted), int(symmetrize), threads, C.byref(h)))
    return _wrap_host(h)


class DeviceGraph:
    """A CSR generated on the device by the library (rak_gen_rmat_device); `csr` is its rak_csr
    (location DEVICE). Freed by close()."""

    def __init__(self, csr: rak_csr):
        self.csr = csr
        self.n, self.m = int(csr.n), int(csr.m)
        self.weighted = bool(csr.weights)

    def to_host(self) -> HostGraph:
        h = rak_host_csr()
        _check(_lib.rak_device_csr_to_host(C.byref(self.csr), C.byref(h)))
        return _wrap_host(h)

    def close(self):
        if _lib is not None and self.csr.offsets:
            _lib.rak_device_csr_free(C.byref(self.csr))

    def __del__(self):
        self.close()


def gen_rmat_device(ctx, scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=42, w_lo=1.0, w_hi=1.0,
                    offset_bits=64) -> DeviceGraph:
    """rak_gen_rmat_device: the graph gen_rmat builds, built on ctx's device."""
    c_ = rak_csr()
    _check(_lib.rak_gen_rmat_device(ctx.handle, scale, edge_factor, a, b, c, seed, w_lo, w_hi, offset_bits,
                                    C.byref(c_)), ctx.handle)
    return DeviceGraph(c_)


def gen_sbm_device(ctx, n, k, avg_degree=16.0, in_out_ratio=20.0, seed=42, offset_bits=64) -> DeviceGraph:
    """rak_gen_sbm_device: the graph gen_sbm builds, built on ctx's device."""
    c_ = rak_csr()
    _check(_lib.rak_gen_sbm_device(ctx.handle, n, k, avg_degree, in_out_ratio, seed, offset_bits, C.byref(c_)),
           ctx.handle)
    return DeviceGraph(c_)


def gen_sbm(n, k, avg_degree=16.0, in_out_ratio=20.0, seed=42, threads=0) -> HostGraph:
    h = rak_host_csr()
    _check(_lib.rak_gen_sbm(n, k, avg_degree, in_out_ratio, seed, threads, C.byref(h)))
    return _wrap_host(h)


def gen_lattice(width, height, p_delete=0.05, shortcut_frac=0.01, seed=42, threads=0) -> HostGraph:
    h = rak_host_csr()
    _check(_lib.rak_gen_lattice(width, height, p_delete, shortcut_frac, seed, threads, C.byref(h)))
    return _wrap_host(h)


def validate_host(g: HostGraph) -> int:
    c = g.csr()
    return _lib.rak_csr_validate_host(C.byref(c))


def plan_summary(g: HostGraph, **opts):
    c = g.csr()
    counts = (C.c_int64 * 8)()
    chunks = C.c_int64(0)
    o = options(**opts)
    _check(_lib.rak_plan_summary_host(C.byref(c), C.byref(o), counts, C.byref(chunks)))
    return list(counts), chunks.value


def _ptr(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


def device_csr(offsets, targets, weights=None) -> rak_csr:
    """rak_csr over torch CUDA tensors (offsets int32/int64, targets int32 holding uint32 ids)."""
    import torch
    n = offsets.numel() - 1
    return rak_csr(n, targets.numel(), 64 if offsets.dtype == torch.int64 else 32, DEVICE,
                   offsets.data_ptr(), _ptr(targets) if targets.numel() else None, _ptr(weights))


class Context:
    """A device context (rak_ctx): one device, one stream."""

    def __init__(self, device: int = 0):
        self._c = P()
        _check(_lib.rak_ctx_create(device, C.byref(self._c)))

    def close(self):
        if self._c and _lib is not None:
            _lib.rak_ctx_destroy(self._c)
            self._c = P()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._c

    def set_stream(self, stream_ptr: Optional[int]):
        _check(_lib.rak_ctx_set_stream(self._c, stream_ptr), self._c)

    def set_memory_keep(self, nbytes: int):
        """rak_ctx_set_memory_keep: device bytes kept mapped between lowmem() calls."""
        _check(_lib.rak_ctx_set_memory_keep(self._c, int(nbytes)), self._c)

    def last_error(self) -> str:
        return _lib.rak_ctx_last_error(self._c).decode()

    def lowmem(self, g: HostGraph, q: Optional[np.ndarray] = None, flags: Optional[np.ndarray] = None,
               **opts):
        """rakLowmemStaticCuda<slots>(x, o) on a host graph: (membership, Result)."""
        o = options(**opts)
        if flags is not None:
            flags = np.ascontiguousarray(flags, dtype=np.uint8)
            o.initial_flags = flags.ctypes.data
        c = g.csr()
        out = np.empty(g.n, dtype=np.uint32)
        r = rak_result()
        qp = None
        if q is not None:
            q = np.ascontiguousarray(q, dtype=np.uint32)
            qp = q.ctypes.data
        _check(_lib.rak_lowmem_cuda(self._c, C.byref(c), qp, C.byref(o), out.ctypes.data, C.byref(r)), self._c)
        return out, Result.of(r)

    def reference_vertex_order(self, csr: rak_csr, ks):
        """rak_reference_vertex_order into the torch CUDA tensor ks (n entries)."""
        _check(_lib.rak_reference_vertex_order(self._c, C.byref(csr), ks.data_ptr()), self._c)

    def lowmem_device(self, csr: rak_csr, membership, q=None, **opts):
        """The same on a device-located csr; membership (and q) are torch CUDA tensors."""
        o = options(**opts)
        r = rak_result()
        _check(_lib.rak_lowmem_cuda(self._c, C.byref(csr), _ptr(q), C.byref(o), membership.data_ptr(),
                                    C.byref(r)), self._c)
        return Result.of(r)

    def modularity(self, csr_or_graph, membership) -> float:
        """FP64 modularity on the device (rak_modularity_f64)."""
        if isinstance(csr_or_graph, HostGraph):
            c = csr_or_graph.csr()
            membership = np.ascontiguousarray(membership, dtype=np.uint32)
            mp = membership.ctypes.data
        else:
            c = csr_or_graph
            mp = membership.data_ptr()
        q = C.c_double(math.nan)
        _check(_lib.rak_modularity_f64(self._c, C.byref(c), mp, C.byref(q)), self._c)
        return q.value


def lowmem_noalloc(device: int, stream_ptr: Optional[int], csr: rak_csr, membership, q=None, **opts) -> Result:
    """rak_lowmem_cuda_noalloc: a run on a device-located csr that allocates no device memory
    (working buffers come from the library's fixed device array of NOALLOC_SCRATCH_BYTES)."""
    o = options(**opts)
    r = rak_result()
    st = _lib.rak_lowmem_cuda_noalloc(device, stream_ptr, C.byref(csr), _ptr(q), C.byref(o), membership.data_ptr(),
                                       C.byref(r))
    if st != 0:
        raise RakError(st, f"needs {r.peak_device_bytes} bytes of scratch" if st == 3 else "")
    return Result.of(r)


class ResidentGraph:
    """A device-resident graph with its plan (rak_graph)."""

    def __init__(self, ctx: Context, csr_or_graph, **opts):
        self.ctx = ctx
        self._keep = csr_or_graph
        c = csr_or_graph.csr() if isinstance(csr_or_graph, HostGraph) else csr_or_graph
        self.n = c.n
        self._g = P()
        o = options(**opts)
        _check(_lib.rak_graph_create(ctx.handle, C.byref(c), C.byref(o), C.byref(self._g)), ctx.handle)

    def close(self):
        if self._g and _lib is not None:
            _lib.rak_graph_destroy(self._g)
            self._g = P()

    def __del__(self):
        self.close()

    def device_bytes(self) -> int:
        return _lib.rak_graph_device_bytes(self._g)

    def autotune(self, membership, space=None, **base_opts):
        """rak_graph_autotune: returns ({lane_max, hub_min, hub_chunk, slots, label_order} of the best
        run, the list of candidates run)."""
        o, best = options(**base_opts), rak_options()
        log, n = (rak_tune_entry * 64)(), C.c_int32(0)
        sp = space if space is not None else tune_space()
        _check(_lib.rak_graph_autotune(self.ctx.handle, self._g, C.byref(o), C.byref(sp), membership.data_ptr(),
                                       C.byref(best), log, 64, C.byref(n)), self.ctx.handle)
        return _tune_out(best, log, n.value)

    def run(self, membership, q=None, **opts) -> Result:
        o = options(**opts)
        r = rak_result()
        _check(_lib.rak_graph_run(self.ctx.handle, self._g, _ptr(q), C.byref(o), membership.data_ptr(),
                                  C.byref(r)), self.ctx.handle)
        return Result.of(r)

    def step(self, iteration, vcom_prev, aff_prev, vcom_next, aff_next, **opts) -> int:
        o = options(**opts)
        ch = C.c_uint64(0)
        _check(_lib.rak_graph_step(self.ctx.handle, self._g, C.byref(o), iteration, vcom_prev.data_ptr(),
                                   aff_prev.data_ptr(), vcom_next.data_ptr(), aff_next.data_ptr(),
                                   C.byref(ch)), self.ctx.handle)
        return ch.value


class HostBatch:
    """Graphs concatenated into one CSR: graph g owns vertices [graph_offsets[g], graph_offsets[g+1]),
    offsets (int64) index the concatenated targets (ids local to each graph) and weights."""

    def __init__(self, graph_offsets, offsets, targets, weights=None, truths=None):
        self.graph_offsets = np.ascontiguousarray(graph_offsets, dtype=np.int64)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        self.targets = np.ascontiguousarray(targets, dtype=np.uint32)
        self.weights = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
        self.truths = truths
        self.graphs = len(self.graph_offsets) - 1
        self.n = int(self.graph_offsets[-1])
        self.m = int(self.offsets[-1])

    @staticmethod
    def concat(graphs, weighted=None) -> "HostBatch":
        """Packs HostGraphs into a batch (weights kept if every graph has them, unless weighted=False)."""
        if weighted is None:
            weighted = all(g.weights is not None for g in graphs) and len(graphs) > 0
        go = np.zeros(len(graphs) + 1, np.int64)
        go[1:] = np.cumsum([g.n for g in graphs])
        eo = np.zeros(len(graphs) + 1, np.int64)
        eo[1:] = np.cumsum([g.m for g in graphs])
        off = np.empty(int(go[-1]) + 1, np.int64)
        off[-1] = eo[-1]
        for i, g in enumerate(graphs):
            off[go[i]:go[i + 1]] = g.offsets[:-1].astype(np.int64) + eo[i]
        tgt = np.concatenate([g.targets for g in graphs]) if graphs else np.zeros(0, np.uint32)
        wt = np.concatenate([g.weights for g in graphs]) if weighted else None
        truths = [g.truth for g in graphs] if all(g.truth is not None for g in graphs) and graphs else None
        return HostBatch(go, off, tgt, wt, truths)

    def graph(self, i) -> HostGraph:
        a, b = int(self.graph_offsets[i]), int(self.graph_offsets[i + 1])
        e0, e1 = int(self.offsets[a]), int(self.offsets[b])
        return HostGraph(self.offsets[a:b + 1] - e0, self.targets[e0:e1],
                         None if self.weights is None else self.weights[e0:e1])

    def csr(self) -> rak_batch_csr:
        return rak_batch_csr(self.graphs, self.n, self.m, HOST, 0, self.graph_offsets.ctypes.data,
                             self.offsets.ctypes.data, self.targets.ctypes.data if self.m else None,
                             self.weights.ctypes.data if self.weights is not None else None)


class DeviceBatch:
    """Graphs concatenated into one CSR in device memory (torch CUDA tensors): graph_offsets and
    offsets int64, targets int32 (ids local to each graph), weights float32 or None. Built from
    device graphs by concat without a host round trip of the edges."""

    def __init__(self, graph_offsets, offsets, targets, weights=None):
        self.graph_offsets, self.offsets, self.targets, self.weights = graph_offsets, offsets, targets, weights
        self.graphs = int(graph_offsets.numel()) - 1
        self.n = int(graph_offsets[-1].item())
        self.m = int(offsets[-1].item())
        self.graph_offsets_host = graph_offsets.cpu().numpy()

    @staticmethod
    def concat(graphs) -> "DeviceBatch":
        """Packs device graphs (rak_csr of location DEVICE, unit weights) into one batch."""
        import torch
        go = np.zeros(len(graphs) + 1, np.int64)
        go[1:] = np.cumsum([int(g.n) for g in graphs])
        eo = np.zeros(len(graphs) + 1, np.int64)
        eo[1:] = np.cumsum([int(g.m) for g in graphs])
        off = torch.empty(int(go[-1]) + 1, dtype=torch.int64, device="cuda")
        tgt = torch.empty(max(int(eo[-1]), 1), dtype=torch.int32, device="cuda")
        for i, g in enumerate(graphs):
            n, m = int(g.n), int(g.m)
            off_i = _device_view(g.offsets, n + 1, torch.int64 if g.offset_bits == 64 else torch.int32)
            off[go[i]:go[i + 1]] = off_i[:n].to(torch.int64) + int(eo[i])
            if m:
                tgt[eo[i]:eo[i + 1]] = _device_view(g.targets, m, torch.int32)
        off[-1] = int(eo[-1])
        return DeviceBatch(torch.from_numpy(go).cuda(), off, tgt[:int(eo[-1])])

    def csr(self) -> rak_batch_csr:
        return rak_batch_csr(self.graphs, self.n, self.m, DEVICE, 0, self.graph_offsets.data_ptr(),
                             self.offsets.data_ptr(), self.targets.data_ptr() if self.m else None,
                             self.weights.data_ptr() if self.weights is not None else None)


def _device_view(ptr, count, dtype):
    """A torch CUDA tensor over `count` elements of device memory at ptr (not owned)."""
    import torch
    if count == 0:
        return torch.empty(0, dtype=dtype, device="cuda")
    esz = torch.empty(0, dtype=dtype).element_size()
    return _ViewHolder.wrap(ptr, count * esz).view(dtype)[:count]


class _ViewHolder:
    """Wraps raw device memory as a uint8 torch tensor through __cuda_array_interface__."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3, "strides": None}

    @staticmethod
    def wrap(ptr, nbytes):
        import torch
        return torch.as_tensor(_ViewHolder(ptr, nbytes), device="cuda")


class Batch:
    """A device-resident batch of graphs (rak_batch): one persistent launch runs them all."""

    def __init__(self, ctx: Context, host_batch, **opts):
        """host_batch: a HostBatch, or a DeviceBatch (bound in place, not copied)."""
        self.ctx = ctx
        self._keep = host_batch
        self.graphs = host_batch.graphs
        self.n = host_batch.n
        self._b = P()
        c = host_batch.csr()
        o = options(**opts)
        _check(_lib.rak_batch_create(ctx.handle, C.byref(c), C.byref(o), C.byref(self._b)), ctx.handle)

    def close(self):
        if self._b and _lib is not None:
            _lib.rak_batch_destroy(self._b)
            self._b = P()

    def __del__(self):
        self.close()

    def autotune(self, membership, space=None, **base_opts):
        """rak_batch_autotune (quality: mean modularity over the graphs); see ResidentGraph.autotune."""
        o, best = options(**base_opts), rak_options()
        log, n = (rak_tune_entry * 64)(), C.c_int32(0)
        sp = space if space is not None else tune_space()
        _check(_lib.rak_batch_autotune(self.ctx.handle, self._b, self.graphs, C.byref(o), C.byref(sp),
                                       membership.data_ptr(), C.byref(best), log, 64, C.byref(n)), self.ctx.handle)
        return _tune_out(best, log, n.value)

    def reference_vertex_order(self, ks):
        """rak_batch_reference_vertex_order into the torch CUDA tensor ks (n entries): each graph's
        local vertex ids in its reference order."""
        _check(_lib.rak_batch_reference_vertex_order(self.ctx.handle, self._b, ks.data_ptr()), self.ctx.handle)

    def launch(self, membership, q=None, **opts):
        o = options(**opts)
        _check(_lib.rak_batch_launch(self.ctx.handle, self._b, _ptr(q), C.byref(o), membership.data_ptr()),
               self.ctx.handle)

    def results(self):
        it = np.zeros(self.graphs, np.int32)
        r = rak_result()
        _check(_lib.rak_batch_results(self.ctx.handle, self._b, it.ctypes.data if self.graphs else None,
                                      C.byref(r)), self.ctx.handle)
        return it, Result.of(r)

    def capture(self, membership, q=None, **opts):
        o = options(**opts)
        _check(_lib.rak_batch_capture(self.ctx.handle, self._b, _ptr(q), C.byref(o), membership.data_ptr()),
               self.ctx.handle)

    def replay(self):
        _check(_lib.rak_batch_replay(self.ctx.handle, self._b), self.ctx.handle)

    def modularity(self, membership) -> np.ndarray:
        q = np.zeros(max(self.graphs, 1), np.float64)
        _check(_lib.rak_batch_modularity_f64(self.ctx.handle, self._b, membership.data_ptr(), q.ctypes.data),
               self.ctx.handle)
        return q[:self.graphs]


class _DeviceRequest:
    def __init__(self, n, keep):
        self.n, self.keep = n, keep


class Server:
    """Continuous-batching request loop (rak_server_*). submit() takes host graphs and
    submit_device() device-located graphs (a rak_csr from device_csr()); either must stay alive and
    unchanged until wait() returns for it (the object keeps a reference to what it is given)."""

    def __init__(self, ctx: Context, budget_bytes=16 << 30, max_graphs_per_launch=256, slots=2,
                 queue_capacity=65536, **run_opts):
        o = rak_server_options()
        _lib.rak_server_options_default(C.byref(o))
        o.budget_bytes, o.max_graphs_per_launch, o.slots, o.queue_capacity = \
            budget_bytes, max_graphs_per_launch, slots, queue_capacity
        o.run = options(**run_opts)
        self.ctx = ctx
        self._s = P()
        self._keep = {}
        _check(_lib.rak_server_create(ctx.handle, C.byref(o), C.byref(self._s)), ctx.handle)

    def submit(self, g: HostGraph) -> int:
        c = g.csr()
        t = C.c_uint64(0)
        _check(_lib.rak_server_submit(self._s, C.byref(c), C.byref(t)))
        self._keep[t.value] = g
        return t.value

    def submit_device(self, csr, keep=None) -> int:
        """Queues a device-located graph (rak_csr with location DEVICE, on the server's device);
        `keep` is held until the request completes (the tensors behind the pointers)."""
        t = C.c_uint64(0)
        _check(_lib.rak_server_submit(self._s, C.byref(csr), C.byref(t)))
        self._keep[t.value] = _DeviceRequest(int(csr.n), keep)
        return t.value

    def wait(self, ticket: int, timeout=120.0):
        g = self._keep.get(ticket)
        out = np.empty(g.n if g is not None else 0, dtype=np.uint32)
        r = rak_result()
        st = _lib.rak_server_wait(self._s, ticket, timeout, out.ctypes.data if len(out) else None, C.byref(r))
        if st != 5:                      # not a timeout: the ticket is released
            self._keep.pop(ticket, None)
        if st != 0:
            raise RakError(st)
        return out, Result.of(r)

    def stats(self) -> dict:
        st = rak_server_stats()
        _check(_lib.rak_server_stats_get(self._s, C.byref(st)))
        return {f[0]: getattr(st, f[0]) for f in rak_server_stats._fields_}

    def close(self):
        if self._s and _lib is not None:
            _lib.rak_server_destroy(self._s)
            self._s = P()
        self._keep = {}

    def __del__(self):
        self.close()


def write_rakcsr(path: str, g: HostGraph):
    """Binary CSR file: b"RAKCSR01", int64 n, int64 m, int32 has_weights, int64 offsets[n+1],
    uint32 targets[m], float32 weights[m] (if present)."""
    with open(path, "wb") as f:
        f.write(b"RAKCSR01")
        f.write(np.array([g.n, g.m], dtype=np.int64).tobytes())
        f.write(np.array([1 if g.weights is not None else 0], dtype=np.int32).tobytes())
        f.write(g.offsets.astype(np.int64).tobytes())
        f.write(g.targets.astype(np.uint32).tobytes())
        if g.weights is not None:
            f.write(g.weights.astype(np.float32).tobytes())
