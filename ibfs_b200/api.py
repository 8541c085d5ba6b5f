"""Python mirror of the C ABI in include/ibfs.h (ctypes; no torch types).

Names follow the reference's host interface where one exists:
``graph_reader`` (graph_reader.cuh:63-119), ``GroupBy`` (GroupBy.cuh:6-115),
``read_src_v`` (graph.cuh:99-133), ``report`` (validate.h:59-76).  The
product path is the CUDA library ``libibfs.so``; when it cannot be loaded
every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_PKG, "libibfs.so")

IBFS_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "IO", 2: "FORMAT", 3: "RANGE", 4: "OOM", 5: "CUDA", 6: "TIMEOUT",
    7: "INVALID_ARG", 8: "UNSUPPORTED", 9: "BUSY", 10: "NOT_FOUND",
}
MODE_PLAIN, MODE_PERSISTENT, MODE_DEVICE_LOOP, MODE_AUTO = 0, 1, 2, 3
LAYOUT_SOURCE_MAJOR, LAYOUT_VERTEX_MAJOR = 0, 1
OUT_DEVICE = 1


class IbfsError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        msg = _lib().ibfs_strerror(status).decode() if _LIB is not None else self.name
        super().__init__(f"{what}: IBFS_ERR_{self.name} ({msg})" if what else msg)


class Opts(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("concurrent", C.c_int32), ("switch_level", C.c_int32),
        ("alpha", C.c_float), ("beta", C.c_float), ("sml_shed", C.c_int32),
        ("lrg_shed", C.c_int32), ("mode", C.c_int32), ("groupby", C.c_int32),
        ("depth_bytes", C.c_int32), ("groups", C.c_int32), ("threads", C.c_int32),
        ("ctas_per_sm", C.c_int32), ("use_graph", C.c_int32), ("timeout_ms", C.c_int32),
        ("max_levels", C.c_int32), ("debug_withhold", C.c_int32), ("occupancy", C.c_int32),
        ("bu_filter", C.c_int32), ("bu_thread_max", C.c_int32), ("td_stage", C.c_int32),
        ("sparse_push", C.c_int32), ("reserved", C.c_int32 * 2),
    ]


class LevelRec(C.Structure):
    _fields_ = [("batch", C.c_int32), ("level", C.c_int32), ("dir", C.c_int32), ("pad", C.c_int32),
                ("frontier", C.c_int64), ("frontier_edges", C.c_int64), ("expand_ns", C.c_int64),
                ("inspect_ns", C.c_int64)]


class Stats(C.Structure):
    _fields_ = [
        ("n_sources", C.c_int64), ("n_batches", C.c_int64), ("max_level", C.c_int32),
        ("depth_bytes", C.c_int32), ("width", C.c_int32), ("groups", C.c_int32),
        ("levels_total", C.c_int64), ("td_levels", C.c_int64), ("bu_levels", C.c_int64),
        ("traversed_edges", C.c_int64), ("gpu_launches", C.c_int64), ("device_ms", C.c_double),
        ("total_ms", C.c_double), ("levels", C.POINTER(LevelRec)), ("levels_cap", C.c_int32),
        ("levels_len", C.c_int32),
    ]


class ServerOpts(C.Structure):
    _fields_ = [("run", Opts), ("arena_bytes", C.c_int64), ("max_waiting", C.c_int32),
                ("round_batches", C.c_int32), ("max_wait_us", C.c_int32), ("groupby", C.c_int32),
                ("reserved", C.c_int32 * 6)]


class QueryInfo(C.Structure):
    _fields_ = [("n_sources", C.c_int64), ("latency_ms", C.c_double), ("queue_ms", C.c_double),
                ("status", C.c_int32), ("depth_bytes", C.c_int32), ("delivered_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("refused", C.c_int64),
                ("rounds", C.c_int64), ("sources", C.c_int64), ("traversed_edges", C.c_int64),
                ("busy_ms", C.c_double), ("wall_ms", C.c_double), ("arena_rows", C.c_int64),
                ("arena_rows_used", C.c_int64), ("launches", C.c_int64)]


_LIB = None

# (name, restype, argtypes) for every entry point of include/ibfs.h
_P = C.c_void_p
_I64P = C.POINTER(C.c_int64)
_I32P = C.POINTER(C.c_int32)
_SIGS = [
    ("ibfs_strerror", C.c_char_p, [C.c_int]),
    ("ibfs_version", C.c_char_p, []),
    ("ibfs_graph_open", C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(_P)]),
    ("ibfs_graph_from_csr", C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_int, C.POINTER(_P)]),
    ("ibfs_csr_read", C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_P), C.POINTER(_P), _I64P, _I64P]),
    ("ibfs_graph_info", C.c_int, [_P, _I64P, _I64P, _I64P]),
    ("ibfs_graph_device_csr", C.c_int, [_P, C.POINTER(_P), C.POINTER(_P)]),
    ("ibfs_graph_vertex_order", C.c_int, [_P, C.POINTER(_P)]),
    ("ibfs_graph_close", C.c_int, [_P]),
    ("ibfs_groupby", C.c_int, [_P, _P, C.c_int64, _P]),
    ("ibfs_groupby_device", C.c_int, [_P, _P, C.c_int64, _P, _P]),
    ("ibfs_groupby_maxhub", C.c_int, [_P, _P, C.c_int64, _P]),
    ("ibfs_convert_text", C.c_int, [C.c_char_p, C.c_int32, C.c_int64, C.c_int32, C.c_char_p,
                                    C.c_char_p, C.c_int32, C.POINTER(C.c_int64),
                                    C.POINTER(C.c_int64)]),
    ("ibfs_groupby_csr", C.c_int, [_P, _P, C.c_int64, _P, C.c_int64, _P]),
    ("ibfs_groupby_csr_maxhub", C.c_int, [_P, _P, C.c_int64, _P, C.c_int64, _P]),
    ("ibfs_read_sources", C.c_int, [C.c_char_p, _P, C.c_int64, _I64P]),
    ("ibfs_write_sources", C.c_int, [C.c_char_p, _P, C.c_int64]),
    ("ibfs_opts_default", None, [C.POINTER(Opts)]),
    ("ibfs_run", C.c_int, [_P, _P, C.c_int64, C.POINTER(Opts), _P, C.c_int32, C.c_uint32,
                           C.POINTER(Stats)]),
    ("ibfs_set_stream", C.c_int, [_P, _P]),
    ("ibfs_teps", C.c_int, [_P, _P, C.c_int64, C.c_int32, _I64P]),
    ("ibfs_autotune", C.c_int, [_P, _P, C.c_int64, C.POINTER(Opts), C.c_int32, C.POINTER(Opts),
                                C.POINTER(C.c_double), C.c_char_p, C.c_int32]),
    ("ibfs_bytes_alg", C.c_int, [_P, _P, C.c_int64, C.c_int32, C.c_int32, _I64P]),
    ("ibfs_run_static_scratch", C.c_int, [_P, _P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int32,
                                          _P, _P, _I64P]),
    ("ibfs_server_opts_default", None, [C.POINTER(ServerOpts)]),
    ("ibfs_server_create", C.c_int, [_P, C.POINTER(ServerOpts), C.POINTER(_P)]),
    ("ibfs_server_submit", C.c_int, [_P, _P, C.c_int64, C.POINTER(C.c_uint64)]),
    ("ibfs_server_poll", C.c_int, [_P, C.c_uint64, _P, C.c_uint32, C.POINTER(C.c_int32),
                                   C.POINTER(QueryInfo)]),
    ("ibfs_server_wait", C.c_int, [_P, C.c_uint64, C.c_int32, _P, C.c_uint32,
                                   C.POINTER(QueryInfo)]),
    ("ibfs_server_stats_get", C.c_int, [_P, C.POINTER(ServerStats)]),
    ("ibfs_server_arena_rows", C.c_int64, [C.c_int64, C.c_int64, C.c_int32]),
    ("ibfs_server_destroy", C.c_int, [_P]),
    ("ibfs_gen_rmat", C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                C.c_uint64, C.POINTER(_P), C.POINTER(_P), _I64P, _I64P]),
    ("ibfs_gen_grid", C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_uint64,
                                C.POINTER(_P), C.POINTER(_P), _I64P, _I64P]),
    ("ibfs_gen_chung_lu", C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_uint64,
                                    C.POINTER(_P), C.POINTER(_P), _I64P, _I64P]),
    ("ibfs_csr_from_edges", C.c_int, [_P, _P, C.c_int64, C.c_int64, C.POINTER(_P), C.POINTER(_P),
                                      _I64P]),
    ("ibfs_write_csr", C.c_int, [C.c_char_p, C.c_char_p, _P, _P, C.c_int64]),
    ("ibfs_sample_sources", C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_uint64, C.c_int32, _P]),
    ("ibfs_free", None, [_P]),
]


def exported_names() -> list[str]:
    return [s[0] for s in _SIGS]


def _lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"libibfs.so is not built ({_LIB_PATH}); run __graft_entry__.build()")
        lib = C.CDLL(_LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def lib_path() -> str:
    return _LIB_PATH


def _check(st: int, what: str) -> None:
    if st != IBFS_OK:
        raise IbfsError(st, what)


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def default_opts(**kw) -> Opts:
    o = Opts()
    _lib().ibfs_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


def _take_csr(bp: C.c_void_p, cp: C.c_void_p, V: int, E: int) -> tuple[np.ndarray, np.ndarray]:
    L = _lib()
    beg = np.ctypeslib.as_array(C.cast(bp, C.POINTER(C.c_int64)), shape=(V + 1,)).copy()
    col = (np.ctypeslib.as_array(C.cast(cp, C.POINTER(C.c_int32)), shape=(E,)).copy()
           if E > 0 else np.zeros(0, np.int32))
    L.ibfs_free(bp)
    L.ibfs_free(cp)
    return beg, col


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, seed: int = 1) -> tuple[np.ndarray, np.ndarray]:
    """Seeded undirected R-MAT graph (symmetrised, no loops, no duplicates)."""
    bp, cp = C.c_void_p(), C.c_void_p()
    V, E = C.c_int64(), C.c_int64()
    _check(_lib().ibfs_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(bp), C.byref(cp),
                                C.byref(V), C.byref(E)), "ibfs_gen_rmat")
    return _take_csr(bp, cp, V.value, E.value)


def gen_grid(rows: int, cols: int, delete_frac: float = 0.05, shortcut_frac: float = 0.001,
             seed: int = 4) -> tuple[np.ndarray, np.ndarray]:
    bp, cp = C.c_void_p(), C.c_void_p()
    V, E = C.c_int64(), C.c_int64()
    _check(_lib().ibfs_gen_grid(rows, cols, delete_frac, shortcut_frac, seed, C.byref(bp),
                                C.byref(cp), C.byref(V), C.byref(E)), "ibfs_gen_grid")
    return _take_csr(bp, cp, V.value, E.value)


def gen_chung_lu(n: int, m: int, gamma: float = 2.1, max_degree: float = 33000.0,
                 seed: int = 5) -> tuple[np.ndarray, np.ndarray]:
    bp, cp = C.c_void_p(), C.c_void_p()
    V, E = C.c_int64(), C.c_int64()
    _check(_lib().ibfs_gen_chung_lu(n, m, gamma, max_degree, seed, C.byref(bp), C.byref(cp),
                                    C.byref(V), C.byref(E)), "ibfs_gen_chung_lu")
    return _take_csr(bp, cp, V.value, E.value)


def csr_from_edges(src: np.ndarray, dst: np.ndarray, V: int) -> tuple[np.ndarray, np.ndarray]:
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    bp, cp = C.c_void_p(), C.c_void_p()
    E = C.c_int64()
    _check(_lib().ibfs_csr_from_edges(_ptr(src), _ptr(dst), len(src), V, C.byref(bp), C.byref(cp),
                                      C.byref(E)), "ibfs_csr_from_edges")
    return _take_csr(bp, cp, V, E.value)


def read_csr(beg_path: str, csr_path: str) -> tuple[np.ndarray, np.ndarray]:
    """Host read of the binary CSR pair (graph_reader, graph_reader.cuh:63-119)."""
    bp, cp = C.c_void_p(), C.c_void_p()
    V, E = C.c_int64(), C.c_int64()
    _check(_lib().ibfs_csr_read(beg_path.encode(), csr_path.encode(), C.byref(bp), C.byref(cp),
                                C.byref(V), C.byref(E)), "ibfs_csr_read")
    return _take_csr(bp, cp, V.value, E.value)


def write_csr(beg_path: str, csr_path: str, beg: np.ndarray, col: np.ndarray) -> None:
    beg = np.ascontiguousarray(beg, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    _check(_lib().ibfs_write_csr(beg_path.encode(), csr_path.encode(), _ptr(beg), _ptr(col),
                                 len(beg) - 1), "ibfs_write_csr")


def sample_sources(beg: np.ndarray, col: np.ndarray, n: int, seed: int,
                   giant_component: bool = False) -> np.ndarray:
    beg = np.ascontiguousarray(beg, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    out = np.zeros(n, np.int32)
    _check(_lib().ibfs_sample_sources(_ptr(beg), _ptr(col), len(beg) - 1, n, seed,
                                      0 if giant_component else -1, _ptr(out)),
           "ibfs_sample_sources")
    return out


def groupby_csr(beg: np.ndarray, col: np.ndarray, src: np.ndarray) -> np.ndarray:
    """GroupBy (GroupBy.cuh:19-84) on host CSR arrays."""
    beg = np.ascontiguousarray(beg, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    src = np.ascontiguousarray(src, np.int32)
    out = np.zeros_like(src)
    _check(_lib().ibfs_groupby_csr(_ptr(beg), _ptr(col), len(beg) - 1, _ptr(src), len(src),
                                   _ptr(out)), "ibfs_groupby_csr")
    return out


def convert_text(text_path: str, reverse: bool = True, skip_lines: int = 0, clean: bool = False,
                 out_prefix: str | None = None, device: int = 0) -> tuple[str, str, int, int]:
    """Edge-list text -> <prefix>_beg_pos.bin / <prefix>_csr.bin on the GPU
    (tuple_text_to_bin.cpp:56-310; prefix defaults to the input path).
    Returns (beg_path, csr_path, V, E)."""
    pre = out_prefix or text_path
    bp, cp = pre + "_beg_pos.bin", pre + "_csr.bin"
    V, E = C.c_int64(), C.c_int64()
    _check(_lib().ibfs_convert_text(text_path.encode(), 1 if reverse else 0, skip_lines,
                                    1 if clean else 0, bp.encode(), cp.encode(), device,
                                    C.byref(V), C.byref(E)), "ibfs_convert_text")
    return bp, cp, V.value, E.value


def groupby_csr_maxhub(beg: np.ndarray, col: np.ndarray, src: np.ndarray) -> np.ndarray:
    """The largest-hub GroupBy variant (groupby = 3) on host CSR arrays."""
    beg = np.ascontiguousarray(beg, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    src = np.ascontiguousarray(src, np.int32)
    out = np.zeros_like(src)
    _check(_lib().ibfs_groupby_csr_maxhub(_ptr(beg), _ptr(col), len(beg) - 1, _ptr(src),
                                          len(src), _ptr(out)), "ibfs_groupby_csr_maxhub")
    return out


def read_src_v(path: str) -> np.ndarray:
    """read_src_v (graph.cuh:99-133): one decimal vertex id per line."""
    n = C.c_int64()
    _check(_lib().ibfs_read_sources(path.encode(), None, 0, C.byref(n)), "ibfs_read_sources")
    out = np.zeros(n.value, np.int32)
    _check(_lib().ibfs_read_sources(path.encode(), _ptr(out), n.value, C.byref(n)),
           "ibfs_read_sources")
    return out


def write_src_v(path: str, ids: np.ndarray) -> None:
    ids = np.ascontiguousarray(ids, np.int32)
    _check(_lib().ibfs_write_sources(path.encode(), _ptr(ids), len(ids)), "ibfs_write_sources")


@dataclass
class RunResult:
    depth: np.ndarray | None
    stats: dict
    levels: list = field(default_factory=list)


class Graph:
    """Resident CSR on one GPU (ibfs_graph handle)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle
        V, E, md = C.c_int64(), C.c_int64(), C.c_int64()
        _check(_lib().ibfs_graph_info(self._h, C.byref(V), C.byref(E), C.byref(md)), "info")
        self.V, self.E, self.max_degree = V.value, E.value, md.value

    @classmethod
    def open(cls, beg_path: str, csr_path: str, device: int = 0) -> "Graph":
        h = C.c_void_p()
        _check(_lib().ibfs_graph_open(beg_path.encode(), csr_path.encode(), device, C.byref(h)),
               "ibfs_graph_open")
        return cls(h)

    @classmethod
    def from_csr(cls, beg: np.ndarray, col: np.ndarray, device: int = 0) -> "Graph":
        beg = np.ascontiguousarray(beg, np.int64)
        col = np.ascontiguousarray(col, np.int32)
        h = C.c_void_p()
        _check(_lib().ibfs_graph_from_csr(_ptr(beg), _ptr(col), len(beg) - 1, len(col), device,
                                          C.byref(h)), "ibfs_graph_from_csr")
        return cls(h)

    def close(self) -> None:
        if self._h:
            _lib().ibfs_graph_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def device_csr(self) -> tuple[int, int]:
        b, c = C.c_void_p(), C.c_void_p()
        _check(_lib().ibfs_graph_device_csr(self._h, C.byref(b), C.byref(c)), "device_csr")
        return b.value, c.value

    def vertex_order(self) -> int:
        """Device pointer of new_of_old[V] (caller id -> internal id)."""
        m = C.c_void_p()
        _check(_lib().ibfs_graph_vertex_order(self._h, C.byref(m)), "ibfs_graph_vertex_order")
        return m.value

    def set_stream(self, stream_ptr: int | None) -> None:
        _check(_lib().ibfs_set_stream(self._h, C.c_void_p(stream_ptr or 0)), "ibfs_set_stream")

    def groupby(self, src: np.ndarray) -> np.ndarray:
        src = np.ascontiguousarray(src, np.int32)
        out = np.zeros_like(src)
        _check(_lib().ibfs_groupby(self._h, _ptr(src), len(src), _ptr(out)), "ibfs_groupby")
        return out

    def groupby_maxhub(self, src: np.ndarray) -> np.ndarray:
        """The batch order of groupby = 3 (sources keyed by their highest-degree hub)."""
        src = np.ascontiguousarray(src, np.int32)
        out = np.zeros_like(src)
        _check(_lib().ibfs_groupby_maxhub(self._h, _ptr(src), len(src), _ptr(out)),
               "ibfs_groupby_maxhub")
        return out

    def groupby_device(self, src_ptr: int, n: int, out_ptr: int, pos_ptr: int | None = None):
        """GroupBy of n device int32 sources into out_ptr (and their input
        positions into pos_ptr), on the graph's stream."""
        _check(_lib().ibfs_groupby_device(self._h, C.c_void_p(src_ptr), n, C.c_void_p(out_ptr),
                                          C.c_void_p(pos_ptr) if pos_ptr else None),
               "ibfs_groupby_device")

    def teps(self, depth: np.ndarray) -> int:
        depth = np.ascontiguousarray(depth)
        e = C.c_int64()
        _check(_lib().ibfs_teps(self._h, _ptr(depth), depth.shape[0], depth.dtype.itemsize,
                                C.byref(e)), "ibfs_teps")
        return e.value

    def autotune(self, src, base: Opts | None = None, reps: int = 2) -> tuple[Opts, float, list]:
        """Tune the options on this graph with a sample of sources."""
        import json

        src = np.ascontiguousarray(src, np.int32)
        best = Opts()
        g = C.c_double()
        buf = C.create_string_buffer(1 << 16)
        _check(_lib().ibfs_autotune(self._h, _ptr(src), len(src),
                                    C.byref(base) if base is not None else None, reps,
                                    C.byref(best), C.byref(g), buf, len(buf)), "ibfs_autotune")
        log = [json.loads(ln) for ln in buf.value.decode().split("\n") if ln.strip()]
        return best, g.value, log

    def bytes_alg(self, depth_dev_ptr: int, n: int, depth_bytes: int, width: int) -> int:
        b = C.c_int64()
        _check(_lib().ibfs_bytes_alg(self._h, C.c_void_p(depth_dev_ptr), n, depth_bytes, width,
                                     C.byref(b)), "ibfs_bytes_alg")
        return b.value

    def run(self, src, opts: Opts | None = None, layout: int = LAYOUT_SOURCE_MAJOR,
            out: np.ndarray | None = None, out_ptr: int | None = None, on_device: bool = False,
            levels_cap: int = 0, **kw) -> RunResult:
        """Concurrent BFS; returns per-source depths (uint8, or uint16 when a
        level exceeds 254) unless the output is a device pointer."""
        src = np.ascontiguousarray(src, np.int32)
        o = opts if opts is not None else default_opts(**kw)
        if opts is not None and kw:
            for k, v in kw.items():
                setattr(o, k, v)
        st = Stats()
        recs = None
        if levels_cap:
            recs = (LevelRec * levels_cap)()
            st.levels = C.cast(recs, C.POINTER(LevelRec))
            st.levels_cap = levels_cap
        n = len(src)
        flags = OUT_DEVICE if on_device else 0
        if on_device:
            if out_ptr is None:
                raise ValueError("on_device needs out_ptr")
            _check(_lib().ibfs_run(self._h, _ptr(src), n, C.byref(o), C.c_void_p(out_ptr), layout,
                                   flags, C.byref(st)), "ibfs_run")
            return RunResult(None, _stats_dict(st), _levels(recs, st))
        db = o.depth_bytes or 1
        if out is not None and (not out.flags.c_contiguous or out.size != n * self.V):
            raise ValueError(f"out must be a C-contiguous array of {n}*{self.V} depths, "
                             f"got shape {out.shape}")
        while True:
            dt = np.uint8 if db == 1 else np.uint16
            if out is None or out.dtype != dt:
                buf = np.empty((n, self.V), dt)
            else:
                buf = out
            o2 = Opts.from_buffer_copy(o)
            if o.depth_bytes == 0:
                o2.depth_bytes = db
            stc = _check_run(self._h, src, o2, buf, layout, st)
            if stc == 3 and o.depth_bytes == 0 and db == 1:
                db = 2
                continue
            _check(stc, "ibfs_run")
            break
        if layout == LAYOUT_VERTEX_MAJOR:
            buf = buf.reshape(-1)
        return RunResult(buf, _stats_dict(st), _levels(recs, st))


def _check_run(h, src, o, buf, layout, st) -> int:
    return _lib().ibfs_run(h, _ptr(src), len(src), C.byref(o), _ptr(buf), layout, 0, C.byref(st))


def _stats_dict(st: Stats) -> dict:
    return {k: getattr(st, k) for k, _ in Stats._fields_ if k not in ("levels", "levels_cap")}


def _levels(recs, st: Stats) -> list:
    if recs is None:
        return []
    return [dict(batch=recs[i].batch, level=recs[i].level, dir=recs[i].dir,
                 frontier=recs[i].frontier, frontier_edges=recs[i].frontier_edges,
                 expand_ns=recs[i].expand_ns, inspect_ns=recs[i].inspect_ns)
            for i in range(st.levels_len)]


class Server:
    """Continuous-batching query server on a resident graph (ibfs_server_*)."""

    def __init__(self, graph: "Graph", **kw):
        so = ServerOpts()
        _lib().ibfs_server_opts_default(C.byref(so))
        for k, v in kw.items():
            if hasattr(so, k):
                setattr(so, k, v)
            elif hasattr(so.run, k):
                setattr(so.run, k, v)
            else:
                raise TypeError(f"unknown server option {k}")
        self.graph = graph
        self.V = graph.V
        self.db = 2 if so.run.depth_bytes == 2 else 1
        h = C.c_void_p()
        _check(_lib().ibfs_server_create(graph.handle, C.byref(so), C.byref(h)),
               "ibfs_server_create")
        self._h = h

    def submit(self, src) -> int:
        src = np.ascontiguousarray(src, np.int32)
        qid = C.c_uint64()
        _check(_lib().ibfs_server_submit(self._h, _ptr(src), len(src), C.byref(qid)),
               "ibfs_server_submit")
        return qid.value

    def try_submit(self, src) -> int | None:
        """Submit, or None when admission refuses (IBFS_ERR_BUSY)."""
        src = np.ascontiguousarray(src, np.int32)
        qid = C.c_uint64()
        st = _lib().ibfs_server_submit(self._h, _ptr(src), len(src), C.byref(qid))
        if st == 9:
            return None
        _check(st, "ibfs_server_submit")
        return qid.value

    def poll(self, qid: int, n: int, want_depth: bool = True):
        """(done, depth or None, info dict)"""
        done = C.c_int32()
        info = QueryInfo()
        buf = np.empty((n, self.V), np.uint8 if self.db == 1 else np.uint16) if want_depth \
            else None
        _check(_lib().ibfs_server_poll(self._h, qid, _ptr(buf) if buf is not None else None, 0,
                                       C.byref(done), C.byref(info)), "ibfs_server_poll")
        if not done.value:
            return False, None, None
        return True, buf, _info(info)

    def wait(self, qid: int, n: int, timeout_ms: int = 60000, want_depth: bool = True,
             out_ptr: int | None = None, on_device: bool = False):
        """Block until the query is done and collect it: its depths into a new
        array (want_depth), into caller memory at out_ptr (host, or device
        with on_device; n*V*depth_bytes bytes), or nowhere."""
        info = QueryInfo()
        if out_ptr is not None:
            buf = None
            dst = C.c_void_p(out_ptr)
        else:
            buf = np.empty((n, self.V), np.uint8 if self.db == 1 else np.uint16) if want_depth \
                else None
            dst = _ptr(buf) if buf is not None else None
        _check(_lib().ibfs_server_wait(self._h, qid, timeout_ms, dst,
                                       OUT_DEVICE if (on_device and out_ptr is not None) else 0,
                                       C.byref(info)),
               "ibfs_server_wait")
        return buf, _info(info)

    def stats(self) -> dict:
        st = ServerStats()
        _check(_lib().ibfs_server_stats_get(self._h, C.byref(st)), "ibfs_server_stats_get")
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            _lib().ibfs_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _info(info: QueryInfo) -> dict:
    return {k: getattr(info, k) for k, _ in QueryInfo._fields_}


# Reference-named aliases ----------------------------------------------------
def graph_reader(beg_file: str, csr_file: str, device: int = 0) -> Graph:
    """graph_reader (graph_reader.cuh:63-119) + CSR upload."""
    return Graph.open(beg_file, csr_file, device)


def GroupBy(g: Graph, source_list: np.ndarray) -> np.ndarray:  # noqa: N802
    """GroupBy (GroupBy.cuh:6-115): hub-sharing sources first, by hub id."""
    return g.groupby(source_list)


def report(g: Graph, depth: np.ndarray) -> int:
    """report (validate.h:59-76): sum of deg(v) over reached (s, v)."""
    return g.teps(depth)
