"""CPU oracle (test infrastructure only).

Loads ``oracle/liboracle.so`` (built from oracle/oracle.c) with ctypes.  Only
the tests, ``__graft_entry__.smoke()`` and bench.py's CPU baseline / reference
arm use this module, and only as the checker or the timed CPU baseline --
never on the product path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_DIR = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_DIR, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built; run __graft_entry__.build()")
        lib = C.CDLL(path)
        P, I64 = C.c_void_p, C.c_int64
        lib.oracle_bfs.restype = C.c_int
        lib.oracle_bfs.argtypes = [P, P, I64, P, I64, C.c_int, P, C.POINTER(C.c_int32), C.c_int]
        lib.oracle_teps.restype = I64
        lib.oracle_teps.argtypes = [P, I64, P, I64, C.c_int]
        lib.oracle_groupby.restype = C.c_int
        lib.oracle_groupby.argtypes = [P, P, I64, P, I64, P]
        lib.oracle_bytes_alg.restype = I64
        lib.oracle_bytes_alg.argtypes = [P, P, I64, P, I64, C.c_int, C.c_int]
        lib.oracle_max_threads.restype = C.c_int
        lib.oracle_max_threads.argtypes = []
        _LIB = lib
    return _LIB


def _p(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class OracleRangeError(RuntimeError):
    pass


def bfs(beg: np.ndarray, col: np.ndarray, src, depth_bytes: int = 1,
        threads: int = 0) -> tuple[np.ndarray, int]:
    """Per-source BFS depths, source-major [n][V]; returns (depth, max_level)."""
    beg = np.ascontiguousarray(beg, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    src = np.ascontiguousarray(src, np.int32)
    V = len(beg) - 1
    out = np.empty((len(src), V), np.uint8 if depth_bytes == 1 else np.uint16)
    ml = C.c_int32(0)
    rc = _lib().oracle_bfs(_p(beg), _p(col), V, _p(src), len(src), depth_bytes, _p(out),
                           C.byref(ml), threads)
    if rc == 3:
        raise OracleRangeError("BFS level exceeds the depth type")
    if rc != 0:
        raise RuntimeError(f"oracle_bfs failed ({rc})")
    return out, ml.value


def bfs_auto(beg, col, src, threads: int = 0) -> tuple[np.ndarray, int]:
    """uint8 depths, widened to uint16 when a level exceeds 254."""
    try:
        return bfs(beg, col, src, 1, threads)
    except OracleRangeError:
        return bfs(beg, col, src, 2, threads)


def teps(beg: np.ndarray, depth: np.ndarray) -> int:
    beg = np.ascontiguousarray(beg, np.int64)
    depth = np.ascontiguousarray(depth)
    return int(_lib().oracle_teps(_p(beg), len(beg) - 1, _p(depth), depth.shape[0],
                                  depth.dtype.itemsize))


def groupby(beg, col, src) -> np.ndarray:
    beg = np.ascontiguousarray(beg, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    src = np.ascontiguousarray(src, np.int32)
    out = np.zeros_like(src)
    rc = _lib().oracle_groupby(_p(beg), _p(col), len(beg) - 1, _p(src), len(src), _p(out))
    if rc != 0:
        raise RuntimeError(f"oracle_groupby failed ({rc})")
    return out


def bytes_alg(beg, col, depth: np.ndarray, width: int) -> int:
    beg = np.ascontiguousarray(beg, np.int64)
    col = np.ascontiguousarray(col, np.int32)
    depth = np.ascontiguousarray(depth)
    return int(_lib().oracle_bytes_alg(_p(beg), _p(col), len(beg) - 1, _p(depth), depth.shape[0],
                                       depth.dtype.itemsize, width))


def max_threads() -> int:
    return int(_lib().oracle_max_threads())
