"""CPU oracle (test infrastructure only).

Python access to ``oracle/liboracle.so`` (the plain-C restatement in
``oracle/oracle.c``) and, when it has been built, ``oracle/_ref/
libcigref.so`` (the reference's own chunk store and host checkers compiled
from its sources).  Only tests, the smoke check and the benchmark's CPU
baseline import this package; the product never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libcigref.so")

BFS, SSSP, CC, SSSP_U255 = 0, 1, 2, 3
INF = 0xFFFFFFFF

_vp, _u32, _u64, _i32, _dbl = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
_LIB = None
_REF = None


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build_oracle()
        L = ctypes.CDLL(LIB_PATH)
        L.og_create.restype = _vp
        L.og_create.argtypes = [_u32, _vp, _vp]
        L.og_free.argtypes = [_vp]
        L.og_free.restype = None
        L.og_n.restype = _u32
        L.og_n.argtypes = [_vp]
        L.og_m.restype = _u64
        L.og_m.argtypes = [_vp]
        L.og_degree.restype = _u32
        L.og_degree.argtypes = [_vp, _u32]
        L.og_row.restype = ctypes.POINTER(_u32)
        L.og_row.argtypes = [_vp, _u32]
        L.og_export.argtypes = [_vp, _vp, _vp]
        L.og_export.restype = None
        L.og_delete.restype = _u64
        L.og_delete.argtypes = [_vp, _vp, _vp, _u64]
        L.og_add.restype = _u64
        L.og_add.argtypes = [_vp, _vp, _vp, _u64]
        L.og_sssp_fifo.argtypes = [_vp, _u32, _i32, _vp, _vp]
        L.og_sssp_fifo.restype = None
        L.og_sssp_dial.argtypes = [_vp, _u32, _i32, _vp]
        L.og_sssp_dial.restype = None
        L.og_cc.argtypes = [_vp, _vp]
        L.og_cc.restype = None
        L.og_pr.argtypes = [_vp, _dbl, _i32, _vp]
        L.og_pr.restype = _i32
        L.og_bellman_check.argtypes = [_vp, _vp, _u32, _i32, _vp]
        L.og_bellman_check.restype = None
        L.og_parent_check.argtypes = [_vp, _vp, _vp, _u32, _i32, _vp]
        L.og_parent_check.restype = None
        L.og_checksum.restype = _u64
        L.og_checksum.argtypes = [_vp, _u32]
        L.og_row_hash.restype = _u64
        L.og_row_hash.argtypes = [_vp, _u32]
        L.og_pr_check.argtypes = [_vp, _vp, _vp, _dbl, _vp]
        L.og_pr_check.restype = None
        _LIB = L
    return _LIB


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref_lib():
    global _REF
    if _REF is None:
        if not os.path.exists(REF_PATH):
            raise RuntimeError("oracle/_ref/libcigref.so is not built (needs the reference tree)")
        R = ctypes.CDLL(REF_PATH)
        R.ref_store_create.restype = _vp
        R.ref_store_create.argtypes = [_u32, _vp, _vp, _u32, _u64]
        R.ref_store_free.argtypes = [_vp]
        R.ref_store_free.restype = None
        R.ref_store_apply.restype = _i32
        R.ref_store_apply.argtypes = [_vp, _vp, _vp, _u64, _vp, _vp, _u64, _vp]
        R.ref_store_edges.restype = _u64
        R.ref_store_edges.argtypes = [_vp]
        R.ref_store_degree.restype = _u32
        R.ref_store_degree.argtypes = [_vp, _u32]
        R.ref_store_export.argtypes = [_vp, _vp, _vp]
        R.ref_store_export.restype = None
        R.ref_store_row_hash.restype = _u64
        R.ref_store_row_hash.argtypes = [_vp, _u32]
        R.ref_cc_check.restype = _u64
        R.ref_cc_check.argtypes = [_vp, _vp]
        R.ref_pr_check.restype = _i32
        R.ref_pr_check.argtypes = [_vp, _vp, _vp, _dbl]
        _REF = R
    return _REF


def _u32a(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


class Graph:
    """Mutable multigraph with the reference's row-mutation semantics."""

    def __init__(self, n: int, xadj, adj):
        self.n = int(n)
        self._xadj = np.ascontiguousarray(np.asarray(xadj, dtype=np.uint64))
        self._adj = _u32a(adj) if len(adj) else np.zeros(1, dtype=np.uint32)
        self.h = lib().og_create(self.n, _ptr(self._xadj), _ptr(self._adj))
        if not self.h:
            raise MemoryError("og_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().og_free(self.h)
            self.h = None

    @property
    def m(self) -> int:
        return int(lib().og_m(self.h))

    def delete(self, u, v) -> int:
        u, v = _u32a(u), _u32a(v)
        return int(lib().og_delete(self.h, _ptr(u), _ptr(v), len(u)))

    def add(self, u, v) -> int:
        u, v = _u32a(u), _u32a(v)
        return int(lib().og_add(self.h, _ptr(u), _ptr(v), len(u)))

    def row(self, v: int) -> np.ndarray:
        d = lib().og_degree(self.h, v)
        if d == 0:
            return np.zeros(0, dtype=np.uint32)
        p = lib().og_row(self.h, v)
        return np.ctypeslib.as_array(p, shape=(d,)).copy()

    def export(self):
        xadj = np.empty(self.n + 1, dtype=np.uint64)
        adj = np.empty(max(self.m, 1), dtype=np.uint32)
        lib().og_export(self.h, _ptr(xadj), _ptr(adj))
        return xadj, adj[: self.m]

    def sssp(self, src: int, mode: int = SSSP, parents: bool = False):
        d = np.empty(self.n, dtype=np.uint32)
        p = np.empty(self.n, dtype=np.uint32) if parents else None
        lib().og_sssp_fifo(self.h, src, mode, _ptr(d), _ptr(p) if p is not None else None)
        return (d, p) if parents else d

    def sssp_dial(self, src: int, mode: int = SSSP) -> np.ndarray:
        d = np.empty(self.n, dtype=np.uint32)
        lib().og_sssp_dial(self.h, src, mode, _ptr(d))
        return d

    def cc(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.uint32)
        lib().og_cc(self.h, _ptr(out))
        return out

    def pagerank(self, tol_per_vertex: float = 1e-13, max_rounds: int = 20000):
        x = np.empty(self.n, dtype=np.float64)
        ok = lib().og_pr(self.h, tol_per_vertex, max_rounds, _ptr(x))
        return x, bool(ok)

    def bellman_check(self, dist, src: int, mode: int = SSSP):
        dist = _u32a(dist)
        out = np.zeros(2, dtype=np.uint64)
        lib().og_bellman_check(self.h, _ptr(dist), src, mode, _ptr(out))
        return int(out[0]), int(out[1])

    def parent_check(self, dist, parent, src: int, mode: int = SSSP):
        dist, parent = _u32a(dist), _u32a(parent)
        out = np.zeros(3, dtype=np.uint64)
        lib().og_parent_check(self.h, _ptr(dist), _ptr(parent), src, mode, _ptr(out))
        return int(out[0]), int(out[1]), int(out[2])

    def row_hash(self, v: int) -> int:
        return int(lib().og_row_hash(self.h, v))

    def pr_check(self, rank, residual, epsilon: float):
        rank = np.ascontiguousarray(np.asarray(rank, dtype=np.float32))
        residual = np.ascontiguousarray(np.asarray(residual, dtype=np.float32))
        out = np.zeros(6, dtype=np.float64)
        lib().og_pr_check(self.h, _ptr(rank), _ptr(residual), epsilon, _ptr(out))
        keys = ["ok", "l1", "bound", "max_error", "invariant_l1", "max_residual"]
        return dict(zip(keys, out.tolist()))


def checksum(values) -> int:
    values = _u32a(values)
    return int(lib().og_checksum(_ptr(values), len(values)))


class RefStore:
    """The reference's SourceLocalChunkStore (compiled from its sources)."""

    def __init__(self, n: int, xadj, adj, workers: int = 2, extra_capacity: int = 0):
        self.n = int(n)
        xadj = np.ascontiguousarray(np.asarray(xadj, dtype=np.uint64))
        adj = _u32a(adj) if len(adj) else np.zeros(1, dtype=np.uint32)
        self.h = ref_lib().ref_store_create(self.n, _ptr(xadj), _ptr(adj), workers, extra_capacity)
        if not self.h:
            raise RuntimeError("ref_store_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            ref_lib().ref_store_free(self.h)
            self.h = None

    def apply(self, du, dv, au, av):
        du, dv, au, av = _u32a(du), _u32a(dv), _u32a(au), _u32a(av)
        out = np.zeros(4, dtype=np.uint64)
        rc = ref_lib().ref_store_apply(self.h, _ptr(du), _ptr(dv), len(du), _ptr(au), _ptr(av), len(au), _ptr(out))
        if rc != 0:
            raise RuntimeError("ref_store_apply failed")
        return {"missing_deletes": int(out[0]), "invalid_additions": int(out[1])}

    @property
    def m(self) -> int:
        return int(ref_lib().ref_store_edges(self.h))

    def export(self):
        xadj = np.empty(self.n + 1, dtype=np.uint64)
        total = sum(int(ref_lib().ref_store_degree(self.h, v)) for v in range(self.n))
        adj = np.empty(max(total, 1), dtype=np.uint32)
        ref_lib().ref_store_export(self.h, _ptr(xadj), _ptr(adj))
        return xadj, adj[:total]

    def cc_errors(self, labels) -> int:
        labels = _u32a(labels)
        return int(ref_lib().ref_cc_check(self.h, _ptr(labels)))

    def pr_check(self, rank, residual, epsilon: float) -> bool:
        rank = np.ascontiguousarray(np.asarray(rank, dtype=np.float32))
        residual = np.ascontiguousarray(np.asarray(residual, dtype=np.float32))
        return bool(ref_lib().ref_pr_check(self.h, _ptr(rank), _ptr(residual), epsilon))
