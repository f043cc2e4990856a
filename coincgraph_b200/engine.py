"""ctypes binding of libcig (include/cig.h).

This is a thin host-side mirror of the engine's C ABI for Python callers
(tests, the benchmark, notebooks).  It holds no algorithmic code: every call
goes to the sm_100a library, and importing it fails loudly when the library
has not been built.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# CIG_LIBRARY selects another build of the engine (e.g. the bounds-checked
# libcig_bc.so); the default is the release build next to this file.
LIB_PATH = os.environ.get("CIG_LIBRARY") or os.path.join(_HERE, "libcig.so")

BFS, SSSP, CC, PR = 0, 1, 2, 3
ALGOS = {"bfs": BFS, "sssp": SSSP, "cc": CC, "pr": PR}
FLAG_NO_CACHE_REFRESH = 0x1
FLAG_PR_FP64 = 0x2
FLAG_WEIGHT_U255 = 0x4
FLAG_NO_GRAPHS = 0x8
INF = 0xFFFFFFFF

STATUS = {
    0: "CIG_OK", -1: "CIG_ERR_ARG", -2: "CIG_ERR_NOMEM", -3: "CIG_ERR_DEVICE", -4: "CIG_ERR_ARENA",
    -5: "CIG_ERR_LIMIT", -6: "CIG_ERR_STATE", -7: "CIG_ERR_NOTIMPL",
}


class Options(ctypes.Structure):
    _fields_ = [
        ("algo", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("source", ctypes.c_uint32),
        ("cache_compat", ctypes.c_int32),
        ("cache_gib", ctypes.c_double),
        ("pr_epsilon", ctypes.c_double),
        ("pr_max_rounds", ctypes.c_int32),
        ("max_batch", ctypes.c_uint32),
        ("arena_headroom_pct", ctypes.c_uint32),
        ("flags", ctypes.c_uint32),
        ("index_budget_gib", ctypes.c_double),
    ]


class MemoryInfo(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint64) for name in (
        "total", "edge_cache", "segment_table", "descriptors", "reverse_arena", "position_index", "vertex_state",
        "batch_buffers", "query_buffers", "pinned_host")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchStats(ctypes.Structure):
    _fields_ = [
        ("requested_deletes", ctypes.c_uint64),
        ("missing_deletes", ctypes.c_uint64),
        ("requested_additions", ctypes.c_uint64),
        ("invalid_additions", ctypes.c_uint64),
        ("changed_sources", ctypes.c_uint64),
        ("relocated_rows", ctypes.c_uint64),
        ("affected", ctypes.c_uint64),
        ("seeds", ctypes.c_uint64),
        ("rounds", ctypes.c_uint64),
        ("edges_scanned", ctypes.c_uint64),
        ("edges_scanned_cached", ctypes.c_uint64),
        ("vertices_expanded", ctypes.c_uint64),
        ("cache_segments_loaded", ctypes.c_uint64),
        ("cache_segments_evicted", ctypes.c_uint64),
        ("ms_delete", ctypes.c_double),
        ("ms_insert", ctypes.c_double),
        ("ms_cache", ctypes.c_double),
        ("pr_rounds", ctypes.c_uint64),
        ("pr_residual_l1", ctypes.c_double),
        ("kernel_launches", ctypes.c_uint64),
        ("graph_replays", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class GraphInfo(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint32),
        ("m", ctypes.c_uint64),
        ("arena_capacity_edges", ctypes.c_uint64),
        ("arena_used_edges", ctypes.c_uint64),
        ("segment_edges", ctypes.c_uint64),
        ("segments_total", ctypes.c_uint64),
        ("segments_resident", ctypes.c_uint64),
        ("cache_capacity_segments", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
        ("pinned_bytes", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class UpdateBatch(ctypes.Structure):
    _fields_ = [
        ("del_u", ctypes.c_void_p),
        ("del_v", ctypes.c_void_p),
        ("nd", ctypes.c_uint64),
        ("add_u", ctypes.c_void_p),
        ("add_v", ctypes.c_void_p),
        ("na", ctypes.c_uint64),
    ]


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("blocks_per_sm", ctypes.c_uint32),
        ("split_degree", ctypes.c_uint32),
        ("best_ms", ctypes.c_double),
        ("candidates", ctypes.c_uint32),
        ("pull_divisor", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


REQ_UPDATE, REQ_BFS, REQ_SSSP = 0, 1, 2


class Request(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("source", ctypes.c_uint32),
        ("del_u", ctypes.c_void_p),
        ("del_v", ctypes.c_void_p),
        ("nd", ctypes.c_uint64),
        ("add_u", ctypes.c_void_p),
        ("add_v", ctypes.c_void_p),
        ("na", ctypes.c_uint64),
        ("out", ctypes.c_void_p),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("wave", ctypes.c_uint32),
        ("digest", ctypes.c_uint64),
        ("submit_ms", ctypes.c_double),
        ("start_ms", ctypes.c_double),
        ("done_ms", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServeOptions(ctypes.Structure):
    _fields_ = [
        ("budget_bytes", ctypes.c_uint64),
        ("max_wave", ctypes.c_uint32),
        ("max_pending", ctypes.c_uint32),
    ]


class QueryStats(ctypes.Structure):
    _fields_ = [
        ("ms", ctypes.c_double),
        ("edges_scanned", ctypes.c_uint64),
        ("edges_scanned_cached", ctypes.c_uint64),
        ("rows_expanded", ctypes.c_uint64),
        ("source_edges", ctypes.c_uint64),
        ("rounds", ctypes.c_uint64),
        ("waves", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


STAGES = ["group", "mutate", "seed", "inval", "pull", "push", "pr", "cache", "mutate_rev", "add", "add_rev",
          "del_scan", "index"]


class StageProfile(ctypes.Structure):
    _fields_ = [
        ("ms", ctypes.c_double),
        ("launches", ctypes.c_uint64),
        ("edges", ctypes.c_uint64),
        ("edges_cached", ctypes.c_uint64),
        ("rows", ctypes.c_uint64),
        ("hits", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# (name, restype, argtypes) of every symbol include/cig.h declares.
_vp = ctypes.c_void_p
_u32, _u64, _i32 = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int
SIGNATURES = [
    ("cig_options_default", _i32, [ctypes.POINTER(Options)]),
    ("cig_create", _i32, [ctypes.POINTER(Options), ctypes.POINTER(_vp)]),
    ("cig_destroy", _i32, [_vp]),
    ("cig_last_error", ctypes.c_char_p, [_vp]),
    ("cig_load_csr", _i32, [_vp, _u32, _vp, _vp]),
    ("cig_load_edges", _i32, [_vp, _u32, _vp, _vp, _u64]),
    ("cig_init", _i32, [_vp]),
    ("cig_delete_phase", _i32, [_vp, _vp, _vp, _u64, ctypes.POINTER(BatchStats)]),
    ("cig_insert_phase", _i32, [_vp, _vp, _vp, _u64, ctypes.POINTER(BatchStats)]),
    ("cig_apply_batch", _i32, [_vp, _vp, _vp, _u64, _vp, _vp, _u64, ctypes.POINTER(BatchStats)]),
    ("cig_apply_batch_device", _i32, [_vp, _vp, _vp, _u64, _vp, _vp, _u64, ctypes.POINTER(BatchStats)]),
    ("cig_get_values", _i32, [_vp, _vp]),
    ("cig_get_parents", _i32, [_vp, _vp]),
    ("cig_get_pr", _i32, [_vp, _vp, _vp]),
    ("cig_get_pr64", _i32, [_vp, _vp, _vp]),
    ("cig_value_digest", _i32, [_vp, ctypes.POINTER(_u64)]),
    ("cig_num_edges", _i32, [_vp, ctypes.POINTER(_u64)]),
    ("cig_get_degrees", _i32, [_vp, _vp]),
    ("cig_get_row", _i32, [_vp, _u32, _vp, _u32, ctypes.POINTER(_u32)]),
    ("cig_export_csr", _i32, [_vp, _vp, _vp]),
    ("cig_graph_info_get", _i32, [_vp, ctypes.POINTER(GraphInfo)]),
    ("cig_profile_enable", _i32, [_vp, _i32]),
    ("cig_profile_read", _i32, [_vp, ctypes.POINTER(StageProfile), _u32]),
    ("cig_bfs_csr_noalloc", _i32, [_vp, _vp, _u32, _u32, _vp, _vp]),
    ("cig_memory_info_get", _i32, [_vp, ctypes.POINTER(MemoryInfo)]),
    ("cig_build_info", _i32, [ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
    ("cig_apply_batches_device", _i32, [_vp, ctypes.POINTER(UpdateBatch), _u32, ctypes.POINTER(BatchStats), _vp]),
    ("cig_autotune", _i32, [_vp, ctypes.POINTER(TuneResult)]),
    ("cig_serve_start", _i32, [_vp, ctypes.POINTER(ServeOptions)]),
    ("cig_serve_submit", _i32, [_vp, ctypes.POINTER(Request), ctypes.POINTER(_u64)]),
    ("cig_serve_wait", _i32, [_vp, _u64, ctypes.POINTER(Result)]),
    ("cig_serve_poll", _i32, [_vp, _u64, ctypes.POINTER(Result), ctypes.POINTER(ctypes.c_int)]),
    ("cig_serve_stop", _i32, [_vp]),
    ("cig_query_bfs_multi", _i32, [_vp, _vp, _u32, _vp]),
    ("cig_query_sssp_multi", _i32, [_vp, _vp, _u32, _vp]),
    ("cig_query_multi_device", _i32, [_vp, _i32, _vp, _u32, _u32, _vp, ctypes.POINTER(QueryStats)]),
    ("cig_version", ctypes.c_char_p, []),
]

_LIB = None


def load_library(path: str = LIB_PATH):
    """Load libcig.so and declare its signatures; raises if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m coincgraph_b200.build`")
    lib = ctypes.CDLL(path)
    for name, restype, argtypes in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _LIB = lib
    return lib


class CigError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    if hasattr(a, "data_ptr"):  # torch tensor (device arrays for *_device calls)
        return a.data_ptr()
    raise TypeError(type(a))


def _u32arr(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint32))


def default_options() -> Options:
    o = Options()
    load_library().cig_options_default(ctypes.byref(o))
    return o


class Engine:
    """One graph on one GPU (wraps a cig_handle)."""

    def __init__(self, algo="sssp", device: int = 0, source: int = 0, cache_gib: float = 4.0,
                 cache_compat: bool = False, pr_epsilon: float = 1e-6, pr_max_rounds: int = 100,
                 max_batch: int = 0, headroom_pct: int = 0, flags: int = 0, index_budget_gib: float = 0.0):
        self.lib = load_library()
        o = default_options()
        o.algo = ALGOS[algo] if isinstance(algo, str) else int(algo)
        o.device = device
        o.source = source
        o.cache_gib = cache_gib
        o.cache_compat = int(cache_compat)
        o.pr_epsilon = pr_epsilon
        o.pr_max_rounds = pr_max_rounds
        o.max_batch = max_batch
        o.arena_headroom_pct = headroom_pct
        o.flags = flags
        o.index_budget_gib = index_budget_gib
        self.options = o
        h = ctypes.c_void_p()
        rc = self.lib.cig_create(ctypes.byref(o), ctypes.byref(h))
        if rc != 0:
            raise CigError(rc, self.lib.cig_last_error(None).decode())
        self.h = h
        self.n = 0

    # -- plumbing
    def _check(self, rc: int):
        if rc != 0:
            raise CigError(rc, self.lib.cig_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.cig_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- graph
    def load_csr(self, n: int, xadj, adj):
        xadj = np.ascontiguousarray(np.asarray(xadj, dtype=np.uint64))
        adj = _u32arr(adj)
        self._check(self.lib.cig_load_csr(self.h, n, _ptr(xadj), _ptr(adj)))
        self.n = n

    def load_edges(self, n: int, src, dst):
        src, dst = _u32arr(src), _u32arr(dst)
        self._check(self.lib.cig_load_edges(self.h, n, _ptr(src), _ptr(dst), len(src)))
        self.n = n

    def init(self):
        self._check(self.lib.cig_init(self.h))

    # -- batches (host arrays)
    def delete_phase(self, u, v) -> dict:
        u, v = _u32arr(u), _u32arr(v)
        s = BatchStats()
        self._check(self.lib.cig_delete_phase(self.h, _ptr(u), _ptr(v), len(u), ctypes.byref(s)))
        return s.as_dict()

    def insert_phase(self, u, v) -> dict:
        u, v = _u32arr(u), _u32arr(v)
        s = BatchStats()
        self._check(self.lib.cig_insert_phase(self.h, _ptr(u), _ptr(v), len(u), ctypes.byref(s)))
        return s.as_dict()

    def apply_batch(self, du, dv, au, av) -> dict:
        du, dv, au, av = _u32arr(du), _u32arr(dv), _u32arr(au), _u32arr(av)
        s = BatchStats()
        self._check(self.lib.cig_apply_batch(self.h, _ptr(du), _ptr(dv), len(du), _ptr(au), _ptr(av), len(au),
                                             ctypes.byref(s)))
        return s.as_dict()

    def apply_batch_device(self, du, dv, au, av, stats: BatchStats | None = None) -> BatchStats:
        """Device-resident update arrays (e.g. torch uint32/int32 CUDA tensors)."""
        s = stats if stats is not None else BatchStats()
        nd = int(du.numel()) if hasattr(du, "numel") else len(du)
        na = int(au.numel()) if hasattr(au, "numel") else len(au)
        self._check(self.lib.cig_apply_batch_device(self.h, _ptr(du), _ptr(dv), nd, _ptr(au), _ptr(av), na,
                                                    ctypes.byref(s)))
        return s

    def apply_batches_device(self, batches, digests: bool = True):
        """The batched form: a list of (du, dv, au, av) device arrays applied
        with one synchronisation; returns per-batch stats and digests."""
        arr = (UpdateBatch * max(len(batches), 1))()
        for i, (du, dv, au, av) in enumerate(batches):
            nd = int(du.numel()) if hasattr(du, "numel") else len(du)
            na = int(au.numel()) if hasattr(au, "numel") else len(au)
            arr[i] = UpdateBatch(_ptr(du), _ptr(dv), nd, _ptr(au), _ptr(av), na)
        st = (BatchStats * max(len(batches), 1))()
        dg = np.zeros(max(len(batches), 1), dtype=np.uint64)
        self._check(self.lib.cig_apply_batches_device(self.h, arr, len(batches), st,
                                                      _ptr(dg) if digests else None))
        return [st[i] for i in range(len(batches))], [int(x) for x in dg[: len(batches)]]

    # -- results
    def values(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.uint32)
        self._check(self.lib.cig_get_values(self.h, _ptr(out)))
        return out

    def parents(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.uint32)
        self._check(self.lib.cig_get_parents(self.h, _ptr(out)))
        return out

    def pagerank(self, fp64: bool = False):
        if fp64:
            r = np.empty(self.n, dtype=np.float64)
            s = np.empty(self.n, dtype=np.float64)
            self._check(self.lib.cig_get_pr64(self.h, _ptr(r), _ptr(s)))
        else:
            r = np.empty(self.n, dtype=np.float32)
            s = np.empty(self.n, dtype=np.float32)
            self._check(self.lib.cig_get_pr(self.h, _ptr(r), _ptr(s)))
        return r, s

    def autotune(self) -> dict:
        r = TuneResult()
        self._check(self.lib.cig_autotune(self.h, ctypes.byref(r)))
        return r.as_dict()

    # -- serving
    def serve_start(self, budget_bytes: int = 0, max_wave: int = 0, max_pending: int = 0):
        o = ServeOptions(budget_bytes, max_wave, max_pending)
        self._check(self.lib.cig_serve_start(self.h, ctypes.byref(o)))
        self._keep = {}

    def _serve_check(self, rc: int):
        if rc != 0:
            raise CigError(rc, self.lib.cig_last_error(None).decode(errors="replace"))

    def submit_update(self, du, dv, au, av) -> int:
        du, dv, au, av = _u32arr(du), _u32arr(dv), _u32arr(au), _u32arr(av)
        r = Request(REQ_UPDATE, 0, _ptr(du), _ptr(dv), len(du), _ptr(au), _ptr(av), len(au), None)
        t = ctypes.c_uint64()
        self._serve_check(self.lib.cig_serve_submit(self.h, ctypes.byref(r), ctypes.byref(t)))
        return t.value

    def submit_query(self, algo: str, source: int, out: np.ndarray | None = None) -> int:
        kind = REQ_BFS if algo == "bfs" else REQ_SSSP
        r = Request(kind, int(source), None, None, 0, None, None, 0, _ptr(out) if out is not None else None)
        t = ctypes.c_uint64()
        self._serve_check(self.lib.cig_serve_submit(self.h, ctypes.byref(r), ctypes.byref(t)))
        if out is not None:
            self._keep[t.value] = out  # the library writes into it when the wave ends
        return t.value

    def wait(self, ticket: int) -> dict:
        res = Result()
        self._serve_check(self.lib.cig_serve_wait(self.h, ticket, ctypes.byref(res)))
        self._keep.pop(ticket, None)
        return res.as_dict()

    def poll(self, ticket: int):
        res = Result()
        done = ctypes.c_int()
        self._serve_check(self.lib.cig_serve_poll(self.h, ticket, ctypes.byref(res), ctypes.byref(done)))
        if done.value:
            self._keep.pop(ticket, None)
            return res.as_dict()
        return None

    def serve_stop(self):
        self._check(self.lib.cig_serve_stop(self.h))

    # -- multi-source queries on the current graph
    def query_bfs(self, sources) -> np.ndarray:
        """k x n BFS depths (UINT32_MAX for unreached), k = len(sources)."""
        src = _u32arr(sources)
        out = np.empty((len(src), self.n), dtype=np.uint32)
        self._check(self.lib.cig_query_bfs_multi(self.h, _ptr(src), len(src), _ptr(out)))
        return out

    def query_sssp(self, sources) -> np.ndarray:
        """k x n SSSP distances (UINT32_MAX for unreached), k = len(sources)."""
        src = _u32arr(sources)
        out = np.empty((len(src), self.n), dtype=np.uint32)
        self._check(self.lib.cig_query_sssp_multi(self.h, _ptr(src), len(src), _ptr(out)))
        return out

    def query_device(self, algo: str, sources, out, width: int = 64) -> dict:
        """Results into device memory `out` (k x n words, e.g. a torch CUDA
        tensor); width 64 = batched bitmask waves, 1 = per-source form."""
        src = _u32arr(sources)
        s = QueryStats()
        self._check(self.lib.cig_query_multi_device(self.h, ALGOS[algo], _ptr(src), len(src), width, _ptr(out),
                                                    ctypes.byref(s)))
        return s.as_dict()

    def digest(self) -> int:
        out = ctypes.c_uint64()
        self._check(self.lib.cig_value_digest(self.h, ctypes.byref(out)))
        return out.value

    def num_edges(self) -> int:
        out = ctypes.c_uint64()
        self._check(self.lib.cig_num_edges(self.h, ctypes.byref(out)))
        return out.value

    def degrees(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.uint32)
        self._check(self.lib.cig_get_degrees(self.h, _ptr(out)))
        return out

    def row(self, v: int) -> np.ndarray:
        deg = ctypes.c_uint32()
        self._check(self.lib.cig_get_row(self.h, v, None, 0, ctypes.byref(deg)))
        out = np.empty(max(deg.value, 1), dtype=np.uint32)
        self._check(self.lib.cig_get_row(self.h, v, _ptr(out), deg.value, ctypes.byref(deg)))
        return out[: deg.value]

    def export_csr(self):
        xadj = np.empty(self.n + 1, dtype=np.uint64)
        self._check(self.lib.cig_export_csr(self.h, _ptr(xadj), None))
        adj = np.empty(max(int(xadj[-1]), 1), dtype=np.uint32)
        self._check(self.lib.cig_export_csr(self.h, _ptr(xadj), _ptr(adj)))
        return xadj, adj[: int(xadj[-1])]

    def profile(self, enable: bool = True):
        """Clear the per-stage accumulators and turn stage timing on/off."""
        self._check(self.lib.cig_profile_enable(self.h, int(enable)))

    def profile_read(self) -> dict:
        arr = (StageProfile * len(STAGES))()
        self._check(self.lib.cig_profile_read(self.h, arr, len(STAGES)))
        return {name: arr[i].as_dict() for i, name in enumerate(STAGES)}

    def memory(self) -> dict:
        """Device bytes held by this handle, by part (cig_memory_info_get)."""
        m = MemoryInfo()
        self._check(self.lib.cig_memory_info_get(self.h, ctypes.byref(m)))
        return m.as_dict()

    def info(self) -> dict:
        g = GraphInfo()
        self._check(self.lib.cig_graph_info_get(self.h, ctypes.byref(g)))
        return g.as_dict()


def version() -> str:
    return load_library().cig_version().decode()


def build_info() -> dict:
    """{"binary_version": 100 for sm_100a, "bounds_checked": bool}; needs a GPU."""
    bv, bc = ctypes.c_int(), ctypes.c_int()
    rc = load_library().cig_build_info(ctypes.byref(bv), ctypes.byref(bc))
    if rc != 0:
        raise CigError(rc, load_library().cig_last_error(None).decode())
    return {"binary_version": bv.value, "bounds_checked": bool(bc.value)}
