"""Seeded synthetic graphs and update streams (wraps ``libcig_gen.so``).

See ``include/cig_gen.h`` for the generator's definition.  The seeds follow
one convention: graph seed ``0xC01C0000 + scale`` and update-stream seed
``0xC01C1000 + workload number``.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

GRAPH_SEED_BASE = 0xC01C0000
UPDATE_SEED_BASE = 0xC01C1000


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libcig_gen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run `python -m coincgraph_b200.build`")
        lib = ctypes.CDLL(path)
        u32, u64, i32, dbl = ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int, ctypes.c_double
        vp = ctypes.c_void_p
        lib.cig_gen_rmat.argtypes = [u32, u32, dbl, dbl, dbl, u64, i32, i32, ctypes.POINTER(vp)]
        lib.cig_gen_rmat.restype = i32
        lib.cig_gen_sizes.argtypes = [vp, ctypes.POINTER(u32), ctypes.POINTER(u64)]
        lib.cig_gen_copy_csr.argtypes = [vp, vp, vp]
        lib.cig_gen_updates.argtypes = [vp, u32, vp, vp, u64, i32, vp, vp, vp, vp]
        lib.cig_gen_updates.restype = i32
        lib.cig_gen_free.argtypes = [vp]
        lib.cig_gen_free.restype = None
        lib.cig_gen_threads.restype = i32
        _LIB = lib
    return _LIB


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


@dataclass
class Graph:
    """A directed multigraph in CSR form (rows in stored order)."""

    n: int
    xadj: np.ndarray  # uint64[n+1]
    adj: np.ndarray  # uint32[m]

    @property
    def m(self) -> int:
        return int(self.adj.shape[0])

    def degrees(self) -> np.ndarray:
        return np.diff(self.xadj).astype(np.uint64)


@dataclass
class UpdateStream:
    """Concatenated update batches; batch i spans del/add offsets [off[i], off[i+1])."""

    del_u: np.ndarray
    del_v: np.ndarray
    add_u: np.ndarray
    add_v: np.ndarray
    del_off: np.ndarray
    add_off: np.ndarray

    @property
    def batches(self) -> int:
        return int(self.del_off.shape[0] - 1)

    def batch(self, i: int):
        d0, d1 = int(self.del_off[i]), int(self.del_off[i + 1])
        a0, a1 = int(self.add_off[i]), int(self.add_off[i + 1])
        return self.del_u[d0:d1], self.del_v[d0:d1], self.add_u[a0:a1], self.add_v[a0:a1]


class _Handle:
    def __init__(self, h):
        self.h = h

    def __del__(self):
        if self.h:
            _lib().cig_gen_free(self.h)
            self.h = None


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int | None = None, symmetric: bool = False, permute: bool = True,
         keep_handle: bool = False):
    """R-MAT graph with self-loops and duplicates removed (rows sorted)."""
    lib = _lib()
    if seed is None:
        seed = GRAPH_SEED_BASE + scale
    h = ctypes.c_void_p()
    rc = lib.cig_gen_rmat(scale, edge_factor, a, b, c, seed, int(symmetric), int(permute), ctypes.byref(h))
    if rc != 0:
        raise RuntimeError(f"cig_gen_rmat failed ({rc})")
    handle = _Handle(h)
    n, m = ctypes.c_uint32(), ctypes.c_uint64()
    lib.cig_gen_sizes(h, ctypes.byref(n), ctypes.byref(m))
    xadj = np.empty(n.value + 1, dtype=np.uint64)
    adj = np.empty(m.value, dtype=np.uint32)
    lib.cig_gen_copy_csr(h, _ptr(xadj), _ptr(adj))
    g = Graph(n.value, xadj, adj)
    if keep_handle:
        return g, handle
    return g


def updates(graph_handle, del_sizes, add_sizes, seed: int, symmetric: bool = False) -> UpdateStream:
    """Update batches against the evolving edge set of a generated graph."""
    lib = _lib()
    ds = np.ascontiguousarray(np.asarray(del_sizes, dtype=np.uint64))
    as_ = np.ascontiguousarray(np.asarray(add_sizes, dtype=np.uint64))
    nd, na = int(ds.sum()), int(as_.sum())
    du = np.empty(max(nd, 1), dtype=np.uint32)
    dv = np.empty(max(nd, 1), dtype=np.uint32)
    au = np.empty(max(na, 1), dtype=np.uint32)
    av = np.empty(max(na, 1), dtype=np.uint32)
    rc = lib.cig_gen_updates(graph_handle.h, len(ds), _ptr(ds), _ptr(as_), seed, int(symmetric),
                             _ptr(du), _ptr(dv), _ptr(au), _ptr(av))
    if rc != 0:
        raise RuntimeError(f"cig_gen_updates failed ({rc})")
    del_off = np.concatenate([[0], np.cumsum(ds)]).astype(np.int64)
    add_off = np.concatenate([[0], np.cumsum(as_)]).astype(np.int64)
    return UpdateStream(du[:nd], dv[:nd], au[:na], av[:na], del_off, add_off)


def grid(side: int, seed: int | None = None) -> Graph:
    """Road-like graph: a side x side grid, each vertex joined both ways to
    its 4 neighbours (rows in east, west, south, north order), vertex
    i * side + j at row i, column j.  High diameter (2 * side hops) and
    degree <= 4, unlike R-MAT."""
    n = side * side
    i, j = np.divmod(np.arange(n, dtype=np.int64), side)
    cand = np.stack([np.where(j + 1 < side, i * side + j + 1, -1), np.where(j > 0, i * side + j - 1, -1),
                     np.where(i + 1 < side, (i + 1) * side + j, -1), np.where(i > 0, (i - 1) * side + j, -1)], axis=1)
    deg = (cand >= 0).sum(axis=1)
    xadj = np.zeros(n + 1, dtype=np.uint64)
    xadj[1:] = np.cumsum(deg)
    adj = cand[cand >= 0].astype(np.uint32)
    return Graph(n, xadj, adj)


def local_updates(g: Graph, side: int, del_sizes, add_sizes, seed: int, reach: int = 3) -> UpdateStream:
    """Update batches for a grid: deletions of distinct existing edges in a
    seeded random order (each edge deleted at most once), insertions of new
    pairs (u, v) with v within `reach` rows and columns of u (road-like
    shortcuts), never an existing or already inserted pair."""
    rng = np.random.default_rng(seed)
    src = np.repeat(np.arange(g.n, dtype=np.uint64), np.diff(g.xadj).astype(np.int64))
    order = rng.permutation(g.m)
    nd, na = int(np.sum(del_sizes)), int(np.sum(add_sizes))
    pick = order[:nd]
    du, dv = src[pick].astype(np.uint32), g.adj[pick]
    existing = set((src.astype(np.uint64) << np.uint64(32) | g.adj.astype(np.uint64)).tolist())
    au, av = np.empty(na, dtype=np.uint32), np.empty(na, dtype=np.uint32)
    k = 0
    while k < na:
        u = rng.integers(0, g.n, size=2 * (na - k) + 16)
        di = rng.integers(-reach, reach + 1, size=u.shape[0])
        dj = rng.integers(-reach, reach + 1, size=u.shape[0])
        ui, uj = np.divmod(u, side)
        vi, vj = ui + di, uj + dj
        ok = (vi >= 0) & (vi < side) & (vj >= 0) & (vj < side) & ((di != 0) | (dj != 0))
        for a, b in zip(u[ok].tolist(), (vi[ok] * side + vj[ok]).tolist()):
            key = (a << 32) | b
            if key in existing:
                continue
            existing.add(key)
            au[k], av[k] = a, b
            k += 1
            if k == na:
                break
    del_off = np.concatenate([[0], np.cumsum(del_sizes)]).astype(np.int64)
    add_off = np.concatenate([[0], np.cumsum(add_sizes)]).astype(np.int64)
    return UpdateStream(du, dv, au, av, del_off, add_off)


def write_graph_txt(path: str, g: Graph, weights: bool = True) -> None:
    """Write `u v [w]` lines (the reference's market_big format, weight
    (u+v)%128 as its --weight_num=1 synthesises it)."""
    src = np.repeat(np.arange(g.n, dtype=np.uint64), np.diff(g.xadj).astype(np.int64))
    dst = g.adj.astype(np.uint64)
    cols = [src, dst] + ([(src + dst) % 128] if weights else [])
    np.savetxt(path, np.stack(cols, axis=1), fmt="%d", delimiter=" ")


def write_updates_txt(update_path: str, size_path: str, ups: UpdateStream) -> None:
    """Write updates.txt (`d u v w` lines then `a u v w` lines per batch) and
    batches.txt (`adds dels` per batch), the reference's Loader format."""
    with open(update_path, "w") as f:
        for i in range(ups.batches):
            du, dv, au, av = ups.batch(i)
            for kind, us, vs in (("d", du, dv), ("a", au, av)):
                w = (us.astype(np.uint64) + vs.astype(np.uint64)) % 128
                f.writelines(f"{kind} {u} {v} {x}\n" for u, v, x in zip(us.tolist(), vs.tolist(), w.tolist()))
    with open(size_path, "w") as f:
        for i in range(ups.batches):
            f.write(f"{int(ups.add_off[i + 1] - ups.add_off[i])} {int(ups.del_off[i + 1] - ups.del_off[i])}\n")


def graph_from_edges(n: int, src, dst) -> Graph:
    """CSR from an edge list, rows in input (file) order, as the reference's
    market_big reader builds them (src/utils/parser.cpp:292-402)."""
    src = np.asarray(src, dtype=np.uint32)
    dst = np.asarray(dst, dtype=np.uint32)
    order = np.argsort(src, kind="stable")
    counts = np.bincount(src, minlength=n).astype(np.uint64)
    xadj = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(counts, out=xadj[1:])
    return Graph(n, xadj, dst[order].copy())
