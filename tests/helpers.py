"""Shared test inputs: seeded R-MAT cases and hand-built adversarial cases.

The adversarial cases cover what the reference's chunk store and repair
paths handle (source_local_chunk_store.h:670-848 and the samples' deletion
rules): parallel edges and deleting one copy, repeated deletion requests,
missing deletes, out-of-range ids, self-loops, empty batches, deleting the
parent edge with and without a tight alternative, rows that outgrow their
block several times, and rows large enough for the block-wide paths
(> 4096 entries) and for multi-segment blocks (> 16384 entries).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from coincgraph_b200 import gen


@dataclass
class Case:
    name: str
    n: int
    xadj: np.ndarray
    adj: np.ndarray
    batches: list = field(default_factory=list)  # (du, dv, au, av) uint32 arrays
    source: int = 0


def _csr_from_edges(n, src, dst):
    g = gen.graph_from_edges(n, src, dst)
    return g.xadj, g.adj


def rmat_case(scale: int, batches: int, dels: int, adds: int, seed_offset: int = 0, symmetric=False) -> Case:
    g, h = gen.rmat(scale, keep_handle=True, symmetric=symmetric)
    ups = gen.updates(h, [dels] * batches, [adds] * batches, seed=gen.UPDATE_SEED_BASE + 100 + seed_offset,
                      symmetric=symmetric)
    return Case(f"rmat{scale}", g.n, g.xadj, g.adj, [ups.batch(i) for i in range(batches)], source=0)


def _u32(x):
    return np.asarray(x, dtype=np.uint32)


def adversarial_case() -> Case:
    rng = np.random.default_rng(20240611)
    n = 64
    src, dst = [], []
    # a path with a tight alternative and a weak one
    for a, b in [(0, 1), (1, 2), (2, 3), (3, 4), (0, 5), (5, 2), (0, 6), (6, 3), (4, 7), (7, 8)]:
        src.append(a)
        dst.append(b)
    # parallel edges
    for _ in range(3):
        src.append(0)
        dst.append(9)
    src += [9, 9, 10, 11, 12, 12]
    dst += [10, 10, 11, 12, 13, 13]
    # self loops
    src += [13, 14]
    dst += [13, 14]
    # equal-label cycle for CC (20 -> 21 -> 22 -> 20, fed from 15)
    src += [15, 20, 21, 22]
    dst += [20, 21, 22, 20]
    # random filler
    for _ in range(200):
        a, b = rng.integers(0, n, 2)
        src.append(int(a))
        dst.append(int(b))
    xadj, adj = _csr_from_edges(n, src, dst)
    batches = [
        # delete one copy of a parallel edge, a missing edge and an out-of-range id
        (_u32([0, 40, 70]), _u32([9, 41, 1]), _u32([]), _u32([])),
        # empty batch
        (_u32([]), _u32([]), _u32([]), _u32([])),
        # delete the tree path and the parent edge of 2, repeated requests
        (_u32([1, 1, 0, 9, 9, 9]), _u32([2, 2, 1, 10, 10, 10]), _u32([30, 31, 32, 99]), _u32([31, 32, 2, 3])),
        # break the equal-label cycle feed, re-add parallel edges, grow row 30 through several classes
        (_u32([15, 20]), _u32([20, 21]), _u32([30] * 40 + [0, 0]), _u32(list(range(1, 41)) + [9, 9])),
        # insert only
        (_u32([]), _u32([]), _u32([4, 8, 63]), _u32([63, 0, 1])),
    ]
    return Case("adversarial", n, xadj, adj, batches, source=0)


def big_row_case() -> Case:
    """Rows above the warp path (5000 entries) and above one segment (20000)."""
    rng = np.random.default_rng(7)
    n = 30000
    # vertex 5 has 6000 in-edges and its parent edge (0, 5) is deleted in
    # batch 0, so the pull repair meets an in-row above the split threshold
    src = np.concatenate([np.zeros(20000, np.int64), np.ones(5000, np.int64), rng.integers(0, n, 30000),
                          np.arange(100, 6100), [0]])
    dst = np.concatenate([rng.integers(6, n, 20000), rng.integers(2, n, 5000), rng.integers(0, n, 30000),
                          np.full(6000, 5), [5]])
    xadj, adj = _csr_from_edges(n, src, dst)
    row0 = adj[int(xadj[0]):int(xadj[1])]
    row1 = adj[int(xadj[1]):int(xadj[2])]
    batches = []
    for k in range(3):
        pick0 = row0[rng.integers(0, len(row0), 50)]
        pick1 = row1[rng.integers(0, len(row1), 20)]
        extra = 1 if k == 0 else 0
        du = np.concatenate([np.zeros(50, np.uint32), np.ones(20, np.uint32), rng.integers(0, n, 30).astype(np.uint32),
                             np.zeros(extra, np.uint32)])
        dv = np.concatenate([pick0, pick1, rng.integers(0, n, 30), np.full(extra, 5)]).astype(np.uint32)
        # batch 1 pushes row 0 past its 32768-slot block and row 1 past 8192
        au = np.concatenate([np.zeros(13000 * (k == 1), np.uint32), np.ones(4000 * (k == 1), np.uint32),
                             rng.integers(0, n, 100).astype(np.uint32)])
        av = rng.integers(0, n, len(au)).astype(np.uint32)
        batches.append((du, dv, au, av))
    return Case("bigrow", n, xadj, adj, batches, source=0)


def heavy_delete_case() -> Case:
    """Many deletion keys in one row: a 3000-entry row losing 200 entries
    (more than a warp's 32 key registers) and a 12000-entry row losing 3000
    (more than the block path's 2048 shared-memory keys), with parallel edges
    and repeated requests."""
    rng = np.random.default_rng(11)
    n = 9000
    src = np.concatenate([np.full(3000, 0), np.full(12000, 1), rng.integers(0, n, 20000)])
    dst = np.concatenate([rng.integers(2, 400, 3000), rng.integers(2, n, 12000), rng.integers(0, n, 20000)])
    xadj, adj = _csr_from_edges(n, src, dst)
    row0 = adj[int(xadj[0]):int(xadj[1])]
    row1 = adj[int(xadj[1]):int(xadj[2])]
    batches = []
    for k in range(2):
        d0 = row0[rng.integers(0, len(row0), 200)]
        d1 = row1[rng.integers(0, len(row1), 3000)]
        du = np.concatenate([np.zeros(200, np.uint32), np.ones(3000, np.uint32)])
        dv = np.concatenate([d0, d1]).astype(np.uint32)
        au = rng.integers(0, n, 500).astype(np.uint32)
        av = rng.integers(0, n, 500).astype(np.uint32)
        batches.append((du, dv, au, av))
    return Case("heavydelete", n, xadj, adj, batches, source=0)


def grid_case(side: int = 48, batches: int = 3, size: int = 150) -> Case:
    """Road-like high-diameter case: a side x side grid, local insertions."""
    g = gen.grid(side)
    ups = gen.local_updates(g, side, [size] * batches, [size] * batches, seed=gen.UPDATE_SEED_BASE + 300)
    return Case(f"grid{side}", g.n, g.xadj, g.adj, [ups.batch(i) for i in range(batches)], source=0)


ORACLE_MODE = {"bfs": 0, "sssp": 1, "cc": 2, "sssp_u255": 3}


def make_engine(algo: str, **kw):
    """Engine for a test algorithm name; "sssp_u255" is SSSP with the
    uniform [1, 255] edge weights (CIG_FLAG_WEIGHT_U255)."""
    from coincgraph_b200 import Engine
    from coincgraph_b200.engine import FLAG_WEIGHT_U255

    if algo == "sssp_u255":
        return Engine("sssp", flags=kw.pop("flags", 0) | FLAG_WEIGHT_U255, **kw)
    return Engine(algo, **kw)


def oracle_trace(case: Case, algo: str):
    """Replay the case on the oracle: per batch the values after the deletion
    phase and after the batch, and the rows after the batch."""
    import oracle

    g = oracle.Graph(case.n, case.xadj, case.adj)
    mode = ORACLE_MODE.get(algo)

    def values():
        if algo == "cc":
            return g.cc()
        return g.sssp(case.source, mode)

    out = {"init": values(), "delete": [], "batch": [], "rows": []}
    for du, dv, au, av in case.batches:
        g.delete(du, dv)
        out["delete"].append(values())
        g.add(au, av)
        out["batch"].append(values())
        out["rows"].append(g.export())
    return out, g
