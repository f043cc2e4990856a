"""Seeded generator: determinism and the stated properties of its output."""
import numpy as np

from coincgraph_b200 import gen


def test_rmat_deterministic_and_clean(built):
    a = gen.rmat(10)
    b = gen.rmat(10)
    assert np.array_equal(a.xadj, b.xadj) and np.array_equal(a.adj, b.adj)
    assert a.n == 1024
    src = np.repeat(np.arange(a.n, dtype=np.uint64), np.diff(a.xadj).astype(np.int64))
    keys = (src << np.uint64(32)) | a.adj.astype(np.uint64)
    assert len(np.unique(keys)) == len(keys)  # no duplicates
    assert not np.any(src == a.adj)  # no self-loops
    for v in range(0, a.n, 97):
        row = a.adj[int(a.xadj[v]):int(a.xadj[v + 1])]
        assert np.all(np.diff(row.astype(np.int64)) > 0)  # rows sorted
    # id 0 stays the R-MAT hub
    assert np.argmax(np.diff(a.xadj)) == 0


def test_symmetric_graph(built):
    g = gen.rmat(9, symmetric=True)
    src = np.repeat(np.arange(g.n, dtype=np.uint64), np.diff(g.xadj).astype(np.int64))
    fwd = set(((src << np.uint64(32)) | g.adj.astype(np.uint64)).tolist())
    rev = set(((g.adj.astype(np.uint64) << np.uint64(32)) | src).tolist())
    assert fwd == rev


def test_update_stream_validity(built):
    g, h = gen.rmat(9, keep_handle=True)
    ups = gen.updates(h, [50, 50, 50], [40, 40, 40], seed=gen.UPDATE_SEED_BASE + 7)
    src = np.repeat(np.arange(g.n, dtype=np.uint64), np.diff(g.xadj).astype(np.int64))
    cur = set(((src << np.uint64(32)) | g.adj.astype(np.uint64)).tolist())
    for i in range(ups.batches):
        du, dv, au, av = ups.batch(i)
        for u, v in zip(du.tolist(), dv.tolist()):
            assert (u << 32 | v) in cur  # deletions come from the current edge set
            cur.remove(u << 32 | v)  # without replacement
        for u, v in zip(au.tolist(), av.tolist()):
            assert u != v and (u << 32 | v) not in cur  # insertions are new pairs
            cur.add(u << 32 | v)
    again = gen.updates(h, [50, 50, 50], [40, 40, 40], seed=gen.UPDATE_SEED_BASE + 7)
    assert np.array_equal(ups.del_v, again.del_v) and np.array_equal(ups.add_u, again.add_u)


def test_grid_and_local_updates():
    """Road-like grid: 4-neighbour rows in east/west/south/north order; update
    batches delete existing distinct edges and insert new local pairs only."""
    side = 16
    g = gen.grid(side)
    assert g.n == side * side and g.m == 4 * side * (side - 1)
    row = lambda v: g.adj[int(g.xadj[v]):int(g.xadj[v + 1])].tolist()
    assert row(0) == [1, side]
    assert row(side + 1) == [side + 2, side, 2 * side + 1, 1]
    ups = gen.local_updates(g, side, [20, 20], [30, 30], seed=5)
    edges = set(zip(np.repeat(np.arange(g.n), np.diff(g.xadj.astype(np.int64))).tolist(), g.adj.tolist()))
    dels = list(zip(ups.del_u.tolist(), ups.del_v.tolist()))
    adds = list(zip(ups.add_u.tolist(), ups.add_v.tolist()))
    assert len(set(dels)) == len(dels) == 40 and all(e in edges for e in dels)
    assert len(set(adds)) == len(adds) == 60 and not any(e in edges for e in adds)
    for u, v in adds:
        assert u != v and abs(u // side - v // side) <= 3 and abs(u % side - v % side) <= 3
    again = gen.local_updates(g, side, [20, 20], [30, 30], seed=5)
    assert np.array_equal(again.add_v, ups.add_v) and np.array_equal(again.del_u, ups.del_u)


def test_bench_road_workload_shapes():
    """bench.py's road workload: a grid of --side^2 vertices and batches of
    --batch deletions and insertions (built on the host, no GPU needed)."""
    import argparse
    import importlib.util
    import os

    spec = importlib.util.spec_from_file_location(
        "bench_mod", os.path.join(os.path.dirname(__file__), "..", "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    args = argparse.Namespace(workload="road", side=20, batch=15, scale=24, edge_factor=16)
    g, ups, setup = bench.make_workload(args, 3)
    assert g.n == 400 and ups.batches == 3 and set(setup) == {"gen_graph_s", "gen_updates_s"}
    for i in range(3):
        du, dv, au, av = ups.batch(i)
        assert len(du) == len(dv) == len(au) == len(av) == 15
