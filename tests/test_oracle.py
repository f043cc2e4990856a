"""The CPU oracle against the reference's own code and the golden fixtures.

Pins (see oracle/__init__.py): the oracle's row mutation against the
reference SourceLocalChunkStore compiled from its sources, its CC labels
against the reference CCCheck, its PageRank against the reference
PageRankCheck, and its BFS/SSSP distances against an independent algorithm
and the Bellman certificate.
"""
import os

import numpy as np
import pytest

import oracle
from helpers import adversarial_case, big_row_case, heavy_delete_case, rmat_case

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (no reference tree)")


def _rows_equal(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@needs_ref
@pytest.mark.parametrize("make", [adversarial_case, big_row_case, heavy_delete_case,
                                  lambda: rmat_case(10, 5, 80, 80, seed_offset=3)])
def test_rows_match_reference_store(built, make):
    case = make()
    g = oracle.Graph(case.n, case.xadj, case.adj)
    ref = oracle.RefStore(case.n, case.xadj, case.adj)
    for du, dv, au, av in case.batches:
        missing = g.delete(du, dv)
        g.add(au, av)
        counts = ref.apply(du, dv, au, av)
        assert counts["missing_deletes"] == missing
        assert _rows_equal(g.export(), ref.export())
        assert g.m == ref.m


@needs_ref
def test_random_multiset_deletions_match_reference(built):
    """Heavy duplicates: repeated destinations in rows and repeated requests."""
    rng = np.random.default_rng(5)
    n = 40
    src = rng.integers(0, n, 600)
    dst = rng.integers(0, 6, 600)  # few distinct destinations -> many parallel edges
    from coincgraph_b200 import gen

    csr = gen.graph_from_edges(n, src, dst)
    g = oracle.Graph(n, csr.xadj, csr.adj)
    ref = oracle.RefStore(n, csr.xadj, csr.adj)
    for _ in range(6):
        du = rng.integers(0, n + 2, 150).astype(np.uint32)
        dv = rng.integers(0, 7, 150).astype(np.uint32)
        au = rng.integers(0, n, 80).astype(np.uint32)
        av = rng.integers(0, 6, 80).astype(np.uint32)
        assert g.delete(du, dv) == ref.apply(du, dv, [], [])["missing_deletes"]
        g.add(au, av)
        ref.apply([], [], au, av)
        assert _rows_equal(g.export(), ref.export())


@needs_ref
def test_cc_matches_reference_checker(built):
    case = rmat_case(10, 3, 100, 100, seed_offset=4)
    g = oracle.Graph(case.n, case.xadj, case.adj)
    ref = oracle.RefStore(case.n, case.xadj, case.adj)
    assert ref.cc_errors(g.cc()) == 0
    for du, dv, au, av in case.batches:
        g.delete(du, dv)
        g.add(au, av)
        ref.apply(du, dv, au, av)
        labels = g.cc()
        assert ref.cc_errors(labels) == 0
        bad = labels.copy()
        bad[np.argmax(labels)] = 0 if labels.max() > 0 else 1
        assert ref.cc_errors(bad) > 0  # the checker does reject a wrong label


@needs_ref
def test_pagerank_passes_reference_checker(built):
    case = rmat_case(9, 1, 10, 10, seed_offset=5)
    g = oracle.Graph(case.n, case.xadj, case.adj)
    ref = oracle.RefStore(case.n, case.xadj, case.adj)
    x, ok = g.pagerank(1e-14, 50000)
    assert ok
    xa, aa = g.export()
    nxt = np.full(case.n, 0.15)
    deg = np.diff(xa)
    xf = x.astype(np.float32).astype(np.float64)
    for s in range(case.n):
        if deg[s]:
            np.add.at(nxt, aa[int(xa[s]):int(xa[s + 1])], 0.85 * xf[s] / deg[s])
    residual = (nxt - xf).astype(np.float32)
    assert ref.pr_check(x.astype(np.float32), residual, 1e-6)
    restated = g.pr_check(x.astype(np.float32), residual, 1e-6)
    assert restated["ok"] == 1.0
    # a rank that is clearly off fails both
    bad = x.astype(np.float32).copy()
    bad[0] += 0.5
    assert not ref.pr_check(bad, residual, 1e-6)
    assert g.pr_check(bad, residual, 1e-6)["ok"] == 0.0


@pytest.mark.parametrize("mode", [oracle.BFS, oracle.SSSP, oracle.SSSP_U255])
def test_two_sssp_oracles_agree(built, mode):
    case = rmat_case(11, 2, 200, 200, seed_offset=6)
    g = oracle.Graph(case.n, case.xadj, case.adj)
    for du, dv, au, av in case.batches:
        g.delete(du, dv)
        g.add(au, av)
        d, p = g.sssp(case.source, mode, parents=True)
        assert np.array_equal(d, g.sssp_dial(case.source, mode))
        assert g.bellman_check(d, case.source, mode) == (0, 0)
        assert g.parent_check(d, p, case.source, mode)[0] == 0
        wrong = d.copy()
        finite = np.flatnonzero((wrong != oracle.INF) & (np.arange(case.n) != case.source))
        wrong[finite[0]] += 1
        assert g.bellman_check(wrong, case.source, mode) != (0, 0)


@pytest.mark.parametrize("name", ["rmat8", "adversarial"])
def test_golden_fixtures(built, name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    n, src = int(z["n"]), int(z["source"])
    g = oracle.Graph(n, z["xadj"], z["adj"])

    def check(tag):
        assert np.array_equal(g.sssp(src, oracle.BFS), z[f"{tag}_bfs"])
        assert np.array_equal(g.sssp(src, oracle.SSSP), z[f"{tag}_sssp"])
        assert np.array_equal(g.cc(), z[f"{tag}_cc"])

    check("init")
    for i in range(int(z["nbatches"])):
        assert g.delete(z[f"b{i}_du"], z[f"b{i}_dv"]) == int(z[f"b{i}_missing"])
        check(f"b{i}_del")
        assert g.add(z[f"b{i}_au"], z[f"b{i}_av"]) == int(z[f"b{i}_invalid"])
        xadj, adj = g.export()
        assert np.array_equal(xadj, z[f"b{i}_xadj"]) and np.array_equal(adj, z[f"b{i}_adj"])
        check(f"b{i}_ins")
    x, ok = g.pagerank(1e-14, 50000)
    assert ok and np.allclose(x, z["final_pr"], rtol=1e-12, atol=0)


def test_checksum_restates_reference_formula(built):
    vals = np.array([0, 5, oracle.INF, 7], dtype=np.uint32)
    h = 1469598103934665603
    mask = (1 << 64) - 1
    for v, d in enumerate(vals.tolist()):
        if d == oracle.INF:
            continue
        h ^= (v + 0x9E3779B97F4A7C15 + (d << 6) + (d >> 2)) & mask
        h = (h * 1099511628211) & mask
    assert oracle.checksum(vals) == h


def test_uniform_255_weights_cover_the_range(built):
    """The extension's weight function spans [1, 255] about evenly."""
    import ctypes

    lib = oracle.lib()
    lib.og_weight.restype = ctypes.c_uint32
    lib.og_weight.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
    w = np.array([lib.og_weight(oracle.SSSP_U255, u, v) for u in range(60) for v in range(60)])
    assert w.min() == 1 and w.max() == 255
    counts = np.bincount(w, minlength=256)[1:]
    assert counts.min() > 0 and counts.max() < 4 * counts.mean()
