"""GPU parity on the benchmark configurations themselves (not toy sizes).

- Plain incremental BFS (the reference's hybrid_bfs flow): R-MAT scale 16,
  edge factor 16, seeded as the generator defines it, BFS from source 0,
  `--cache=2` (all resident), 10 batches of 1,000 deletions sampled from the
  current edges + 1,000 insertions of new pairs.  Depths bit-exact against
  the oracle after every deletion phase and every batch, parents checked as
  witnesses, rows equal to the oracle's after every batch.
- Multi-source BFS + CC on a symmetric graph (the shape of the 64-source
  workload at reduced scale): symmetric R-MAT scale 17, batches of
  log-uniform sizes, half deletions and half insertions; CC labels
  bit-exact after every batch, and 64 BFS sources (uniform over vertices of
  degree > 0) answered as one bitmask wave, equal to the oracle's per-source
  BFS and to the plain per-source form (wave width 1).
- Incremental SSSP on a larger-than-cache graph (slow): R-MAT scale 24
  (16.8 M vertices, 263 M edges), `--cache=1` GiB so that a third of the
  adjacency is read zero-copy from host memory, default position index, 2
  batches of 100k deletions + 100k insertions; distances bit-exact after
  each phase, rows equal at the end.  This is the benchmark's own workload.
"""
import numpy as np
import pytest

import oracle
from coincgraph_b200 import Engine, gen

pytestmark = pytest.mark.gpu


def _check_phase(eng, og, source, mode, where):
    got = eng.values()
    want = og.sssp(source, mode)
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, f"values differ {where}: {bad[:10]} ({bad.size} vertices)"
    assert og.bellman_check(got, source, mode) == (0, 0), where
    assert og.parent_check(got, eng.parents(), source, mode)[0] == 0, f"bad parent witness {where}"


def test_plain_bfs_rmat16_cache2_10x1000():
    g, h = gen.rmat(16, 16, keep_handle=True)
    ups = gen.updates(h, [1000] * 10, [1000] * 10, seed=gen.UPDATE_SEED_BASE + 1)
    og = oracle.Graph(g.n, g.xadj, g.adj)
    with Engine("bfs", source=0, cache_gib=2.0) as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        info = eng.info()
        used = info["arena_used_edges"] // info["segment_edges"]
        assert info["segments_resident"] == used, "cache 2 GiB holds the whole graph"
        eng.init()
        _check_phase(eng, og, 0, oracle.BFS, "after init")
        for i in range(ups.batches):
            du, dv, au, av = ups.batch(i)
            missing = og.delete(du, dv)
            s = eng.delete_phase(du, dv)
            assert s["missing_deletes"] == missing == 0
            _check_phase(eng, og, 0, oracle.BFS, f"after deletion phase {i}")
            invalid = og.add(au, av)
            s = eng.insert_phase(au, av)
            assert s["invalid_additions"] == invalid == 0
            _check_phase(eng, og, 0, oracle.BFS, f"after batch {i}")
            xadj, adj = eng.export_csr()
            xo, ao = og.export()
            assert np.array_equal(xadj, xo) and np.array_equal(adj, ao), f"rows differ after batch {i}"


def test_symmetric_cc_and_64_source_bfs_uneven_batches():
    scale = 17
    g, h = gen.rmat(scale, 16, symmetric=True, keep_handle=True)
    rng = np.random.default_rng(0xC01C1003)
    sizes = np.exp(rng.uniform(np.log(500), np.log(40000), size=6)).astype(np.int64)
    # symmetric updates come in (u, v) + (v, u) pairs: even sizes
    sizes = (sizes // 2) * 2
    ups = gen.updates(h, sizes, sizes, seed=gen.UPDATE_SEED_BASE + 3, symmetric=True)
    og = oracle.Graph(g.n, g.xadj, g.adj)
    with Engine("cc", cache_gib=4.0) as cc:
        cc.load_csr(g.n, g.xadj, g.adj)
        cc.init()
        assert np.array_equal(cc.values(), og.cc())
        for i in range(ups.batches):
            du, dv, au, av = ups.batch(i)
            og.delete(du, dv)
            og.add(au, av)
            cc.apply_batch(du, dv, au, av)
            assert np.array_equal(cc.values(), og.cc()), f"CC labels differ after batch {i}"
        xadj, adj = cc.export_csr()
    deg = np.diff(xadj.astype(np.int64))
    sources = rng.choice(np.flatnonzero(deg > 0), size=64, replace=False).astype(np.uint32)
    import torch

    with Engine("bfs", source=int(sources[0]), cache_gib=4.0) as q:
        q.load_csr(g.n, xadj, adj)
        out64 = torch.empty((64, g.n), dtype=torch.int32, device="cuda")
        out1 = torch.empty((64, g.n), dtype=torch.int32, device="cuda")
        q.query_device("bfs", sources, out64, width=64)
        q.query_device("bfs", sources, out1, width=1)
        wave = out64.cpu().numpy().view(np.uint32)
        plain = out1.cpu().numpy().view(np.uint32)
    assert np.array_equal(wave, plain), "64-wide wave differs from the per-source form"
    og2 = oracle.Graph(g.n, xadj, adj)
    for k, s in enumerate(sources.tolist()):
        assert np.array_equal(wave[k], og2.sssp(s, oracle.BFS)), f"source {s}: depths differ from the oracle"


@pytest.mark.slow
def test_sssp_rmat24_cache1g_two_batches():
    g, h = gen.rmat(24, 16, keep_handle=True)
    ups = gen.updates(h, [100_000] * 2, [100_000] * 2, seed=gen.UPDATE_SEED_BASE + 2)
    del h
    og = oracle.Graph(g.n, g.xadj, g.adj)
    with Engine("sssp", source=0, cache_gib=1.0, max_batch=100_000) as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        info = eng.info()
        used = info["arena_used_edges"] // info["segment_edges"]
        assert info["segments_resident"] < used, "1 GiB must not hold the whole graph"
        eng.init()
        _check_phase(eng, og, 0, oracle.SSSP, "after init")
        for i in range(ups.batches):
            du, dv, au, av = ups.batch(i)
            missing = og.delete(du, dv)
            s = eng.delete_phase(du, dv)
            assert s["missing_deletes"] == missing
            _check_phase(eng, og, 0, oracle.SSSP, f"after deletion phase {i}")
            invalid = og.add(au, av)
            s = eng.insert_phase(au, av)
            assert s["invalid_additions"] == invalid
            _check_phase(eng, og, 0, oracle.SSSP, f"after batch {i}")
        xadj, adj = eng.export_csr()
    xo, ao = og.export()
    assert np.array_equal(xadj, xo), "row lengths differ"
    assert np.array_equal(adj, ao), "rows differ"
