"""Multi-source BFS / SSSP queries (bitmask waves) against the CPU oracle.

Each row of a query result must equal the oracle's from-scratch FIFO
recompute for that source (the restated hybrid_sssp_host.cu:34-63 check with
the samples' weights), exactly, on the graph as it stands after update
batches; the batched (64-wide) and per-source (width 1) forms must agree.
"""
import numpy as np
import pytest

import oracle
from coincgraph_b200 import Engine, gen

from helpers import big_row_case, rmat_case

pytestmark = pytest.mark.gpu

MODES = {"bfs": oracle.BFS, "sssp": oracle.SSSP}


def _sources(g, k, seed=7):
    rng = np.random.default_rng(seed)
    deg = np.diff(g.xadj.astype(np.int64))
    live = np.flatnonzero(deg > 0)
    hub = int(np.argmax(deg))
    picks = rng.choice(live, size=k - 3, replace=True)
    return np.concatenate([[0, hub, hub], picks]).astype(np.uint32)  # a repeated source too


@pytest.mark.parametrize("algo", ["bfs", "sssp"])
@pytest.mark.parametrize("k", [1, 5, 64, 70])
def test_query_matches_oracle(built, algo, k):
    g = gen.rmat(11)
    src = _sources(g, max(k, 4))[:k]
    og = oracle.Graph(g.n, g.xadj, g.adj)
    with Engine(algo, cache_gib=4.0) as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        got = eng.query_bfs(src) if algo == "bfs" else eng.query_sssp(src)
    assert got.shape == (k, g.n)
    for j, s in enumerate(src):
        np.testing.assert_array_equal(got[j], og.sssp(int(s), MODES[algo]), err_msg=f"source {s}")


@pytest.mark.parametrize("cache_gib", [0.0, 0.002])
def test_query_after_updates_zero_copy_and_mixed(built, cache_gib):
    case = rmat_case(12, batches=2, dels=300, adds=300)
    og = oracle.Graph(case.n, case.xadj, case.adj)
    with Engine("sssp", cache_gib=cache_gib) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        for du, dv, au, av in case.batches:
            eng.apply_batch(du, dv, au, av)
            og.delete(du, dv)
            og.add(au, av)
        src = _sources(gen.Graph(case.n, *og.export()), 40)
        bfs = eng.query_bfs(src)
        sssp = eng.query_sssp(src)
        # Queries leave the maintained state alone.
        np.testing.assert_array_equal(eng.values(), og.sssp(0, oracle.SSSP))
    for j, s in enumerate(src):
        np.testing.assert_array_equal(bfs[j], og.sssp(int(s), oracle.BFS))
        np.testing.assert_array_equal(sssp[j], og.sssp(int(s), oracle.SSSP))


def test_query_hub_rows_and_width_forms(built):
    """Rows past the hub-split threshold (deferred grid-wide expansion) and the
    device-output form at widths 64 and 1 give the same distances."""
    import torch

    case = big_row_case()
    og = oracle.Graph(case.n, case.xadj, case.adj)
    src = np.arange(0, min(case.n, 48), dtype=np.uint32)
    with Engine("bfs", cache_gib=1.0) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        outs = {}
        for width in (64, 1):
            out = torch.empty((len(src), case.n), dtype=torch.int32, device="cuda")
            st = eng.query_device("sssp", src, out, width=width)
            assert st["waves"] == -(-len(src) // width)
            assert st["edges_scanned"] > 0 and st["source_edges"] >= st["edges_scanned"]
            outs[width] = out.cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(outs[64], outs[1])
    for j, s in enumerate(src):
        np.testing.assert_array_equal(outs[64][j], og.sssp(int(s), oracle.SSSP))


def test_query_sssp_uniform_255_weights(built):
    from coincgraph_b200.engine import FLAG_WEIGHT_U255

    g = gen.rmat(11)
    src = _sources(g, 20)
    og = oracle.Graph(g.n, g.xadj, g.adj)
    with Engine("sssp", cache_gib=1.0, flags=FLAG_WEIGHT_U255) as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        got = eng.query_sssp(src)
        np.testing.assert_array_equal(eng.values(), og.sssp(0, oracle.SSSP_U255))
    for j, s in enumerate(src):
        np.testing.assert_array_equal(got[j], og.sssp(int(s), oracle.SSSP_U255))


def test_query_rejects_bad_arguments(built):
    from coincgraph_b200 import CigError

    g = gen.rmat(8)
    with Engine("bfs") as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        with pytest.raises(CigError):
            eng.query_bfs(np.array([g.n], dtype=np.uint32))
        # The handle stays usable after a rejected call.
        np.testing.assert_array_equal(eng.query_bfs([0])[0], eng.values())
