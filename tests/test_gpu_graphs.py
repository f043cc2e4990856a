"""Batch-path CUDA graphs: a batch (or phase) shape seen twice is captured
once and replayed; results must be identical to direct launches and to the
oracle after every batch, through every driver (whole batches from host or
device arrays, the per-phase calls, the batched form), across shape changes,
position-index rebuilds (which retire the captured graphs) and with the
stage profiler on.
"""
import numpy as np
import pytest

import oracle
from coincgraph_b200 import Engine
from helpers import ORACLE_MODE, make_engine, rmat_case

pytestmark = pytest.mark.gpu


def _sizes_case(sizes, seed_offset, scale=11):
    """An R-MAT stream whose batch i has sizes[i] deletions and insertions."""
    from coincgraph_b200 import gen
    from helpers import Case

    g, h = gen.rmat(scale, keep_handle=True)
    ups = gen.updates(h, sizes, sizes, seed=gen.UPDATE_SEED_BASE + 400 + seed_offset)
    return Case(f"rmat{scale}", g.n, g.xadj, g.adj, [ups.batch(i) for i in range(len(sizes))], source=0)


def _oracle_values(og, algo, source):
    return og.cc() if algo == "cc" else og.sssp(source, ORACLE_MODE[algo])


def _stream(case, algo, monkeypatch, graphs, driver):
    monkeypatch.setenv("CIG_GRAPHS", "1" if graphs else "0")
    og = oracle.Graph(case.n, case.xadj, case.adj)
    out = []
    with make_engine(algo, source=case.source, cache_gib=4.0) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        for du, dv, au, av in case.batches:
            og.delete(du, dv)
            og.add(au, av)
            if driver == "host":
                replays = eng.apply_batch(du, dv, au, av)["graph_replays"]
            elif driver == "phases":
                replays = eng.delete_phase(du, dv)["graph_replays"]
                replays += eng.insert_phase(au, av)["graph_replays"]
            else:
                import torch

                t = [torch.from_numpy(x.astype(np.int32)).cuda() for x in (du, dv, au, av)]
                replays = eng.apply_batch_device(*t).graph_replays
            vals = eng.values()
            assert np.array_equal(vals, _oracle_values(og, algo, case.source))
            if algo != "cc":
                mode = ORACLE_MODE[algo]
                assert og.parent_check(vals, eng.parents(), case.source, mode)[0] == 0
            xadj, adj = eng.export_csr()
            xo, ao = og.export()
            assert np.array_equal(xadj, xo) and np.array_equal(adj, ao)
            out.append((eng.digest(), replays))
    return out


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
@pytest.mark.parametrize("driver", ["host", "phases", "device"])
def test_graph_replays_equal_direct_launches(algo, driver, monkeypatch):
    case = rmat_case(11, 5, 250, 250, seed_offset=40)
    on = _stream(case, algo, monkeypatch, True, driver)
    off = _stream(case, algo, monkeypatch, False, driver)
    assert [d for d, _ in on] == [d for d, _ in off]
    assert all(r == 0 for _, r in off)
    # first sighting direct, then captured and replayed on every later batch
    assert on[0][1] == 0 and all(r >= 1 for _, r in on[1:]), on


# A whole batch replays three graphs: key sort + deletion phase and the
# insertion phase (both keyed by the batch shape), then the segment-table
# service (one shape for every batch).
def test_shape_changes_replay_the_right_graph(monkeypatch):
    case = _sizes_case([100, 100, 130, 100, 130, 130, 7, 100], seed_offset=1)
    on = _stream(case, "sssp", monkeypatch, True, "host")
    off = _stream(case, "sssp", monkeypatch, False, "host")
    assert [d for d, _ in on] == [d for d, _ in off]
    assert [r for _, r in on] == [0, 3, 1, 3, 3, 3, 1, 3]


def test_index_rebuilds_retire_graphs(monkeypatch):
    """Position-index tables sized for almost no inserts: rebuilds come every
    few batches and must not leave a graph holding the old tables."""
    monkeypatch.setenv("CIG_POS_INDEX_CLS", "2")
    monkeypatch.setenv("CIG_POS_INDEX_HEADROOM", "64")
    monkeypatch.setenv("CIG_POS_INDEX_SPARE", "0")
    case = rmat_case(10, 8, 300, 300, seed_offset=41)
    on = _stream(case, "bfs", monkeypatch, True, "host")
    off = _stream(case, "bfs", monkeypatch, False, "host")
    assert [d for d, _ in on] == [d for d, _ in off]


def test_batched_form_with_graphs(monkeypatch):
    import torch

    case = _sizes_case([200, 200, 200, 50, 200, 50, 50], seed_offset=2)
    batches = [[torch.from_numpy(x.astype(np.int32)).cuda() for x in b] for b in case.batches]
    digests = {}
    for graphs in (True, False):
        monkeypatch.setenv("CIG_GRAPHS", "1" if graphs else "0")
        with Engine("sssp", cache_gib=4.0) as eng:
            eng.load_csr(case.n, case.xadj, case.adj)
            eng.init()
            stats, digests[graphs] = eng.apply_batches_device(batches)
            if graphs:
                assert [s.graph_replays for s in stats] == [0, 3, 3, 1, 3, 3, 3]
    assert digests[True] == digests[False]
    og = oracle.Graph(case.n, case.xadj, case.adj)
    for du, dv, au, av in case.batches:
        og.delete(du, dv)
        og.add(au, av)
    with Engine("sssp", cache_gib=4.0) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        eng.apply_batches_device(batches)
        assert np.array_equal(eng.values(), og.sssp(0, oracle.SSSP))


def test_stage_profile_under_graphs(monkeypatch):
    monkeypatch.setenv("CIG_GRAPHS", "1")
    case = rmat_case(11, 4, 300, 300, seed_offset=42)
    with Engine("sssp", cache_gib=4.0) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        eng.profile(True)
        replays = 0
        for b in case.batches:
            replays += eng.apply_batch(*b)["graph_replays"]
        prof = eng.profile_read()
    assert replays == 9
    for stage in ("group", "mutate", "inval", "pull", "push", "add", "cache"):
        assert prof[stage]["launches"] >= len(case.batches), (stage, prof[stage])
        assert prof[stage]["ms"] > 0, stage
