"""GPU parity: the sm_100a engine (through the C ABI) against the oracle.

Bar: BFS depths, SSSP distances and CC labels bit-exact after the deletion
phase and after every batch; parents checked as witnesses (they are not
unique: samples/hybrid_bfs/README.md:7-9); rows equal to the oracle's (and so
to the reference chunk store's) element for element; missing/invalid counts
equal.  Cache budgets cover all-resident, mixed residency and zero-copy only.
"""
import os

import numpy as np
import pytest

import oracle
from coincgraph_b200 import Engine
from helpers import (ORACLE_MODE, adversarial_case, big_row_case, grid_case, heavy_delete_case, make_engine,
                     oracle_trace, rmat_case)

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ONE_SEGMENT_GIB = 65536 / 2**30  # one 64 KiB cache slot
CACHES = {"resident": 4.0, "mixed": ONE_SEGMENT_GIB, "zerocopy": 0.0}


def _check_values(eng, g, case, algo, expect, where):
    got = eng.values()
    assert np.array_equal(got, expect), f"{algo} values differ {where}: {np.flatnonzero(got != expect)[:10]}"
    if algo != "cc":
        mode = ORACLE_MODE[algo]
        assert g.bellman_check(got, case.source, mode) == (0, 0)
        assert g.parent_check(got, eng.parents(), case.source, mode)[0] == 0, f"bad parent witness {where}"


def run_case(case, algo, cache_gib):
    trace, _ = oracle_trace(case, algo)
    g = oracle.Graph(case.n, case.xadj, case.adj)
    with make_engine(algo, source=case.source, cache_gib=cache_gib) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        _check_values(eng, g, case, algo, trace["init"], "after init")
        for i, (du, dv, au, av) in enumerate(case.batches):
            missing = g.delete(du, dv)
            s = eng.delete_phase(du, dv)
            assert s["missing_deletes"] == missing
            _check_values(eng, g, case, algo, trace["delete"][i], f"after delete phase {i}")
            invalid = g.add(au, av)
            s = eng.insert_phase(au, av)
            assert s["invalid_additions"] == invalid
            _check_values(eng, g, case, algo, trace["batch"][i], f"after batch {i}")
            xadj, adj = eng.export_csr()
            assert np.array_equal(xadj, trace["rows"][i][0]) and np.array_equal(adj, trace["rows"][i][1])


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
@pytest.mark.parametrize("cache", list(CACHES))
def test_rmat_stream(algo, cache):
    run_case(rmat_case(11, 4, 300, 300, seed_offset=10), algo, CACHES[cache])


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_adversarial(algo):
    run_case(adversarial_case(), algo, 4.0)


@pytest.mark.parametrize("algo", ["sssp", "cc"])
@pytest.mark.parametrize("cache", ["resident", "mixed"])
def test_big_rows(algo, cache):
    run_case(big_row_case(), algo, CACHES[cache])


@pytest.mark.parametrize("algo", ["sssp", "cc"])
@pytest.mark.parametrize("cache", ["resident", "zerocopy"])
def test_heavy_deletions(algo, cache):
    run_case(heavy_delete_case(), algo, CACHES[cache])


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_symmetric_stream(algo):
    run_case(rmat_case(10, 3, 200, 200, seed_offset=11, symmetric=True), algo, 4.0)


@pytest.mark.parametrize("name", ["rmat8", "adversarial"])
@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_golden(name, algo):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    n, src = int(z["n"]), int(z["source"])
    with Engine(algo, source=src, cache_gib=4.0) as eng:
        eng.load_csr(n, z["xadj"], z["adj"])
        eng.init()
        assert np.array_equal(eng.values(), z[f"init_{algo}"])
        for i in range(int(z["nbatches"])):
            s = eng.delete_phase(z[f"b{i}_du"], z[f"b{i}_dv"])
            assert s["missing_deletes"] == int(z[f"b{i}_missing"])
            assert np.array_equal(eng.values(), z[f"b{i}_del_{algo}"])
            s = eng.insert_phase(z[f"b{i}_au"], z[f"b{i}_av"])
            assert s["invalid_additions"] == int(z[f"b{i}_invalid"])
            assert np.array_equal(eng.values(), z[f"b{i}_ins_{algo}"])
            xadj, adj = eng.export_csr()
            assert np.array_equal(xadj, z[f"b{i}_xadj"]) and np.array_equal(adj, z[f"b{i}_adj"])


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_whole_batch_equals_phases(algo):
    """cig_apply_batch (one sync) gives the same state as the two phase calls."""
    case = rmat_case(10, 3, 150, 150, seed_offset=12)
    with Engine(algo, cache_gib=4.0) as a, Engine(algo, cache_gib=4.0) as b:
        for e in (a, b):
            e.load_csr(case.n, case.xadj, case.adj)
            e.init()
        for du, dv, au, av in case.batches:
            a.apply_batch(du, dv, au, av)
            b.delete_phase(du, dv)
            b.insert_phase(au, av)
            assert np.array_equal(a.values(), b.values())
            assert a.digest() == b.digest()


def run_case_whole_batches(case, algo, cache_gib):
    """Batches through cig_apply_batch (one key sort for the whole batch and
    the per-batch segment-table service); values and rows after every batch."""
    trace, _ = oracle_trace(case, algo)
    g = oracle.Graph(case.n, case.xadj, case.adj)
    stats = []
    with make_engine(algo, source=case.source, cache_gib=cache_gib) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        for i, (du, dv, au, av) in enumerate(case.batches):
            missing = g.delete(du, dv)
            invalid = g.add(au, av)
            s = eng.apply_batch(du, dv, au, av)
            assert s["missing_deletes"] == missing and s["invalid_additions"] == invalid
            stats.append(s)
            _check_values(eng, g, case, algo, trace["batch"][i], f"after batch {i}")
            xadj, adj = eng.export_csr()
            assert np.array_equal(xadj, trace["rows"][i][0]) and np.array_equal(adj, trace["rows"][i][1])
    return stats


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
@pytest.mark.parametrize("cache", list(CACHES))
def test_rmat_stream_whole_batches(algo, cache):
    run_case_whole_batches(rmat_case(11, 4, 300, 300, seed_offset=14), algo, CACHES[cache])


@pytest.mark.parametrize("cache", ["resident", "mixed"])
def test_uniform_255_weights(cache):
    """The [1, 255] weight extension against the oracle's same weights."""
    run_case(rmat_case(11, 3, 300, 300, seed_offset=16), "sssp_u255", CACHES[cache])
    run_case_whole_batches(heavy_delete_case(), "sssp_u255", CACHES[cache])


@pytest.mark.parametrize("algo", ["sssp", "cc"])
def test_adversarial_and_big_rows_whole_batches(algo):
    run_case_whole_batches(adversarial_case(), algo, CACHES["mixed"])
    run_case_whole_batches(big_row_case(), algo, CACHES["mixed"])


@pytest.mark.parametrize("algo", ["bfs", "sssp"])
def test_segment_table_churn(algo, monkeypatch):
    """Every segment counts as cold and every touched host segment as hot, so
    each batch evicts (writing dirty segments back) and admits segments; the
    results and rows must not change."""
    monkeypatch.setenv("CIG_CACHE_ADMIT_SCORE", "1")
    monkeypatch.setenv("CIG_CACHE_COLD_SCORE", str(1 << 30))
    stats = run_case_whole_batches(rmat_case(14, 6, 2000, 2000, seed_offset=15), algo, 8 * ONE_SEGMENT_GIB)
    assert sum(s["cache_segments_evicted"] for s in stats) > 0
    assert sum(s["cache_segments_loaded"] for s in stats) > 0


@pytest.mark.parametrize("small_pct", [None, 0, 50, 100])
def test_split_initial_residency(small_pct, monkeypatch):
    """The initially resident slots hold the last segments of the arena (the
    small row classes; by default as many as there are, else the given
    share of the slots) and the first ones: values and rows stay exact
    against the oracle, also while the segment table evicts and admits."""
    if small_pct is not None:
        monkeypatch.setenv("CIG_CACHE_SMALL_PCT", str(small_pct))
    monkeypatch.setenv("CIG_CACHE_ADMIT_SCORE", "64")
    run_case_whole_batches(rmat_case(14, 5, 2000, 2000, seed_offset=16), "sssp", 8 * ONE_SEGMENT_GIB)


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_batched_form_equals_single_batches(algo):
    """cig_apply_batches_device (uneven batch sizes, one synchronisation)
    leaves every batch's values (digest per batch) and the final rows and
    values equal to one cig_apply_batch call per batch."""
    import torch

    from coincgraph_b200 import gen

    g, h = gen.rmat(12, keep_handle=True)
    sizes = [7, 900, 60, 0, 2500, 1]
    ups = gen.updates(h, sizes, sizes[::-1], seed=gen.UPDATE_SEED_BASE + 140)
    batches = [ups.batch(i) for i in range(len(sizes))]
    with Engine(algo, cache_gib=2 * ONE_SEGMENT_GIB) as a, Engine(algo, cache_gib=2 * ONE_SEGMENT_GIB) as b:
        for e in (a, b):
            e.load_csr(g.n, g.xadj, g.adj)
            e.init()
        expect = []
        for du, dv, au, av in batches:
            a.apply_batch(du, dv, au, av)
            expect.append(a.digest())
        dev = [[torch.from_numpy(x.astype(np.int32)).cuda() for x in bt] for bt in batches]
        stats, digests = b.apply_batches_device(dev)
        assert digests == expect
        assert [s.requested_deletes for s in stats] == sizes
        assert np.array_equal(a.values(), b.values())
        xa, aa = a.export_csr()
        xb, ab = b.export_csr()
        assert np.array_equal(xa, xb) and np.array_equal(aa, ab)


def test_device_inputs_match_host_inputs():
    import torch

    case = rmat_case(11, 2, 400, 400, seed_offset=13)
    with Engine("sssp", cache_gib=4.0) as a, Engine("sssp", cache_gib=4.0) as b:
        for e in (a, b):
            e.load_csr(case.n, case.xadj, case.adj)
            e.init()
        for du, dv, au, av in case.batches:
            a.apply_batch(du, dv, au, av)
            t = [torch.from_numpy(x.astype(np.int32)).cuda() for x in (du, dv, au, av)]
            b.apply_batch_device(*t)
            assert np.array_equal(a.values(), b.values())


def test_errors_are_reported():
    from coincgraph_b200 import CigError

    case = adversarial_case()
    with Engine("sssp") as eng:
        with pytest.raises(CigError):
            eng.init()  # no graph yet
        eng.load_csr(case.n, case.xadj, case.adj)
        with pytest.raises(CigError):
            eng.delete_phase([0], [1])  # before init
        eng.init()
        with pytest.raises(CigError):
            eng.load_csr(case.n, case.xadj, case.adj)  # already loaded
    with Engine("sssp") as eng:
        bad = case.adj.copy()
        bad[0] = case.n + 5
        with pytest.raises(CigError):
            eng.load_csr(case.n, case.xadj, bad)


def test_arena_exhaustion_is_an_error_not_a_fault():
    """A tiny arena runs out of room; the call fails cleanly with CIG_ERR_ARENA."""
    from coincgraph_b200 import CigError

    n = 2048
    src = np.arange(n, dtype=np.uint32)
    dst = (src + 1) % n
    from coincgraph_b200 import gen

    csr = gen.graph_from_edges(n, src, dst)
    with Engine("bfs", headroom_pct=1) as eng:
        eng.load_csr(n, csr.xadj, csr.adj)
        eng.init()
        rng = np.random.default_rng(3)
        with pytest.raises(CigError) as err:
            for _ in range(400):
                au = rng.integers(0, n, 5000).astype(np.uint32)
                av = rng.integers(0, n, 5000).astype(np.uint32)
                eng.apply_batch([], [], au, av)
        assert err.value.code == -4


def test_autotune_keeps_values_and_parity():
    """cig_autotune re-runs the static solve under each launch shape; the
    values stay the same and later batches still match the oracle."""
    case = rmat_case(12, 3, 500, 500, seed_offset=17)
    trace, _ = oracle_trace(case, "sssp")
    with Engine("sssp", cache_gib=4.0) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        before = eng.values()
        r = eng.autotune()
        assert r["candidates"] == 14 and r["blocks_per_sm"] in (2, 4, 8) and r["split_degree"] in (1024, 4096, 16384)
        assert r["pull_divisor"] in (0, 8, 16, 32, 64)
        assert np.array_equal(eng.values(), before)
        for i, b in enumerate(case.batches):
            eng.apply_batch(*b)
            assert np.array_equal(eng.values(), trace["batch"][i])


INDEX_MODES = {
    "off": {"CIG_POS_INDEX": "0"},
    "all_rows": {"CIG_POS_INDEX_CLS": "0"},
    "all_rows_rebuilt": {"CIG_POS_INDEX_CLS": "0", "CIG_POS_INDEX_HEADROOM": "64", "CIG_POS_INDEX_SPARE": "0"},
}


@pytest.mark.parametrize("mode", list(INDEX_MODES))
@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_position_index_modes(algo, mode, monkeypatch):
    """Deletion positions from the hub-row position index (every row indexed,
    and with a table small enough that appends force rebuilds) or from the
    flat scan alone (index off) give the reference's rows and values: parallel
    edges, repeated requests, compaction and relocation of indexed rows."""
    for k, v in INDEX_MODES[mode].items():
        monkeypatch.setenv(k, v)
    run_case(adversarial_case(), algo, CACHES["resident"])
    run_case(heavy_delete_case(), algo, CACHES["zerocopy"])
    run_case_whole_batches(big_row_case(), algo, CACHES["mixed"])
    run_case_whole_batches(rmat_case(11, 3, 400, 400, seed_offset=17), algo, CACHES["resident"])


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_grid_stream(algo):
    """High-diameter road-like graph (hundreds of rounds per closure)."""
    run_case(grid_case(), algo, CACHES["resident"])
    run_case_whole_batches(grid_case(40, 2, 100), algo, CACHES["zerocopy"])


@pytest.mark.parametrize("sweeps", ["0", "1", "4"])
@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_local_sweeps(algo, sweeps, monkeypatch):
    """Block-local sweeps in the push and invalidation closures
    (CIG_LOCAL_SWEEPS; 0 turns them off) keep values, parent witnesses and
    rows equal to the oracle's, including local-queue overflow (hub rows)
    and the grid case."""
    monkeypatch.setenv("CIG_LOCAL_SWEEPS", sweeps)
    run_case(grid_case(), algo, CACHES["resident"])
    run_case(adversarial_case(), algo, CACHES["resident"])
    run_case_whole_batches(big_row_case(), algo, CACHES["mixed"])
    run_case_whole_batches(rmat_case(11, 3, 400, 400, seed_offset=18), algo, CACHES["zerocopy"])


def _check_cc_witness(eng, case_n, xadj, adj, labels):
    """Every vertex that is not its own seed has a parent with its label and an
    edge parent -> vertex, and following parents reaches the seed (the vertex
    whose id is the label) without revisiting a vertex."""
    parents = eng.parents()
    rows = {}
    for v in range(case_n):
        if labels[v] == v:
            continue
        p = int(parents[v])
        assert p < case_n and labels[p] == labels[v], f"vertex {v}: parent {p} has another label"
        if p not in rows:
            rows[p] = set(adj[int(xadj[p]):int(xadj[p + 1])].tolist())
        assert v in rows[p], f"vertex {v}: no edge from its parent {p}"
    for v in range(case_n):
        seen, x = set(), v
        while labels[x] != x:
            assert x not in seen, f"parent cycle through {x}"
            seen.add(x)
            x = int(parents[x])
        assert x == labels[v]


@pytest.mark.parametrize("case", ["rmat", "adversarial", "grid"])
def test_cc_parents_are_rooted_witnesses(case):
    """CC parents form a forest rooted at each label's seed after the static
    solve and after every batch (depths never saturate at these sizes), which
    is what lets a deletion invalidate only the subtree below it."""
    c = {"rmat": lambda: rmat_case(11, 3, 300, 300, seed_offset=19), "adversarial": adversarial_case,
         "grid": lambda: grid_case(32, 3, 100)}[case]()
    g = oracle.Graph(c.n, c.xadj, c.adj)
    with make_engine("cc", cache_gib=CACHES["resident"]) as eng:
        eng.load_csr(c.n, c.xadj, c.adj)
        eng.init()
        _check_cc_witness(eng, c.n, c.xadj, c.adj, eng.values())
        for du, dv, au, av in c.batches:
            g.delete(du, dv)
            g.add(au, av)
            eng.apply_batch(du, dv, au, av)
            labels = eng.values()
            assert np.array_equal(labels, g.cc())
            xadj, adj = eng.export_csr()
            _check_cc_witness(eng, c.n, xadj, adj, labels)


@pytest.mark.parametrize("bits", ["0", "2"])
def test_cc_saturated_depths(bits, monkeypatch):
    """With the CC depth field capped (CIG_CC_DEPTH_BITS: 0 bits, or 2 bits so
    that depths saturate at 3 hops), saturated vertices fall back to the
    equal-label invalidation rule; labels and rows still equal the oracle's."""
    monkeypatch.setenv("CIG_CC_DEPTH_BITS", bits)
    run_case(rmat_case(11, 3, 300, 300, seed_offset=20), "cc", CACHES["resident"])
    run_case(adversarial_case(), "cc", CACHES["resident"])
    run_case(grid_case(24, 3, 80), "cc", CACHES["resident"])
    run_case_whole_batches(rmat_case(10, 3, 200, 200, seed_offset=21, symmetric=True), "cc", CACHES["mixed"])


@pytest.mark.parametrize("algo", ["bfs", "sssp", "cc"])
def test_whole_batch_single_push_closure(algo, monkeypatch):
    """Whole batches run one push closure after the insertions (the repaired
    vertices' frontier joins the insertion seeds); the values, rows and
    parent witnesses equal the oracle's and those of one push per phase
    (CIG_MERGE_PUSH=0) after every batch."""
    case = rmat_case(11, 4, 300, 300, seed_offset=23)
    out = {}
    for merged in ("1", "0"):
        monkeypatch.setenv("CIG_MERGE_PUSH", merged)
        run_case_whole_batches(case, algo, CACHES["mixed"])
        with make_engine(algo, cache_gib=4.0) as eng:
            eng.load_csr(case.n, case.xadj, case.adj)
            eng.init()
            out[merged] = []
            for b in case.batches:
                eng.apply_batch(*b)
                out[merged].append(eng.digest())
    assert out["1"] == out["0"]


def test_pinned_host_arrays_equal_pageable():
    """cig_apply_batch copies page-locked caller arrays by DMA directly and
    pageable ones through its pinned staging buffer: the same batches give
    the same values and rows either way, and the oracle's."""
    import torch

    case = rmat_case(12, 3, 400, 400, seed_offset=17)
    trace, _ = oracle_trace(case, "sssp")

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a).astype(np.int32)).pin_memory()
        return t, t.numpy().view(np.uint32)

    with Engine("sssp", cache_gib=ONE_SEGMENT_GIB) as a, Engine("sssp", cache_gib=ONE_SEGMENT_GIB) as b:
        for e in (a, b):
            e.load_csr(case.n, case.xadj, case.adj)
            e.init()
        for i, batch in enumerate(case.batches):
            held = [pinned(x) for x in batch]
            a.apply_batch(*(h[1] for h in held))
            b.apply_batch(*(np.asarray(x, dtype=np.uint32) for x in batch))
            assert np.array_equal(a.values(), trace["batch"][i]), f"batch {i}"
            assert np.array_equal(a.values(), b.values()) and a.digest() == b.digest()
            assert a.digest() == _value_digest(a.values())
            assert np.array_equal(a.export_csr()[1], trace["rows"][i][1])


def _value_digest(values):
    """cig_value_digest restated on the host: the sum mod 2^64 over reached
    vertices v of SplitMix64((v << 32) | value)."""
    v = np.flatnonzero(values != 0xFFFFFFFF).astype(np.uint64)
    with np.errstate(over="ignore"):
        z = (v << np.uint64(32)) | values[v.astype(np.int64)].astype(np.uint64)
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
        return int(np.sum(z, dtype=np.uint64))
