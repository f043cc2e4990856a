"""Serving loop: results in the mix equal results alone.

A stream of update batches and BFS/SSSP queries is submitted to a serving
handle (from one thread, and from several at once); each query's depths or
distances must equal those of the same query run alone on the oracle graph
holding exactly the updates submitted before it, and each update's digest
must equal the value digest of one-call-per-batch processing.  Admission by
memory footprint is exercised by a budget that forces updates into chunks
and narrow waves.
"""
import threading

import numpy as np
import pytest

import oracle
from coincgraph_b200 import CigError, Engine, gen

pytestmark = pytest.mark.gpu


def _stream(scale=12, nbatches=4, size=400, seed=150):
    g, h = gen.rmat(scale, keep_handle=True)
    ups = gen.updates(h, [size] * nbatches, [size] * nbatches, seed=gen.UPDATE_SEED_BASE + seed)
    return g, [ups.batch(i) for i in range(nbatches)]


def _plan(g, batches, queries_per_gap=5, seed=3):
    """Requests in submission order: queries between batches."""
    rng = np.random.default_rng(seed)
    deg = np.diff(g.xadj.astype(np.int64))
    live = np.flatnonzero(deg > 0)
    plan = []
    for i in range(len(batches) + 1):
        for _ in range(queries_per_gap):
            plan.append(("bfs" if rng.random() < 0.5 else "sssp", int(rng.choice(live)), i))
        if i < len(batches):
            plan.append(("update", i, i))
    return plan


def _alone(g, batches, plan):
    """Expected result of every request, computed one at a time on the oracle."""
    og = oracle.Graph(g.n, g.xadj, g.adj)
    applied = 0
    expect = []
    for kind, x, epoch in plan:
        while applied < epoch:
            du, dv, au, av = batches[applied]
            og.delete(du, dv)
            og.add(au, av)
            applied += 1
        if kind == "update":
            expect.append(None)
        else:
            expect.append(og.sssp(x, oracle.BFS if kind == "bfs" else oracle.SSSP))
    return expect


def _update_digests(g, batches):
    out = []
    with Engine("sssp", cache_gib=1.0) as e:
        e.load_csr(g.n, g.xadj, g.adj)
        e.init()
        for b in batches:
            e.apply_batch(*b)
            out.append(e.digest())
    return out


# budget 0: half of free memory; 700 kB: updates of 1500 records run as
# 1024-record chunks and waves hold at most 21 sources.
@pytest.mark.parametrize("budget", [0, 700_000])
def test_serve_mix_equals_alone(built, budget):
    g, batches = _stream(size=1500)
    plan = _plan(g, batches)
    expect = _alone(g, batches, plan)
    upd_digest = _update_digests(g, batches)
    outs = [np.zeros(g.n, dtype=np.uint32) if k != "update" else None for k, _, _ in plan]
    with Engine("sssp", cache_gib=1.0) as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        eng.serve_start(budget_bytes=budget)
        tickets = []
        for (kind, x, _), out in zip(plan, outs):
            if kind == "update":
                tickets.append(eng.submit_update(*batches[x]))
            else:
                tickets.append(eng.submit_query(kind, x, out))
        results = [eng.wait(t) for t in tickets]
        with pytest.raises(CigError):  # other calls are refused while serving
            eng.values()
        eng.serve_stop()
        final = eng.values()
    waves = []
    for (kind, x, epoch), out, exp, res in zip(plan, outs, expect, results):
        assert res["status"] == 0
        if kind == "update":
            assert res["digest"] == upd_digest[x], f"update {x}"
        else:
            np.testing.assert_array_equal(out, exp, err_msg=f"{kind} from {x} after {epoch} updates")
            waves.append(res["wave"])
    assert max(waves) > 1, "queries were never batched into one wave"
    og = oracle.Graph(g.n, g.xadj, g.adj)
    for b in batches:
        og.delete(b[0], b[1])
        og.add(b[2], b[3])
    np.testing.assert_array_equal(final, og.sssp(0, oracle.SSSP))


def test_serve_concurrent_submitters(built):
    """Two threads submit queries while the main thread submits updates; each
    query's depths must equal the oracle's answer on one of the graph states
    the stream passes through (which one depends on the interleaving)."""
    g, batches = _stream(nbatches=3, size=300, seed=151)
    og = oracle.Graph(g.n, g.xadj, g.adj)
    states = []
    for i in range(len(batches) + 1):
        states.append(og.export())
        if i < len(batches):
            og.delete(batches[i][0], batches[i][1])
            og.add(batches[i][2], batches[i][3])
    deg = np.diff(g.xadj.astype(np.int64))
    sources = [int(s) for s in np.flatnonzero(deg > 0)[:12]]
    answers = {}
    for si, (xadj, adj) in enumerate(states):
        o = oracle.Graph(g.n, xadj, adj)
        for s in sources:
            answers[(si, s)] = o.sssp(s, oracle.BFS)
    with Engine("bfs", cache_gib=1.0) as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        eng.serve_start(max_wave=8)
        got = []
        lock = threading.Lock()

        def querier(seed):
            for s in sources:
                out = np.zeros(g.n, dtype=np.uint32)
                t = eng.submit_query("bfs", s, out)
                r = eng.wait(t)
                with lock:
                    got.append((s, out, r))

        threads = [threading.Thread(target=querier, args=(k,)) for k in range(2)]
        for t in threads:
            t.start()
        for b in batches:
            eng.wait(eng.submit_update(*b))
        for t in threads:
            t.join()
        eng.serve_stop()
    assert len(got) == 2 * len(sources)
    for s, out, r in got:
        assert r["status"] == 0
        assert any(np.array_equal(out, answers[(si, s)]) for si in range(len(states))), f"source {s}"


def test_serve_rejects_bad_requests(built):
    g, _ = _stream(scale=8, nbatches=1, size=10)
    with Engine("bfs") as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        eng.serve_start()
        with pytest.raises(CigError):
            eng.submit_query("bfs", g.n)
        t = eng.submit_query("bfs", 0)
        r = eng.wait(t)
        assert r["status"] == 0 and r["digest"] == eng_digest_alone(g)
        with pytest.raises(CigError):
            eng.wait(t)  # a result is taken once
        eng.serve_stop()


def eng_digest_alone(g):
    with Engine("bfs", source=0) as e:
        e.load_csr(g.n, g.xadj, g.adj)
        e.init()
        return e.digest()
