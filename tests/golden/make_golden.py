"""Generate the golden fixtures in tests/golden/ (run from the repository root).

The reference ships no golden vectors, graphs or known-answer files, so the
fixtures are made here and pinned to the reference's own code before they
are frozen:
  - rows after every batch: the plain-C oracle must equal the reference's
    SourceLocalChunkStore compiled from its sources (oracle/_ref), row for row;
  - CC labels: the reference's CCCheck must report 0 errors;
  - BFS/SSSP distances: two independent oracles (FIFO label-correcting as in
    the reference host code, and Dial's bucket queue) must agree and pass the
    restated Bellman certificate;
  - PageRank: the reference's PageRankCheck must pass on the FP64 fixed point.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from helpers import adversarial_case, rmat_case  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def pack_batches(batches):
    d = {}
    for i, (du, dv, au, av) in enumerate(batches):
        d[f"b{i}_du"], d[f"b{i}_dv"], d[f"b{i}_au"], d[f"b{i}_av"] = du, dv, au, av
    return d


def make(case):
    assert oracle.ref_available(), "build oracle/_ref first (python oracle/build.py)"
    g = oracle.Graph(case.n, case.xadj, case.adj)
    ref = oracle.RefStore(case.n, case.xadj, case.adj)
    data = {"n": np.uint32(case.n), "xadj": case.xadj, "adj": case.adj, "source": np.uint32(case.source),
            "nbatches": np.uint32(len(case.batches))}
    data.update(pack_batches(case.batches))

    def solve(tag):
        for name, mode in (("bfs", oracle.BFS), ("sssp", oracle.SSSP)):
            d = g.sssp(case.source, mode)
            assert np.array_equal(d, g.sssp_dial(case.source, mode)), "FIFO and Dial disagree"
            assert g.bellman_check(d, case.source, mode) == (0, 0)
            data[f"{tag}_{name}"] = d
        labels = g.cc()
        assert ref.cc_errors(labels) == 0, "reference CCCheck rejects the oracle's labels"
        data[f"{tag}_cc"] = labels

    solve("init")
    empty = np.zeros(0, dtype=np.uint32)
    for i, (du, dv, au, av) in enumerate(case.batches):
        missing = g.delete(du, dv)
        counts = ref.apply(du, dv, empty, empty)
        assert counts["missing_deletes"] == missing, (counts, missing)
        solve(f"b{i}_del")
        invalid = g.add(au, av)
        ref.apply(empty, empty, au, av)
        xo, ao = g.export()
        xr, ar = ref.export()
        assert np.array_equal(xo, xr) and np.array_equal(ao, ar), "oracle rows differ from the reference store"
        data[f"b{i}_xadj"], data[f"b{i}_adj"] = xo, ao
        data[f"b{i}_missing"] = np.uint64(missing)
        data[f"b{i}_invalid"] = np.uint64(invalid)
        solve(f"b{i}_ins")
    x, ok = g.pagerank(1e-14, 50000)
    assert ok
    nxt = np.full(case.n, 0.15)
    xa, aa = g.export()
    deg = np.diff(xa)
    for s in range(case.n):
        if deg[s]:
            np.add.at(nxt, aa[int(xa[s]):int(xa[s + 1])], 0.85 * np.float64(np.float32(x[s])) / deg[s])
    residual = (nxt - x.astype(np.float32).astype(np.float64)).astype(np.float32)
    assert ref.pr_check(x.astype(np.float32), residual, 1e-6), "reference PageRankCheck rejects the oracle"
    data["final_pr"] = x
    return data


def main():
    for case in (rmat_case(8, 4, 24, 24, seed_offset=1), adversarial_case()):
        data = make(case)
        path = os.path.join(OUT, f"{case.name}.npz")
        np.savez_compressed(path, **data)
        print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
