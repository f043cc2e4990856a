"""GPU PageRank against the FP64 oracle.

Tolerance: max relative error <= 1e-5 against the FP64 Jacobi fixed point of
the current graph (FP32 ranks with Kahan-compensated sums, epsilon 1e-9);
<= 1e-9 in FP64 mode.  With the reference's default --error=1e-6 the result
must pass the reference's own PageRankCheck bound.
"""
import numpy as np
import pytest

import oracle
from coincgraph_b200 import Engine
from coincgraph_b200.engine import FLAG_PR_FP64
from helpers import adversarial_case, big_row_case, rmat_case

pytestmark = pytest.mark.gpu


def max_rel(x, ref):
    return float(np.max(np.abs(x.astype(np.float64) - ref) / np.abs(ref)))


@pytest.mark.parametrize("fp64,eps,tol", [(False, 1e-9, 1e-5), (True, 1e-13, 1e-9)])
@pytest.mark.parametrize("make", [lambda: rmat_case(10, 4, 200, 200, seed_offset=20), adversarial_case,
                                  big_row_case])
def test_pr_stream(make, fp64, eps, tol):
    case = make()
    g = oracle.Graph(case.n, case.xadj, case.adj)
    flags = FLAG_PR_FP64 if fp64 else 0
    with Engine("pr", pr_epsilon=eps, pr_max_rounds=100000, flags=flags) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        x, ok = g.pagerank(1e-15, 100000)
        assert ok
        assert max_rel(eng.pagerank(fp64=fp64)[0], x) <= tol
        for du, dv, au, av in case.batches:
            g.delete(du, dv)
            g.add(au, av)
            s = eng.apply_batch(du, dv, au, av)
            assert s["pr_residual_l1"] <= case.n * eps * 1.01
            x, ok = g.pagerank(1e-15, 100000)
            assert ok
            assert max_rel(eng.pagerank(fp64=fp64)[0], x) <= tol
            xadj, adj = eng.export_csr()
            xo, ao = g.export()
            assert np.array_equal(xadj, xo) and np.array_equal(adj, ao)


def test_pr_reference_check_at_default_error():
    case = rmat_case(10, 3, 100, 100, seed_offset=21)
    g = oracle.Graph(case.n, case.xadj, case.adj)
    ref = oracle.RefStore(case.n, case.xadj, case.adj) if oracle.ref_available() else None
    with Engine("pr", pr_epsilon=1e-6, pr_max_rounds=100) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        for du, dv, au, av in case.batches:
            g.delete(du, dv)
            g.add(au, av)
            if ref is not None:
                ref.apply(du, dv, au, av)
            eng.apply_batch(du, dv, au, av)
            rank, res = eng.pagerank()
            assert g.pr_check(rank, res, 1e-6)["ok"] == 1.0
            if ref is not None:
                assert ref.pr_check(rank, res, 1e-6)
