"""Device memory accounting (cig_memory_info_get) and the position-index
budget (cig_options.index_budget_gib): the reported parts add up to the
device memory the handle actually took, the index tables stay inside the
budget, and results stay exact against the oracle when the budget leaves
most rows unindexed."""
import numpy as np
import pytest

from coincgraph_b200 import Engine
from helpers import oracle_trace, rmat_case

pytestmark = pytest.mark.gpu


def test_memory_parts_match_the_device():
    import torch

    case = rmat_case(14, 2, 500, 500, seed_offset=70)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    with Engine("sssp", cache_gib=0.01, max_batch=500) as eng:
        eng.load_csr(case.n, case.xadj, case.adj)
        eng.init()
        for b in case.batches:
            eng.apply_batch(*b)
        m = eng.memory()
        used = free0 - torch.cuda.mem_get_info()[0]
    parts = sum(v for k, v in m.items() if k not in ("total", "pinned_host"))
    assert parts == m["total"]
    for k in ("edge_cache", "descriptors", "reverse_arena", "vertex_state", "batch_buffers"):
        assert m[k] > 0, k
    assert m["pinned_host"] > 0
    # cudaMalloc rounds every allocation up to its granule, and the CUDA
    # graphs and events hold some device memory of their own
    assert m["total"] <= used <= m["total"] + (256 << 20), (m["total"], used)


def test_index_budget_bounds_the_tables_and_keeps_results():
    case = rmat_case(13, 3, 400, 400, seed_offset=71)
    trace, _ = oracle_trace(case, "bfs")
    sizes = {}
    for budget in (0.0, 1.0 / 1024):  # default, then 1 MiB for both tables
        with Engine("bfs", cache_gib=4.0, index_budget_gib=budget) as eng:
            eng.load_csr(case.n, case.xadj, case.adj)
            eng.init()
            for i, b in enumerate(case.batches):
                eng.apply_batch(*b)
                assert np.array_equal(eng.values(), trace["batch"][i]), f"budget {budget}: batch {i}"
                xadj, adj = eng.export_csr()
                assert np.array_equal(adj, trace["rows"][i][1])
            sizes[budget] = eng.memory()["position_index"]
    assert sizes[1.0 / 1024] <= (1 << 20)
    assert sizes[0.0] > sizes[1.0 / 1024]
