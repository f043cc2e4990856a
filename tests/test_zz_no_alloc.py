"""cig_bfs_csr_noalloc: BFS depths over a device CSR without device allocation.

The entry point is for callers that cannot call cudaMalloc where they need a
traversal: plugins whose host framework owns the device memory pool, and
latency-bound loops that must not take cudaFree's device-wide
synchronisation.  Its scratch is one fixed __device__ array shared by every
call, so these tests run it twice in a row on different sources (the second
call starts from what the first left in the array) and compare the depths
exactly with the oracle's BFS and with the regular handle-based path
(cig_create/cig_load_csr/cig_init/cig_get_values with CIG_BFS).  They also
check that free device memory does not move across calls after the first
(the first may load the library's device code, which holds the array), and
cover a row long enough for the block-wide and multi-segment expansion
paths.  This file is named to be collected last so that a `-x` run has
executed every other test first.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def _handle_depths(g, source):
    from coincgraph_b200 import Engine

    with Engine("bfs", source=source, cache_gib=4.0) as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        return eng.values()


def _hub_graph():
    """4096 random edges plus vertex 3 with 20000 out-edges (more than one
    64 KiB segment) and vertex 7 with 600 (block-wide tier)."""
    from coincgraph_b200 import gen

    rng = np.random.default_rng(99)
    n = 30000
    src = np.concatenate([np.full(20000, 3), np.full(600, 7), rng.integers(0, n, 4096), [0, 0]])
    dst = np.concatenate([rng.integers(0, n, 20000), rng.integers(0, n, 600), rng.integers(0, n, 4096), [3, 7]])
    return gen.graph_from_edges(n, src, dst)


def _run_twice(lib, g, sources):
    import torch

    dev = torch.device("cuda", 0)
    expect = {s: (oracle.Graph(g.n, g.xadj, g.adj).sssp(s, oracle.BFS), _handle_depths(g, s)) for s in sources}
    xadj = torch.from_numpy(g.xadj.astype(np.int64)).to(dev)
    adj = torch.from_numpy(g.adj.astype(np.int32)).to(dev)
    depth = torch.empty(g.n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize()
    free = []
    for source in sources:
        rc = lib.cig_bfs_csr_noalloc(xadj.data_ptr(), adj.data_ptr(), g.n, source, depth.data_ptr(), stream)
        assert rc == 0, lib.cig_last_error(None).decode()
        got = depth.cpu().numpy().view(np.uint32)
        want_oracle, want_handle = expect[source]
        assert np.array_equal(got, want_oracle), f"source {source}: depths differ from the oracle"
        assert np.array_equal(got, want_handle), f"source {source}: depths differ from the handle path"
        free.append(torch.cuda.mem_get_info(dev)[0])
    return free


def test_noalloc_bfs_matches_oracle_and_handle_path_on_consecutive_calls():
    from coincgraph_b200 import engine, gen

    lib = engine.load_library()
    g = gen.rmat(12)  # 4096 vertices
    sources = [0, int(np.argmax(np.diff(g.xadj.astype(np.int64)))), 0]
    free = _run_twice(lib, g, sources)
    # calls after the first allocate nothing
    assert free[1] == free[0] and free[2] == free[0], f"free device memory moved across calls: {free}"


def test_noalloc_bfs_long_rows():
    from coincgraph_b200 import engine

    lib = engine.load_library()
    g = _hub_graph()
    free = _run_twice(lib, g, [0, 3, 7])
    assert free[1] == free[0] and free[2] == free[0], f"free device memory moved across calls: {free}"


def test_noalloc_rejects_sizes_beyond_its_scratch_and_null_arrays():
    import torch

    from coincgraph_b200 import engine

    lib = engine.load_library()
    limit = 1 << 18  # CIG_NOALLOC_MAX_VERTICES
    xadj = torch.zeros(limit + 2, dtype=torch.int64, device="cuda")
    adj = torch.zeros(1, dtype=torch.int32, device="cuda")
    depth = torch.empty(limit + 1, dtype=torch.int32, device="cuda")
    rc = lib.cig_bfs_csr_noalloc(xadj.data_ptr(), adj.data_ptr(), limit + 1, 0, depth.data_ptr(), None)
    assert rc == -1
    assert "vertex count" in lib.cig_last_error(None).decode()
    rc = lib.cig_bfs_csr_noalloc(xadj.data_ptr(), None, 16, 0, depth.data_ptr(), None)
    assert rc == -1
    assert "null" in lib.cig_last_error(None).decode()
