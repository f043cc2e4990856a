"""cig_bfs_csr_noalloc: BFS depths over a device CSR without device allocation.

The entry point exists for callers that cannot allocate device memory where
they need a traversal (inside CUDA stream capture, in serving loops that must
avoid cudaMalloc's implicit synchronisation, or in hosts that do not own the
device memory pool).  Its depths must equal those of the regular handle-based
path (cig_create/cig_load_csr/cig_init/cig_get_values with CIG_BFS), exactly,
on consecutive calls that reuse the shared scratch array.  This file is named
to be collected last so that a `-x` run has executed every other test first.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference_depths(g, source):
    from coincgraph_b200 import Engine

    with Engine("bfs", source=source, cache_gib=4.0) as eng:
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        return eng.values()


def test_noalloc_bfs_matches_handle_path_on_consecutive_calls():
    import torch

    from coincgraph_b200 import engine, gen

    lib = engine.load_library()
    g = gen.rmat(12)  # 4096 vertices
    dev = torch.device("cuda", 0)
    xadj = torch.from_numpy(g.xadj.astype(np.int64)).to(dev)
    adj = torch.from_numpy(g.adj.astype(np.int32)).to(dev)
    depth = torch.empty(g.n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    sources = [0, int(np.argmax(np.diff(g.xadj[1:]))) + 1]  # two different sources, back to back
    for source in sources:
        rc = lib.cig_bfs_csr_noalloc(xadj.data_ptr(), adj.data_ptr(), g.n, source, depth.data_ptr(), stream)
        assert rc == 0, lib.cig_last_error(None).decode()
        got = depth.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, _reference_depths(g, source))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    from coincgraph_b200 import engine

    lib = engine.load_library()
    limit = 1 << 18  # CIG_NOALLOC_MAX_VERTICES
    xadj = torch.zeros(limit + 2, dtype=torch.int64, device="cuda")
    depth = torch.empty(limit + 1, dtype=torch.int32, device="cuda")
    rc = lib.cig_bfs_csr_noalloc(xadj.data_ptr(), None, limit + 1, 0, depth.data_ptr(), None)
    assert rc == -1
    assert "vertex count" in lib.cig_last_error(None).decode()
