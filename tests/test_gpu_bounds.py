"""The bounds-checked engine build (libcig_bc.so, -DCIG_BOUNDS_CHECK) and the
build's target architecture.

compute-sanitizer is closed on this pool, so the engine has a build that
checks every arena slot it reads or writes and every vertex id it reads from
a row against its bound, and reports a violation through the device status
word instead of touching memory outside its arrays.  These tests run the
parity cases (adversarial rows, hub rows above the split threshold and a
segment, heavy deletions, R-MAT streams under all cache budgets, the
multi-source queries) through that build in a child process and require
identical results to the oracle and no reported violation.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_release_build_runs_sm100_code():
    from coincgraph_b200 import engine

    info = engine.build_info()
    assert info["binary_version"] == 100, info
    assert not info["bounds_checked"]


CHILD = r"""
import os, sys
sys.path[:0] = [{root!r}, os.path.join({root!r}, "tests")]
import numpy as np
from coincgraph_b200 import engine
assert engine.build_info()["bounds_checked"], "CIG_LIBRARY did not select the bounds-checked build"
from helpers import adversarial_case, big_row_case, heavy_delete_case, rmat_case
from test_gpu_parity import CACHES, run_case, run_case_whole_batches
for algo in ("bfs", "sssp", "cc"):
    run_case(adversarial_case(), algo, 4.0)
    run_case(rmat_case(11, 3, 300, 300, seed_offset=60), algo, CACHES["mixed"])
    run_case_whole_batches(rmat_case(11, 3, 300, 300, seed_offset=61), algo, CACHES["zerocopy"])
for algo in ("sssp", "cc"):
    run_case(big_row_case(), algo, CACHES["mixed"])
    run_case(heavy_delete_case(), algo, CACHES["resident"])
from coincgraph_b200 import Engine, gen
import oracle
g = gen.rmat(11, symmetric=True)
src = np.arange(0, 640, 10, dtype=np.uint32)
with Engine("bfs", cache_gib=4.0) as eng:
    eng.load_csr(g.n, g.xadj, g.adj)
    got = eng.query_bfs(src)
og = oracle.Graph(g.n, g.xadj, g.adj)
for k, s in enumerate(src.tolist()):
    assert np.array_equal(got[k], og.sssp(s, oracle.BFS))
print("bounds-checked build: all cases equal the oracle, no violation")
"""


def test_bounds_checked_build_parity():
    lib = os.path.join(ROOT, "coincgraph_b200", "libcig_bc.so")
    assert os.path.exists(lib), "build libcig_bc.so first (python -m coincgraph_b200.build)"
    env = dict(os.environ, CIG_LIBRARY=lib)
    proc = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True, text=True,
                          timeout=900)
    assert proc.returncode == 0, proc.stdout[-3000:] + proc.stderr[-3000:]
    assert "no violation" in proc.stdout
