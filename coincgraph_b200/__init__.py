"""coincgraph_b200 - B200-native incremental streaming-graph engine.

The compute path is ``libcig.so`` (hand-written sm_100a CUDA behind the C ABI
in ``include/cig.h``); the ``hybrid_bfs`` / ``hybrid_sssp`` / ``hybrid_cc`` /
``hybrid_pr`` tools in ``coincgraph_b200/bin`` are drop-in replacements for
the reference's executables.  ``engine`` is a ctypes binding of the C ABI and
``gen`` produces seeded R-MAT graphs and update streams.
"""
from .engine import BFS, CC, PR, SSSP, CigError, Engine, load_library, version  # noqa: F401

__all__ = ["Engine", "CigError", "load_library", "version", "BFS", "SSSP", "CC", "PR"]
