"""The C-ABI libraries load and export every symbol their headers declare.

No compute call is made here (no GPU in the CPU suite).
"""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header: str) -> list[str]:
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(cig_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.mark.parametrize("header,lib", [("cig.h", "libcig.so"), ("cig.h", "libcig_bc.so"),
                                        ("cig_gen.h", "libcig_gen.so")])
def test_library_exports_header(built, header, lib):
    path = os.path.join(ROOT, "coincgraph_b200", lib)
    so = ctypes.CDLL(path)
    names = declared(header)
    assert len(names) >= 5
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_binding_covers_header(built):
    from coincgraph_b200 import engine

    bound = {name for name, _, _ in engine.SIGNATURES}
    assert set(declared("cig.h")) == bound


def test_engine_builds_for_sm100a_only(built):
    # The compile lines name one target, sm_100a (the GPU tests confirm it
    # through cig_build_info: binaryVersion 100).
    from coincgraph_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_bounds_checked_library_reports_itself(built):
    lib = ctypes.CDLL(os.path.join(ROOT, "coincgraph_b200", "libcig_bc.so"))
    bc = ctypes.c_int(-1)
    assert lib.cig_build_info(None, ctypes.byref(bc)) == 0 and bc.value == 1
    rel = ctypes.CDLL(os.path.join(ROOT, "coincgraph_b200", "libcig.so"))
    assert rel.cig_build_info(None, ctypes.byref(bc)) == 0 and bc.value == 0


def test_options_defaults_match_reference_flags(built):
    from coincgraph_b200 import engine

    o = engine.default_options()
    assert o.algo == engine.SSSP
    assert o.cache_gib == 4.0          # --cache=4 (app_skeleton.h:89)
    assert abs(o.pr_epsilon - 1e-6) < 1e-18  # --error (hybrid_pr.cu:23)
    assert o.pr_max_rounds == 100      # --pr_max_rounds (hybrid_pr.cu:22)


def test_struct_layouts(built):
    from coincgraph_b200 import engine

    assert ctypes.sizeof(engine.Options) == 56
    assert ctypes.sizeof(engine.MemoryInfo) == 10 * 8
    assert ctypes.sizeof(engine.BatchStats) == 21 * 8
    assert ctypes.sizeof(engine.StageProfile) == 6 * 8
    assert ctypes.sizeof(engine.QueryStats) == 8 * 8
    assert ctypes.sizeof(engine.UpdateBatch) == 6 * 8
    assert ctypes.sizeof(engine.Request) == 8 * 8
    assert ctypes.sizeof(engine.Result) == 5 * 8
    assert ctypes.sizeof(engine.ServeOptions) == 16
    assert ctypes.sizeof(engine.TuneResult) == 24
