"""bench.py's host-side arithmetic, on CPU: the stage byte model and its
roofline fractions, the traffic ratios' consistency with their sources, and
the workload keys both arms report."""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_model_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.path.insert(0, ROOT)
    spec.loader.exec_module(mod)
    return mod


def test_traversal_stage_bytes_split_hbm_and_link():
    b = _bench()
    st = {"edges": 1000, "edges_cached": 600, "rows": 50, "hits": 20, "ms": 1.0, "launches": 1}
    hbm, link = b.stage_bytes("push", st)
    assert link == 400 * b.ADJ_BYTES
    assert hbm == 50 * b.ROW_BYTES + 1000 * b.EDGE_STATE_BYTES + 600 * b.ADJ_BYTES + 20 * b.HIT_BYTES
    # an all-resident stage crosses no host link
    st["edges_cached"] = 1000
    assert b.stage_bytes("inval", st)[1] == 0


def test_stage_roofline_fractions():
    b = _bench()
    st = {"edges": 0, "edges_cached": 0, "rows": 4, "hits": 0, "ms": 2.0, "launches": 2}
    r = b.stage_roofline("cache", st, hbm_peak=1000.0, link_peak=50.0, batches=2)
    seg = 4 * b.SEG_BYTES
    assert r["ms_per_batch"] == pytest.approx(1.0)
    assert r["launches_per_batch"] == pytest.approx(1.0)
    assert r["achieved_hbm_gbs"] == pytest.approx(seg / 2e-3 / 1e9)
    t_roof = seg / 1000e9 + seg / 50e9
    assert r["frac_combined"] == pytest.approx(t_roof / 2e-3)
    assert b.stage_roofline("push", dict(st, ms=0.0), 1000.0, 50.0, 1) is None


def test_traffic_ratios_match_their_stated_captures():
    """Each ratio is the DRAM bytes over the algorithmic bytes its source
    text quotes (MB figures rounded to 0.1 / 0.01)."""
    import re

    b = _bench()
    for kernel, (ratio, source) in b.TRAFFIC_RATIO.items():
        dram, alg = (float(x) for x in re.findall(r"([\d.]+) MB", source)[:2])
        assert ratio == pytest.approx(dram / alg, rel=0.02), kernel


def test_both_arms_report_the_same_workload_keys():
    b = _bench()

    class G:
        n, m = 16, 40

    sys.argv = ["bench.py"]
    args = b.parse_args()
    ours = b.stream_config(args, G)
    assert ours["workload"] == b.WORKLOAD  # the default run is the named benchmark workload
    assert set(ours) == {"workload", "algo", "scale", "vertices", "edges", "batch", "cache_gib", "source", "l2",
                         "parallelism"}
    args.algo = "cc"
    other = b.stream_config(args, G)
    assert set(other) == set(ours) and other["workload"] != b.WORKLOAD
