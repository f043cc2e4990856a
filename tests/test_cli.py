"""The drop-in command-line tools (hybrid_bfs / hybrid_sssp / hybrid_cc /
hybrid_pr): flag handling and input errors on the CPU, full runs with
--check and --output on the GPU, compared with the oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from coincgraph_b200 import gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "coincgraph_b200", "bin")


def tool(name):
    return os.path.join(BIN, f"hybrid_{name}")


def run(name, *args, timeout=600):
    return subprocess.run([tool(name), *args], capture_output=True, text=True, timeout=timeout)


@pytest.fixture
def dataset(tmp_path):
    g, h = gen.rmat(10, keep_handle=True)
    ups = gen.updates(h, [40] * 3, [40] * 3, seed=gen.UPDATE_SEED_BASE + 30)
    graph = tmp_path / "graph.txt"
    upd = tmp_path / "updates.txt"
    sizes = tmp_path / "batches.txt"
    gen.write_graph_txt(str(graph), g)
    gen.write_updates_txt(str(upd), str(sizes), ups)
    return g, ups, str(graph), str(upd), str(sizes), tmp_path


@pytest.mark.parametrize("name", ["bfs", "sssp", "cc", "pr"])
def test_unknown_flag_is_an_error(built, name):
    r = run(name, "--no_such_flag=1")
    assert r.returncode != 0
    assert "unknown command line flag" in r.stderr


@pytest.mark.parametrize("name", ["bfs", "sssp"])
def test_missing_graph_is_an_error(built, name):
    r = run(name)
    assert r.returncode != 0
    assert "A Graph File must be provided" in r.stderr
    assert "Overall: Test FAILED" in r.stdout


def test_help_lists_reference_flags(built):
    r = run("sssp", "--help")
    assert r.returncode == 0
    for flag in ("graphfile", "updatefile", "update_size", "cache", "weight_num", "source_node", "check",
                 "sssp_max_batches", "sssp_print_checksum", "SEGMENT", "n_stream"):
        assert f"--{flag} " in r.stdout


def test_pr_flag_validation(built, dataset):
    _, _, graph, _, _, _ = dataset
    r = run("pr", f"--graphfile={graph}", "--pr_max_rounds=0")
    assert r.returncode != 0 and "pr_max_rounds" in r.stderr


def test_malformed_inputs(built, tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("0 1\n1 x\n")
    r = run("cc", f"--graphfile={bad}")
    assert r.returncode != 0 and "malformed graph line" in r.stderr
    good = tmp_path / "g.txt"
    good.write_text("0 1\n1 2\n")
    upd = tmp_path / "u.txt"
    upd.write_text("a 0 2 1\nq 1 2 3\n")
    sizes = tmp_path / "s.txt"
    sizes.write_text("1 0\n")
    r = run("sssp", f"--graphfile={good}", f"--updatefile={upd}", f"--update_size={sizes}")
    assert r.returncode != 0 and "malformed update line" in r.stderr
    upd.write_text("a 0 2 1\n")
    sizes.write_text("5 0\n")
    r = run("sssp", f"--graphfile={good}", f"--updatefile={upd}", f"--update_size={sizes}")
    assert r.returncode != 0 and "more records" in r.stderr


def _oracle_final(g, ups, mode):
    og = oracle.Graph(g.n, g.xadj, g.adj)
    for i in range(ups.batches):
        du, dv, au, av = ups.batch(i)
        og.delete(du, dv)
        og.add(au, av)
    return og


@pytest.mark.gpu
@pytest.mark.parametrize("name,mode", [("bfs", oracle.BFS), ("sssp", oracle.SSSP)])
def test_traversal_tool_end_to_end(dataset, name, mode):
    g, ups, graph, upd, sizes, tmp = dataset
    out = tmp / "out.txt"
    r = run(name, f"--graphfile={graph}", "--format=market_big", "--weight_num=1", f"--updatefile={upd}",
            f"--update_size={sizes}", "--weight=true", "--cache=2", f"--{name}_max_batches=10", "--check=true",
            f"--{name}_print_checksum=true", f"--output={out}")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    up = name.upper()
    assert len(re.findall(rf"\[TIMER\]\[{up}\]\[batch \d+\] total_batch: [0-9.]+ ms", r.stdout)) == 3
    assert len(re.findall(rf"\[{up}-DELETE-STAGE-CHECK\]\[batch \d+\] passed", r.stdout)) == 3
    assert len(re.findall(rf"\[{up}-BATCH-CHECK\]\[batch \d+\] passed", r.stdout)) == 3
    assert f"[{up}-BELLMAN-CHECK] passed" in r.stdout
    assert "clamp" in r.stdout and "Overall: Test passed" in r.stdout
    cols = np.loadtxt(out, dtype=np.uint64)
    og = _oracle_final(g, ups, mode)
    assert np.array_equal(cols[:, 1].astype(np.uint32), og.sssp(0, mode))
    m = re.search(r"distance_checksum=(\d+) parent_checksum", r.stdout)
    assert int(m.group(1)) == oracle.checksum(og.sssp(0, mode))


@pytest.mark.gpu
def test_sssp_tool_extensions(dataset):
    """--weight_u255 (weights in [1, 255]), --write_cigb then a run from the
    binary sidecar, and --autotune: checks pass and distances match the
    oracle with the same weights."""
    g, ups, graph, upd, sizes, tmp = dataset
    out = tmp / "out_u255.txt"
    common = [f"--updatefile={upd}", f"--update_size={sizes}", "--cache=2", "--check=true", "--weight_u255=true"]
    r = run("sssp", f"--graphfile={graph}", "--write_cigb=true", "--autotune=true", *common)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    assert os.path.exists(graph + ".cigb") and "[AUTOTUNE] blocks_per_sm=" in r.stdout
    r = run("sssp", f"--graphfile={graph}", f"--output={out}", *common)
    assert r.returncode == 0 and "Overall: Test passed" in r.stdout, r.stdout[-2000:] + r.stderr
    cols = np.loadtxt(out, dtype=np.uint64)
    og = _oracle_final(g, ups, oracle.SSSP_U255)
    assert np.array_equal(cols[:, 1].astype(np.uint32), og.sssp(0, oracle.SSSP_U255))


@pytest.mark.gpu
def test_cc_tool_end_to_end(dataset):
    g, ups, graph, upd, sizes, tmp = dataset
    out = tmp / "labels.txt"
    r = run("cc", f"--graphfile={graph}", f"--updatefile={upd}", f"--update_size={sizes}", "--check=true",
            "--cc_print_checksum=true", f"--output={out}")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    assert len(re.findall(r"\[CC-BATCH-CHECK\]\[batch \d+\] passed", r.stdout)) == 3
    assert "[CC-FINAL-CHECK] passed errors=0" in r.stdout
    labels = np.loadtxt(out, dtype=np.uint64)[:, 1].astype(np.uint32)
    assert np.array_equal(labels, _oracle_final(g, ups, oracle.CC).cc())


@pytest.mark.gpu
def test_pr_tool_end_to_end(dataset):
    g, ups, graph, upd, sizes, tmp = dataset
    out = tmp / "ranks.txt"
    r = run("pr", f"--graphfile={graph}", f"--updatefile={upd}", f"--update_size={sizes}", "--check=true",
            "--error=1e-6", f"--output={out}")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr
    assert len(re.findall(r"\[PR-CHECK\] stage=batch batch=\d+ passed", r.stdout)) == 3
    assert "[PR-CHECK] stage=final" in r.stdout and "Overall: Test passed" in r.stdout
    ranks = np.loadtxt(out)[:, 1]
    x, _ = _oracle_final(g, ups, None).pagerank(1e-14, 50000)
    assert np.max(np.abs(ranks - x) / x) < 1e-3  # --error=1e-6 absolute residual threshold
