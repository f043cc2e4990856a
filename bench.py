#!/usr/bin/env python
"""Benchmark: incremental SSSP update stream on B200.

Workload (default): R-MAT scale 24 (16.8M vertices, ~250M directed edges
after dedup, a/b/c = 0.57/0.19/0.19, seeded), SSSP from vertex 0 with the
reference's implicit weight (u+v)%128+1, HBM edge-cache budget 1 GiB (the
rest of the adjacency is read zero-copy from pinned host memory), batches of
100k deletions + 100k insertions.  One step = one update batch (deletion
phase + insertion phase, with all repairs), as the reference's per-batch
timer measures it (samples/hybrid_sssp/hybrid_sssp.cu:417-524).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm prints one JSON line: `value` = update batches/s with the batch
arrays resident in HBM (device time from CUDA events on the engine stream),
`e2e` = the same through the C ABI with host arrays (host->device copy of the
batch and an 8-byte result digest read back inside the timed region).  The
reference arm times the reference's CPU path on the host cores: its own
SourceLocalChunkStore batch maintenance (compiled from its sources into
oracle/_ref) plus the from-scratch FIFO recompute its --check uses
(restated in oracle/).  N>1 runs independent replicas (no collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "GTEPS + batch latency p50/p99, batched vs plain on 1 B200 (exact; PR 1e-5)"
UNIT = "batches/s"
WORKLOAD = "incremental SSSP, RMAT s24 ef16, cache 1 GiB, 100k del + 100k ins per batch"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--scale", type=int, default=24)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--batch", type=int, default=100_000, help="deletions and insertions per batch")
    p.add_argument("--cache", type=float, default=1.0, help="HBM edge-cache budget, GiB")
    p.add_argument("--algo", default="sssp", choices=["bfs", "sssp", "cc"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-budget-s", type=float, default=150.0,
                   help="reference arm: stop timing after this much CPU time")
    p.add_argument("--workload", default="stream", choices=["stream", "msbfs", "mssssp"],
                   help="stream: the update-stream benchmark (default); msbfs/mssssp: 64-source queries "
                        "on a symmetric R-MAT graph, batched bitmask waves vs the per-source form")
    p.add_argument("--sources", type=int, default=64)
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_workload(args, nbatches):
    from coincgraph_b200 import gen

    t0 = time.perf_counter()
    g, h = gen.rmat(args.scale, args.edge_factor, keep_handle=True)
    t1 = time.perf_counter()
    ups = gen.updates(h, [args.batch] * nbatches, [args.batch] * nbatches, seed=gen.UPDATE_SEED_BASE + 2)
    t2 = time.perf_counter()
    return g, ups, {"gen_graph_s": round(t1 - t0, 2), "gen_updates_s": round(t2 - t1, 2)}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, flag in zip(names, parts[5:9]):
                    if flag.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def link_peak_gbs(torch, dev):
    """Pinned host -> HBM copy bandwidth (the host link's usable peak)."""
    src = torch.empty(256 << 20, dtype=torch.uint8).pin_memory()
    dst = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(2):
        dst.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        dst.copy_(src, non_blocking=True)
        b.record()
        b.synchronize()
        best = max(best, src.numel() / (a.elapsed_time(b) * 1e-3) / 1e9)
    return best


# Algorithmic bytes per unit of work for the traversal stages (our layout):
# per expanded row a 16-byte descriptor + 8-byte packed state + 4-byte queue
# entry; per scanned edge a 4-byte adjacency entry (billed to HBM when it
# comes from the edge cache or the device arena, to the host link otherwise)
# + an 8-byte state read; per hit (relaxation, invalidation or pull update)
# an 8-byte state write + 4-byte stamp + 4-byte queue append.
ROW_BYTES, EDGE_STATE_BYTES, ADJ_BYTES, HIT_BYTES = 28, 8, 4, 16


def stage_roofline(prof_stage, hbm_peak, link_peak):
    edges, cached = prof_stage["edges"], prof_stage["edges_cached"]
    hbm = prof_stage["rows"] * ROW_BYTES + edges * EDGE_STATE_BYTES + cached * ADJ_BYTES + prof_stage["hits"] * HIT_BYTES
    link = (edges - cached) * ADJ_BYTES
    t = prof_stage["ms"] * 1e-3
    if t <= 0:
        return None
    t_roof = hbm / (hbm_peak * 1e9) + link / (link_peak * 1e9)
    return {"hbm_bytes": hbm, "link_bytes": link, "seconds": t, "achieved_hbm_gbs": hbm / t / 1e9,
            "achieved_link_gbs": link / t / 1e9, "t_roof_s": t_roof, "frac_combined": t_roof / t}


def cpu_baseline(g, ups, args, batch_index):
    """Reference CPU path on one batch: its SourceLocalChunkStore maintenance
    (compiled from the reference sources) + the FIFO recompute of --check."""
    import oracle

    workers = min(os.cpu_count() or 1, 256)
    og = oracle.Graph(g.n, g.xadj, g.adj)
    mode = {"bfs": oracle.BFS, "sssp": oracle.SSSP, "cc": oracle.CC}[args.algo]
    du, dv, au, av = ups.batch(batch_index)
    t_mut = None
    kind = "port"
    if oracle.ref_available():
        ref = oracle.RefStore(g.n, g.xadj, g.adj, workers=workers)
        t0 = time.perf_counter()
        ref.apply(du, dv, au, av)
        t_mut = time.perf_counter() - t0
        kind = "reference"
        del ref
    t0 = time.perf_counter()
    og.delete(du, dv)
    og.add(au, av)
    t_port = time.perf_counter() - t0
    if t_mut is None:
        t_mut = t_port
    t0 = time.perf_counter()
    if args.algo == "cc":
        og.cc()
    else:
        og.sssp(0, mode)
    t_solve = time.perf_counter() - t0
    total = t_mut + t_solve
    return {
        "value": 1.0 / total, "unit": UNIT, "cores": workers, "kind": kind,
        "sample": (f"1 batch ({len(du)} del + {len(au)} ins): reference SourceLocalChunkStore maintenance "
                   f"({workers} workers, {t_mut:.3f} s) + single-thread FIFO {args.algo} recompute "
                   f"({t_solve:.2f} s)"),
    }


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle

    nb = args.warmup + args.steps
    g, ups, setup = make_workload(args, nb)
    workers = min(os.cpu_count() or 1, 256)
    mode = {"bfs": oracle.BFS, "sssp": oracle.SSSP, "cc": oracle.CC}[args.algo]
    have_ref = oracle.ref_available()
    ref = oracle.RefStore(g.n, g.xadj, g.adj, workers=workers) if have_ref else None
    og = oracle.Graph(g.n, g.xadj, g.adj)
    times = []
    spent = 0.0
    for i in range(nb):
        du, dv, au, av = ups.batch(i)
        t0 = time.perf_counter()
        if ref is not None:
            ref.apply(du, dv, au, av)
        t1 = time.perf_counter()
        og.delete(du, dv)  # keeps the recompute's graph in step (not timed when the reference store ran)
        og.add(au, av)
        t2 = time.perf_counter()
        if i < args.warmup:
            continue  # warm-up: maintenance only
        if args.algo == "cc":
            og.cc()
        else:
            og.sssp(0, mode)
        t3 = time.perf_counter()
        step = (t1 - t0 if ref is not None else t2 - t1) + (t3 - t2)
        times.append(step)
        spent += step
        if spent > args.ref_budget_s:
            break
    mean = sum(times) / len(times)
    value = 1.0 / mean
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": WORKLOAD if args.scale == 24 else f"{WORKLOAD} (scale {args.scale})",
                   "scale": args.scale, "batch": args.batch, "algo": args.algo, "setup": setup},
        "p50_ms": statistics.median(times) * 1e3, "p99_ms": float(np.percentile(np.array(times) * 1e3, 99)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "reference" if have_ref else "port",
                         "sample": (f"{len(times)} timed batches (of {args.steps} requested, CPU-time budget "
                                    f"{args.ref_budget_s:.0f} s): reference SourceLocalChunkStore maintenance with "
                                    f"{workers} workers + single-thread FIFO {args.algo} recompute")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    from coincgraph_b200 import Engine

    nb = args.warmup + 2 * args.steps
    g, ups, setup = make_workload(args, nb)
    t0 = time.perf_counter()
    eng = Engine(args.algo, device=local, source=0, cache_gib=args.cache, max_batch=args.batch)
    eng.load_csr(g.n, g.xadj, g.adj)
    t1 = time.perf_counter()
    eng.init()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    setup.update({"load_s": round(t1 - t0, 2), "init_s": round(t2 - t1, 2)})
    info = eng.info()

    def dev_batch(i):
        return [torch.from_numpy(x.astype(np.int32)).to(dev) for x in ups.batch(i)]

    batches = [dev_batch(i) for i in range(args.warmup + args.steps)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for i in range(args.warmup):
        eng.apply_batch_device(*batches[i])

    eng.profile(True)
    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    ms, edges, launches, stats = [], 0, 0, []
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        s = eng.apply_batch_device(*batches[args.warmup + k])
        ms.append(s.ms_delete + s.ms_insert + s.ms_cache)
        edges += s.edges_scanned
        launches += s.kernel_launches
        stats.append(s.as_dict())
    barrier()
    clocks = sampler.stop()
    prof = eng.profile_read()
    eng.profile(False)
    total_s = sum(ms) * 1e-3

    # e2e: host arrays through cig_apply_batch + 8-byte digest read-back.
    e2e_t, h2d = [], 0
    for k in range(args.steps):
        du, dv, au, av = ups.batch(args.warmup + args.steps + k)
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        eng.apply_batch(du, dv, au, av)
        eng.digest()
        e2e_t.append(time.perf_counter() - t)
        h2d += 4 * (len(du) + len(dv) + len(au) + len(av))
    e2e_total = sum(e2e_t)

    if world > 1:
        t = torch.tensor([total_s, e2e_total], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_s, e2e_total = float(t[0]), float(t[1])

    hbm_peak, peak_kind = load_peaks()
    link_peak = link_peak_gbs(torch, dev)
    stages = {}
    for name in ("group", "mutate", "mutate_rev", "add", "add_rev", "seed", "inval", "pull", "push"):
        stages[name] = {"ms_per_batch": prof[name]["ms"] / args.steps, "launches": prof[name]["launches"]}
    trav = {n: stage_roofline(prof[n], hbm_peak, link_peak) for n in ("inval", "pull", "push")}
    dominant = max(("push", "inval", "pull"), key=lambda n: prof[n]["ms"])
    rf = trav[dominant]
    roofline = None
    if rf:
        roofline = {
            "kernel": f"{dominant}_closure" if dominant != "pull" else "pull_repair",
            "bound": "hbm", "achieved": rf["achieved_hbm_gbs"], "peak": hbm_peak, "unit": "GB/s",
            "frac": rf["achieved_hbm_gbs"] / hbm_peak, "traffic": None,
            "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
            "hbm_bytes_per_launch": rf["hbm_bytes"] / max(prof[dominant]["launches"], 1),
            "link_bytes_per_launch": rf["link_bytes"] / max(prof[dominant]["launches"], 1),
            "achieved_link_gbs": rf["achieved_link_gbs"], "link_peak_gbs": link_peak,
            "frac_of_combined_roofline": rf["frac_combined"],
        }

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline(g, ups, args, args.warmup)
            except Exception as e:  # reported, not fatal
                cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": f"failed: {e}"}
        value = world * args.steps / total_s
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": WORKLOAD if args.scale == 24 and args.batch == 100_000 else
                       f"incremental {args.algo.upper()}, RMAT s{args.scale} ef{args.edge_factor}, cache "
                       f"{args.cache} GiB, {args.batch} del + {args.batch} ins per batch",
                       "algo": args.algo, "vertices": g.n, "edges": g.m, "cache_gib": args.cache,
                       "segments_resident": info["segments_resident"], "segments_total": info["segments_total"],
                       "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                       "setup": setup},
            "gteps": edges / total_s / 1e9 * world if total_s else None,
            "p50_ms": statistics.median(ms), "p99_ms": float(np.percentile(ms, 99)),
            "updates_per_s": value * 2 * args.batch,
            "e2e": {"value": world * args.steps / e2e_total, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": 8 + 144, "p50_ms": statistics.median(e2e_t) * 1e3},
            "roofline": roofline,
            "stages": stages,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches,
            "mean_batch": {k: float(np.mean([s[k] for s in stats])) for k in
                           ("affected", "seeds", "rounds", "edges_scanned", "edges_scanned_cached",
                            "changed_sources", "relocated_rows", "missing_deletes")},
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def run_queries(args):
    """64 sources uniform over vertices of degree > 0 on a symmetric R-MAT
    graph: one step = all sources answered (k x n results in HBM)."""
    import torch

    from coincgraph_b200 import Engine, gen

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    algo = "bfs" if args.workload == "msbfs" else "sssp"
    t0 = time.perf_counter()
    g = gen.rmat(args.scale, args.edge_factor, symmetric=True)
    t1 = time.perf_counter()
    rng = np.random.default_rng(0xC01C1003)
    deg = np.diff(g.xadj.astype(np.int64))
    src = rng.choice(np.flatnonzero(deg > 0), size=args.sources, replace=False).astype(np.uint32)
    eng = Engine(algo, device=local, source=int(src[0]), cache_gib=args.cache)
    eng.load_csr(g.n, g.xadj, g.adj)
    t2 = time.perf_counter()
    out = torch.empty((args.sources, g.n), dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def timed(width, steps):
        res = []
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            res.append(eng.query_device(algo, src, out, width=width))
        return res

    timed(64, args.warmup)
    sampler = ClockSampler(local)
    sampler.start()
    batched = timed(64, args.steps)
    clocks = sampler.stop()
    check = out.cpu()
    plain = timed(1, 1)  # per-source form: 64 waves of one source each
    same = bool(torch.equal(check, out.cpu()))
    ms = [r["ms"] for r in batched]
    total_s = sum(ms) * 1e-3
    edges = sum(r["edges_scanned"] for r in batched)
    line = {
        "metric": f"multi-source {algo.upper()} queries", "value": args.steps / total_s, "unit": "queries-of-64/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps,
        "higher_is_better": True, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"{args.sources}-source {algo.upper()}, symmetric RMAT s{args.scale} ef{args.edge_factor}",
                   "vertices": g.n, "edges": g.m, "cache_gib": args.cache, "l2": "flushed between steps",
                   "setup": {"gen_graph_s": round(t1 - t0, 2), "load_s": round(t2 - t1, 2)}},
        "gteps_edge_scans": edges / total_s / 1e9,
        "gteps_source_edges": sum(r["source_edges"] for r in batched) / total_s / 1e9,
        "plain_per_source_ms": plain[0]["ms"], "batched_ms": statistics.median(ms),
        "speedup_vs_plain": plain[0]["ms"] / statistics.median(ms), "plain_equals_batched": same,
        "per_step": {k: batched[-1][k] for k in ("edges_scanned", "edges_scanned_cached", "rows_expanded",
                                                 "source_edges", "rounds", "waves", "kernel_launches")},
        "plain_edges_scanned": plain[0]["edges_scanned"], "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    eng.close()


def main():
    args = parse_args()
    if args.workload != "stream":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "query workloads have no reference CPU arm"}))
            return
        run_queries(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
