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
`e2e` = the same through the C ABI with host arrays in page-locked memory
(host->device copy of the batch and an 8-byte result digest read back inside
the timed region; the pageable-array form is reported beside it).  The
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
    p.add_argument("--no-parity", action="store_true", help="skip the oracle replay after the timed region")
    p.add_argument("--no-extras", action="store_true",
                   help="stream: skip the uneven batched-vs-plain and served measurements after the main line")
    p.add_argument("--index-budget", type=float, default=0.0,
                   help="GiB for the two position-index tables (0: a quarter of free device memory each)")
    p.add_argument("--served-requests", type=int, default=200, help="default line: served-stream requests")
    p.add_argument("--served-rate", type=float, default=40.0, help="default line: served Poisson rate, requests/s")
    p.add_argument("--ref-budget-s", type=float, default=150.0,
                   help="reference arm: stop timing after this much CPU time")
    p.add_argument("--workload", default="stream",
                   choices=["stream", "road", "msbfs", "mssssp", "uneven", "served", "pr"],
                   help="stream: the update-stream benchmark (default); msbfs/mssssp: 64-source queries "
                        "on a symmetric R-MAT graph, batched bitmask waves vs the per-source form; uneven: "
                        "batches of log-uniform sizes, batched form (one sync) vs one call per batch; road: the "
                        "update stream on a high-diameter grid graph (--side) with local insertions")
    p.add_argument("--side", type=int, default=2048, help="road: grid side (side^2 vertices)")
    p.add_argument("--requests", type=int, default=400, help="served: requests in the stream")
    p.add_argument("--update-frac", type=float, default=0.1, help="served: share of update requests")
    p.add_argument("--rate", type=float, default=0.0, help="served: Poisson arrival rate, requests/s (0: all at once)")
    p.add_argument("--uneven-batches", type=int, default=20)
    p.add_argument("--uneven-max", type=int, default=1_000_000)
    p.add_argument("--sources", type=int, default=64)
    return p.parse_args()


def max_over_ranks(values, device):
    """Replica timing: every rank's timed totals, reduced to the maximum over
    ranks (the job is as slow as its slowest replica).  NCCL on the GPUs in
    the bench; the same code runs over gloo on CPU in the tests."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def replica_value(world, steps, total_s):
    """Whole-job batches/s of `world` independent replicas that each applied
    `steps` batches, timed as the maximum over ranks (weak scaling)."""
    return world * steps / total_s


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
    if args.workload == "road":
        g = gen.grid(args.side)
        t1 = time.perf_counter()
        ups = gen.local_updates(g, args.side, [args.batch] * nbatches, [args.batch] * nbatches,
                                seed=gen.UPDATE_SEED_BASE + 7)
        t2 = time.perf_counter()
        return g, ups, {"gen_graph_s": round(t1 - t0, 2), "gen_updates_s": round(t2 - t1, 2)}
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


# Flat deletion scan: per row entry read a 4-byte adjacency word (HBM when
# its segment is resident, else the host link); per deletion key an 8-byte
# key read and a 4-byte first-match word.
DEL_KEY_BYTES = 12
# Whole-batch key sort, per key (4 keys per update pair): 8 B written by
# make_keys_batch, 7 radix passes of 8 B read + 8 B written, 20 B by
# unpack_keys_batch (key read, key + flag written), 8 B by the flag scan and
# 16 B by group_scatter_batch.
SORT_KEY_BYTES = 8 + 7 * 16 + 20 + 8 + 16
# Deletion phase per request and arena (mutate, mutate_rev; the row scan is
# billed to del_scan): key 8 B + descriptor 16 B (del_classify), index probe
# 16 B read + 8 B written (del_index), tombstone 4 B + first match 4 B
# (del_apply), descriptor 16 B written (del_finish).
DEL_REQ_BYTES = 8 + 16 + 24 + 8 + 16
# Addition phase per request and arena (add, add_rev): key 8 B + plan 8 B +
# descriptor 16 B read and 16 B written + value 4 B + index entry 16 B; per
# entry of a relocated row 4 B read + 4 B written.
ADD_REQ_BYTES = 8 + 8 + 32 + 4 + 16
MOVE_ENTRY_BYTES = 8
# Segment-table service: a loaded or evicted 64 KiB segment crosses the host
# link once and is read or written once in HBM.
SEG_BYTES = 65536

# Kernels of each profiler stage (the stage time covers all of them).
STAGE_KERNELS = {
    "group": "make_keys_batch + CUB radix sort + unpack_keys_batch + scan + group_scatter_batch",
    "mutate": "del_classify, del_chunk_map, del_scan, del_index, del_apply, del_finish, mutate_delete(_big), "
              "compact_rows (forward rows)",
    "mutate_rev": "the same on the reverse rows",
    "del_scan": "del_scan + del_index (inside mutate and mutate_rev)",
    "seed": "seed_deletions, seed_insertions",
    "inval": "inval_closure",
    "pull": "reset_affected, pull_repair, pull_deferred, enqueue_affected",
    "push": "push_closure",
    "add": "plan_add, alloc_classes, seg_assign_new, mutate_add, mutate_add_big (forward rows)",
    "add_rev": "the same on the reverse rows",
    "cache": "seg_rescore, seg_plan, seg_pick, seg_evict, seg_admit",
}

# ncu DRAM bytes (read + write) per algorithmic HBM byte, measured on a
# smaller case of the same kernel (the full-size launch is too large for a
# multi-pass capture under the capture-size rule).  The bench scales the
# ratio by this run's algorithmic bytes: an estimate, labelled as such.
TRAFFIC_RATIO = {
    "push_closure": (6.58, "ncu capture of push_closure, SSSP R-MAT s22 cache 4 GiB, 100k+100k batch, "
                           "22.8 MB DRAM against 3.46 MB algorithmic"),
    "inval_closure": (5.97, "ncu capture of inval_closure, SSSP R-MAT s22 cache 4 GiB, 100k+100k batch, "
                            "14.2 MB DRAM against 2.38 MB algorithmic"),
}


def stage_bytes(name, st):
    """(HBM bytes, host-link bytes) of a profiler stage from its counters."""
    edges, cached, rows, hits = st["edges"], st["edges_cached"], st["rows"], st["hits"]
    if name == "del_scan":
        return cached * ADJ_BYTES + hits * DEL_KEY_BYTES, (edges - cached) * ADJ_BYTES
    if name in ("inval", "pull", "push"):
        return (rows * ROW_BYTES + edges * EDGE_STATE_BYTES + cached * ADJ_BYTES + hits * HIT_BYTES,
                (edges - cached) * ADJ_BYTES)
    if name == "group":
        return hits * SORT_KEY_BYTES, 0
    if name in ("mutate", "mutate_rev"):
        return hits * DEL_REQ_BYTES, 0
    if name in ("add", "add_rev"):
        return hits * ADD_REQ_BYTES + edges * MOVE_ENTRY_BYTES, 0
    if name == "cache":
        return rows * SEG_BYTES, rows * SEG_BYTES
    return 0, 0


def stage_roofline(name, st, hbm_peak, link_peak, batches):
    t = st["ms"] * 1e-3
    if t <= 0:
        return None
    hbm, link = stage_bytes(name, st)
    t_roof = hbm / (hbm_peak * 1e9) + link / (link_peak * 1e9)
    return {"kernels": STAGE_KERNELS.get(name, name), "ms_per_batch": st["ms"] / batches,
            "launches_per_batch": st["launches"] / batches, "hbm_bytes_per_batch": hbm / batches,
            "link_bytes_per_batch": link / batches, "achieved_hbm_gbs": hbm / t / 1e9,
            "achieved_link_gbs": link / t / 1e9, "frac_hbm": hbm / t / 1e9 / hbm_peak,
            "frac_combined": t_roof / t}


def stream_config(args, g):
    """The workload keys both arms report (identical dicts for one run)."""
    if args.workload == "stream" and args.scale == 24 and args.batch == 100_000 and args.algo == "sssp":
        name = WORKLOAD
    else:
        name = (f"incremental {args.algo.upper()}, "
                + (f"road-like grid {args.side}x{args.side}" if args.workload == "road" else
                   f"RMAT s{args.scale} ef{args.edge_factor}")
                + f", cache {args.cache} GiB, {args.batch} del + {args.batch} ins per batch")
    return {"workload": name, "algo": args.algo, "scale": args.scale if args.workload != "road" else None,
            "vertices": g.n, "edges": g.m, "batch": args.batch, "cache_gib": args.cache, "source": 0,
            "l2": "GPU arm: L2 flushed between steps (256 MiB write)", "parallelism": "replicas"}


def oracle_parity(g, ups, applied, eng, args):
    """Replay every batch the engine applied, in order, on the oracle (the
    CPU restatement of the reference's row mutation and --check solvers),
    outside every timer, and compare the engine's final values and rows with
    the oracle's exactly."""
    import oracle

    t0 = time.perf_counter()
    og = oracle.Graph(g.n, g.xadj, g.adj)
    missing = 0
    for i in range(applied):
        du, dv, au, av = ups.batch(i)
        missing += og.delete(du, dv)
        og.add(au, av)
    mode = {"bfs": oracle.BFS, "sssp": oracle.SSSP, "cc": oracle.CC}[args.algo]
    want = og.cc() if args.algo == "cc" else og.sssp(0, mode)
    got = eng.values()
    diff = int(np.count_nonzero(got != want))
    xadj, adj = eng.export_csr()
    xo, ao = og.export()
    rows_ok = bool(np.array_equal(xadj, xo) and np.array_equal(adj, ao))
    del og, xadj, adj, xo, ao
    return {"values_equal": diff == 0, "values_differing": diff, "rows_equal": rows_ok,
            "batches_replayed": applied, "reached": int(np.count_nonzero(want != oracle.INF)),
            "oracle": f"oracle/ FIFO label-correcting {args.algo} (restated reference --check) after replaying "
                      "every applied batch on the restated chunk-store mutation",
            "seconds": round(time.perf_counter() - t0, 1)}


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
        "config": stream_config(args, g), "setup": setup,
        "p50_ms": statistics.median(times) * 1e3, "p99_ms": float(np.percentile(np.array(times) * 1e3, 99)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "reference" if have_ref else "port",
                         "sample": (f"{len(times)} timed batches (of {args.steps} requested, CPU-time budget "
                                    f"{args.ref_budget_s:.0f} s): reference SourceLocalChunkStore maintenance with "
                                    f"{workers} workers + single-thread FIFO {args.algo} recompute")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    """The update stream: W warm-up batches, K timed batches from HBM (stage
    profiler off), K end-to-end batches from host arrays, then outside every
    timer a profiled pass for the per-stage breakdown and rooflines, the
    oracle replay of every applied batch, and (N=1, default workload) the
    uneven stream batched vs plain and the served Poisson stream."""
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    from coincgraph_b200 import Engine

    nprof = min(args.steps, 10)
    npage = min(args.steps, 10)
    nb = args.warmup + 2 * args.steps + npage + nprof
    g, ups, setup = make_workload(args, nb)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    torch.cuda.synchronize()
    free0, torch0 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_reserved(dev)
    t0 = time.perf_counter()
    eng = Engine(args.algo, device=local, source=0, cache_gib=args.cache, max_batch=args.batch,
                 index_budget_gib=args.index_budget)
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
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for i in range(args.warmup):
        eng.apply_batch_device(*batches[i])
    memory = eng.memory()
    # cudaMemGetInfo difference since before the engine, less torch's own pool
    memory["measured_device_bytes"] = (free0 - torch.cuda.mem_get_info(dev)[0]
                                       - (torch.cuda.memory_reserved(dev) - torch0))

    sampler = ClockSampler(local)
    sampler.start()
    barrier()
    ms, edges, launches, replays, stats = [], 0, 0, 0, []
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        s = eng.apply_batch_device(*batches[args.warmup + k])
        ms.append(s.ms_delete + s.ms_insert + s.ms_cache)
        edges += s.edges_scanned
        launches += s.kernel_launches
        replays += s.graph_replays
        stats.append(s.as_dict())
    barrier()
    clocks = sampler.stop()
    total_s = sum(ms) * 1e-3
    del batches

    # e2e: host arrays through cig_apply_batch + 8-byte digest read-back.
    # The step's four arrays sit in page-locked host memory when the timed
    # region starts (the engine DMAs them directly); the same batches from
    # pageable arrays (copied through the engine's pinned staging) follow.
    def pinned_u32(a):
        t = torch.from_numpy(np.ascontiguousarray(a).astype(np.int32, copy=False)).pin_memory()
        return t, t.numpy().view(np.uint32)

    e2e_t, pageable_t, h2d = [], [], 0
    for k in range(args.steps):
        arrays = ups.batch(args.warmup + args.steps + k)
        held = [pinned_u32(a) for a in arrays]
        du, dv, au, av = (h[1] for h in held)
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        eng.apply_batch(du, dv, au, av)
        eng.digest()
        e2e_t.append(time.perf_counter() - t)
        h2d += 4 * (len(du) + len(dv) + len(au) + len(av))
    e2e_total = sum(e2e_t)
    # not part of the headline: the pageable-input form of the same API
    for k in range(npage):
        du, dv, au, av = (np.ascontiguousarray(a, dtype=np.uint32) for a in ups.batch(args.warmup + 2 * args.steps + k))
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        eng.apply_batch(du, dv, au, av)
        eng.digest()
        pageable_t.append(time.perf_counter() - t)

    if world > 1:
        total_s, e2e_total = max_over_ranks([total_s, e2e_total], dev)

    # Profiled pass (not timed): per-stage device times with CUDA events.
    eng.profile(True)
    for k in range(nprof):
        flush.zero_()
        torch.cuda.synchronize()
        eng.apply_batch_device(*dev_batch(args.warmup + 2 * args.steps + npage + k))
    prof = eng.profile_read()
    eng.profile(False)

    hbm_peak, peak_kind = load_peaks()
    link_peak = link_peak_gbs(torch, dev)
    stages = {n: stage_roofline(n, prof[n], hbm_peak, link_peak, nprof) for n in STAGE_KERNELS}
    stages = {n: v for n, v in stages.items() if v}
    # The dominant kernel: of the stages that are one kernel each (push:
    # push_closure, inval: inval_closure), the one with the most time; they
    # are also the two largest single launches of the batch in an ncu launch
    # list of this workload.  The other stages are chains of 2-10 kernels,
    # and those of the two arenas overlap on two streams.
    dominant = max((n for n in ("push", "inval") if n in stages), key=lambda n: stages[n]["ms_per_batch"])
    main_kernel = {"push": "push_closure", "inval": "inval_closure"}[dominant]
    rf = stages[dominant]
    hbm_launch = rf["hbm_bytes_per_batch"] * nprof / max(prof[dominant]["launches"], 1)
    ratio = TRAFFIC_RATIO.get(main_kernel)
    roofline = {
        "kernel": main_kernel, "stage": dominant, "stage_kernels": rf["kernels"],
        "bound": "hbm", "achieved": rf["achieved_hbm_gbs"], "peak": hbm_peak, "unit": "GB/s",
        "frac": rf["frac_hbm"],
        "traffic": ratio[0] * hbm_launch if ratio else None,
        "traffic_source": (f"estimate: {ratio[1]}, {ratio[0]:.2f} x algorithmic HBM bytes, scaled to this "
                           "launch's algorithmic bytes") if ratio else None,
        "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
        "hbm_bytes_per_launch": hbm_launch,
        "link_bytes_per_launch": rf["link_bytes_per_batch"] * nprof / max(prof[dominant]["launches"], 1),
        "achieved_link_gbs": rf["achieved_link_gbs"], "link_peak_gbs": link_peak,
        "frac_of_combined_roofline": rf["frac_combined"],
        "timing": f"CUDA events around the stage on the engine stream, profiled pass of {nprof} batches",
    }

    parity = None
    if rank == 0 and not args.no_parity:
        try:
            parity = oracle_parity(g, ups, args.warmup + 2 * args.steps + npage + nprof, eng, args)
        except Exception as e:  # reported in the line, not fatal
            parity = {"values_equal": False, "rows_equal": False, "error": str(e)}
    eng.close()
    del eng
    torch.cuda.synchronize()

    extra = {}
    if rank == 0 and world == 1 and args.workload == "stream" and not args.no_extras:
        try:
            extra["batched_vs_plain"] = uneven_stream(args, local, max_size=args.uneven_max, count=args.uneven_batches)
        except Exception as e:  # reported in the line, not fatal
            extra["batched_vs_plain"] = {"error": str(e)}
        try:
            extra["served"] = served_stream(args, local, requests=args.served_requests, rate=args.served_rate)
        except Exception as e:
            extra["served"] = {"error": str(e)}
        try:  # capacity: every request queued at once
            extra["served_saturated"] = served_stream(args, local, requests=args.served_requests, rate=0.0)
        except Exception as e:
            extra["served_saturated"] = {"error": str(e)}

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline(g, ups, args, args.warmup)
            except Exception as e:  # reported, not fatal
                cpu = {"value": None, "unit": UNIT, "cores": None, "kind": "port", "sample": f"failed: {e}"}
        value = replica_value(world, args.steps, total_s)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": stream_config(args, g), "setup": setup,
            "engine": {"segments_resident": info["segments_resident"], "segments_total": info["segments_total"],
                       "graphs": "batch shapes seen twice are replayed from CUDA graphs",
                       "graph_replays_per_batch": replays / args.steps},
            "device_memory": memory,
            "parity": parity["values_equal"] and parity["rows_equal"] if parity else None,
            "parity_detail": parity,
            "gteps": edges / total_s / 1e9 * world if total_s else None,
            "p50_ms": statistics.median(ms), "p99_ms": float(np.percentile(ms, 99)),
            "updates_per_s": value * 2 * args.batch,
            "e2e": {"value": world * args.steps / e2e_total, "unit": UNIT, "h2d_bytes_per_step": h2d // args.steps,
                    # the 8-byte digest + the 344-byte device status word read by every call
                    "d2h_bytes_per_step": 8 + 344, "p50_ms": statistics.median(e2e_t) * 1e3,
                    "inputs": "page-locked host arrays, copied to the device by DMA inside the timed region",
                    "pageable_inputs": {"value": len(pageable_t) / sum(pageable_t) if pageable_t else None,
                                        "p50_ms": statistics.median(pageable_t) * 1e3 if pageable_t else None,
                                        "note": "the same call with pageable arrays (copied through the "
                                                "engine's pinned staging buffer), other batches"}},
            "roofline": roofline,
            "stages": stages,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": launches,
            "mean_batch": {k: float(np.mean([s[k] for s in stats])) for k in
                           ("affected", "seeds", "rounds", "edges_scanned", "edges_scanned_cached",
                            "changed_sources", "relocated_rows", "missing_deletes", "cache_segments_loaded",
                            "cache_segments_evicted", "kernel_launches")},
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
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


def uneven_stream(args, local, max_size, count):
    """Update batches with sizes log-uniform in [1k, max_size] (half
    deletions, half insertions), each form on a freshly loaded engine: the
    plain form (direct launches, CIG_FLAG_NO_GRAPHS; one cig_apply_batch_device
    per batch and a digest read after each) against the batched form (one
    cig_apply_batches_device call for all batches, shapes seen twice replayed
    from CUDA graphs, per-batch digests computed on the device).  The
    per-batch value digests of the two forms must agree."""
    import torch

    from coincgraph_b200 import Engine, gen
    from coincgraph_b200.engine import FLAG_NO_GRAPHS

    dev = torch.device("cuda", local)
    rng = np.random.default_rng(0xC01C1003)
    sizes = np.exp(rng.uniform(np.log(1000), np.log(max_size), count)).astype(np.int64)
    symmetric = args.algo == "cc"
    # symmetric streams come in (u,v)+(v,u) pairs: even phase sizes
    half = np.maximum(sizes // 4 * 2, 2) if symmetric else np.maximum(sizes // 2, 1)
    g, h = gen.rmat(args.scale, args.edge_factor, keep_handle=True, symmetric=symmetric)
    ups = gen.updates(h, half, half, seed=gen.UPDATE_SEED_BASE + 3, symmetric=symmetric)
    del h
    batches = [[torch.from_numpy(x.astype(np.int32)).to(dev) for x in ups.batch(i)] for i in range(len(sizes))]
    res = {}
    for form in ("plain", "batched"):
        eng = Engine(args.algo, device=local, source=0, cache_gib=args.cache, max_batch=int(half.max()),
                     flags=FLAG_NO_GRAPHS if form == "plain" else 0)
        eng.load_csr(g.n, g.xadj, g.adj)
        eng.init()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if form == "plain":
            stats, digests = [], []
            for b in batches:
                stats.append(eng.apply_batch_device(*b))
                digests.append(eng.digest())
        else:
            stats, digests = eng.apply_batches_device(batches)
        wall = time.perf_counter() - t0
        dev_ms = [s.ms_delete + s.ms_insert + s.ms_cache for s in stats]
        res[form] = {"wall_s": wall, "digests": digests, "batch_ms": dev_ms,
                     "launches": sum(s.kernel_launches for s in stats),
                     "graph_replays": sum(s.graph_replays for s in stats)}
        eng.close()
        del eng
    same = res["plain"]["digests"] == res["batched"]["digests"]
    per_batch = {form: [round(x, 3) for x in res[form]["batch_ms"]] for form in res}
    return {
        "workload": f"{args.algo.upper()} RMAT s{args.scale} ef{args.edge_factor}{' symmetric' if symmetric else ''}, "
                    f"{len(sizes)} batches log-uniform [1k, {max_size}] (half del, half ins), cache {args.cache} GiB",
        "batched_batches_per_s": len(sizes) / res["batched"]["wall_s"],
        "plain_batches_per_s": len(sizes) / res["plain"]["wall_s"],
        "ratio": res["plain"]["wall_s"] / res["batched"]["wall_s"], "digests_equal": same,
        "timing": "host wall clock of the whole stream, synchronised at both ends",
        "sizes": sizes.tolist(), "batch_device_ms": per_batch,
        "plain": {"wall_s": res["plain"]["wall_s"], "p50_ms": statistics.median(res["plain"]["batch_ms"]),
                  "p99_ms": float(np.percentile(res["plain"]["batch_ms"], 99)), "launches": res["plain"]["launches"]},
        "batched": {"wall_s": res["batched"]["wall_s"], "launches": res["batched"]["launches"],
                    "graph_replays": res["batched"]["graph_replays"],
                    "p50_ms": statistics.median(res["batched"]["batch_ms"]),
                    "p99_ms": float(np.percentile(res["batched"]["batch_ms"], 99)),
                    "device_ms_sum": sum(res["batched"]["batch_ms"])},
    }


def run_uneven(args):
    import torch

    _, _, local = dist_env()
    torch.cuda.set_device(local)
    r = uneven_stream(args, local, args.uneven_max, args.uneven_batches)
    line = {"metric": "batches/s, batched form vs plain per-batch form", "unit": "batches/s",
            "value": r["batched_batches_per_s"], "n_gpus": 1, "higher_is_better": True, "dtype": "u32",
            "data": "synthetic", "config": {"workload": r["workload"], "sizes": r["sizes"]}}
    line.update({k: v for k, v in r.items() if k not in ("workload", "sizes")})
    print(json.dumps(line), flush=True)


def served_stream(args, local, requests, rate):
    """A request stream (Poisson arrivals at `rate`/s, or all at once for
    rate 0) mixing update batches of log-uniform sizes in [1k, --uneven-max]
    with BFS/SSSP queries from uniform sources, served by cig_serve_* (waves,
    overlap) and by the plain sequential form (one request at a time:
    cig_apply_batch, or a one-source query), each on a freshly loaded engine.
    Reports p50/p99 latency (arrival to result) and requests/s; update
    digests must agree."""
    import torch

    from coincgraph_b200 import Engine, gen

    rng = np.random.default_rng(0xC01C1005)
    nreq = requests
    is_upd = rng.random(nreq) < args.update_frac
    nupd = int(is_upd.sum())
    sizes = np.exp(rng.uniform(np.log(1000), np.log(args.uneven_max), max(nupd, 1))).astype(np.int64)[:nupd]
    half = np.maximum(sizes // 2, 1)
    g, h = gen.rmat(args.scale, args.edge_factor, keep_handle=True)
    ups = gen.updates(h, half, half, seed=gen.UPDATE_SEED_BASE + 5)
    del h
    deg = np.diff(g.xadj.astype(np.int64))
    live = np.flatnonzero(deg > 0)
    reqs, ui = [], 0
    for i in range(nreq):
        if is_upd[i]:
            reqs.append(("update", ups.batch(ui)))
            ui += 1
        else:
            reqs.append(("bfs" if rng.random() < 0.5 else "sssp", int(rng.choice(live))))
    gaps = rng.exponential(1.0 / rate, nreq) if rate > 0 else np.zeros(nreq)
    arrive = np.cumsum(gaps)

    def make_engine():
        e = Engine("sssp", device=local, source=0, cache_gib=args.cache, max_batch=int(half.max()) if nupd else 0)
        e.load_csr(g.n, g.xadj, g.adj)
        e.init()
        torch.cuda.synchronize()
        return e

    out = {}
    # plain sequential form: one request at a time, in arrival order
    eng = make_engine()
    dev_out = torch.empty((1, g.n), dtype=torch.int32, device=torch.device("cuda", local))
    lat, digests = [], []
    t0 = time.perf_counter()
    for (kind, x), ta in zip(reqs, arrive):
        now = time.perf_counter() - t0
        if now < ta:
            time.sleep(ta - now)
        if kind == "update":
            eng.apply_batch(*x)
            digests.append(eng.digest())
        else:
            eng.query_device(kind, [x], dev_out, width=1)
            row = dev_out.cpu().numpy().view(np.uint32)[0]
            digests.append(int(row.astype(np.uint64).sum()))
        lat.append((time.perf_counter() - t0 - ta) * 1e3)
    out["plain"] = {"wall_s": time.perf_counter() - t0, "lat": lat}
    plain_digests = digests
    eng.close()
    del eng, dev_out
    # served form
    eng = make_engine()
    eng.serve_start()
    tickets = []
    t0 = time.perf_counter()
    for (kind, x), ta in zip(reqs, arrive):
        now = time.perf_counter() - t0
        if now < ta:
            time.sleep(ta - now)
        tickets.append(eng.submit_update(*x) if kind == "update" else eng.submit_query(kind, x))
    res = [eng.wait(t) for t in tickets]
    wall = time.perf_counter() - t0
    eng.serve_stop()
    eng.close()
    del eng
    lat_s = [r["done_ms"] - r["submit_ms"] for r in res]
    waves = [r["wave"] for (k, _), r in zip(reqs, res) if k != "update"]
    upd_ok = all(r["digest"] == d for (k, _), r, d in zip(reqs, res, plain_digests) if k == "update")
    out["served"] = {"wall_s": wall, "lat": lat_s}

    def pct(v, q):
        return float(np.percentile(v, q)) if len(v) else None

    def summary(form):
        lat = out[form]["lat"]
        ql = [x for (k, _), x in zip(reqs, lat) if k != "update"]
        ul = [x for (k, _), x in zip(reqs, lat) if k == "update"]
        return {"wall_s": out[form]["wall_s"], "requests_per_s": nreq / out[form]["wall_s"],
                "update_batches_per_s": nupd / out[form]["wall_s"],
                "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "query_p50_ms": pct(ql, 50),
                "query_p99_ms": pct(ql, 99), "update_p50_ms": pct(ul, 50), "update_p99_ms": pct(ul, 99)}

    return {
        "workload": f"RMAT s{args.scale} ef{args.edge_factor}, cache {args.cache} GiB, {nreq} requests "
                    f"({nupd} update batches log-uniform [1k, {args.uneven_max}], the rest BFS/SSSP "
                    f"queries), arrivals {'all at once' if rate <= 0 else f'Poisson {rate}/s'}",
        "served": summary("served"), "plain": summary("plain"),
        "speedup_requests_per_s": out["plain"]["wall_s"] / wall,
        "mean_wave": float(np.mean(waves)) if waves else None, "update_digests_equal": upd_ok,
        "latency": "arrival to result visible on the host, ms",
    }


def run_served(args):
    import torch

    _, _, local = dist_env()
    torch.cuda.set_device(local)
    r = served_stream(args, local, args.requests, args.rate)
    line = {
        "metric": "served request stream: requests/s and p50/p99 latency, served vs plain sequential",
        "unit": "requests/s", "value": r["served"]["requests_per_s"], "n_gpus": 1, "higher_is_better": True,
        "dtype": "u32", "data": "synthetic", "config": {"workload": r["workload"]},
    }
    line.update({k: v for k, v in r.items() if k != "workload"})
    print(json.dumps(line), flush=True)


def run_pr(args):
    """Incremental PageRank (damping 0.85, per-vertex residual threshold
    1e-9, so the FP64 L1 residual stays below 1e-9 x |V|): FP64 ranks and
    FP32 ranks with Kahan-compensated sums on the same stream, each on a
    freshly loaded engine; reports both batch rates and the FP32 ranks'
    max-relative error against the FP64 ranks after every batch."""
    import torch

    from coincgraph_b200 import Engine, gen
    from coincgraph_b200.engine import FLAG_PR_FP64

    _, _, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nb = args.warmup + args.steps
    g, h = gen.rmat(args.scale, args.edge_factor, keep_handle=True)
    ups = gen.updates(h, [args.batch] * nb, [args.batch] * nb, seed=gen.UPDATE_SEED_BASE + 4)
    batches = [[torch.from_numpy(x.astype(np.int32)).to(dev) for x in ups.batch(i)] for i in range(nb)]
    res = {}
    for form, flags in (("fp64", FLAG_PR_FP64), ("fp32_kahan", 0)):
        eng = Engine("pr", device=local, cache_gib=args.cache, pr_epsilon=1e-9, pr_max_rounds=100000, flags=flags,
                     max_batch=args.batch)
        eng.load_csr(g.n, g.xadj, g.adj)
        t0 = time.perf_counter()
        eng.init()
        torch.cuda.synchronize()
        init_s = time.perf_counter() - t0
        init_rank = eng.pagerank(fp64=flags != 0)[0].astype(np.float64)
        ms, l1, ranks = [], [], []
        for i, b in enumerate(batches):
            s = eng.apply_batch_device(*b)
            if i >= args.warmup:
                ms.append(s.ms_delete + s.ms_insert + s.ms_cache)
                l1.append(s.pr_residual_l1)
                ranks.append(eng.pagerank(fp64=flags != 0)[0].astype(np.float64))
        res[form] = {"ms": ms, "l1": l1, "ranks": ranks, "init_s": init_s, "init_rank": init_rank}
        eng.close()
    err = [float(np.max(np.abs(a - b) / np.abs(b))) for a, b in zip(res["fp32_kahan"]["ranks"], res["fp64"]["ranks"])]
    r32, r64 = res["fp32_kahan"]["init_rank"], res["fp64"]["init_rank"]
    init_err = float(np.max(np.abs(r32 - r64) / np.abs(r64)))
    line = {
        "metric": "incremental PageRank batches/s, FP32+Kahan vs FP64 (max-rel error vs FP64)", "unit": "batches/s",
        "value": args.steps / (sum(res["fp32_kahan"]["ms"]) * 1e-3),
        "fp64_value": args.steps / (sum(res["fp64"]["ms"]) * 1e-3), "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "dtype": "f32+kahan / f64", "data": "synthetic",
        "config": {"workload": f"PR RMAT s{args.scale} ef{args.edge_factor}, cache {args.cache} GiB, {args.batch} del "
                               f"+ {args.batch} ins per batch, damping 0.85, per-vertex epsilon 1e-9",
                   "vertices": g.n, "edges": g.m},
        "max_rel_err_fp32_vs_fp64": max(err + [init_err]), "init_max_rel_err": init_err, "per_batch_max_rel_err": err,
        "fp64_l1_residual_max": max(res["fp32_kahan"]["l1"]), "l1_bound": 1e-9 * g.n,
        "p50_ms": {k: statistics.median(v["ms"]) for k, v in res.items()},
        "p99_ms": {k: float(np.percentile(v["ms"], 99)) for k, v in res.items()},
        "init_s": {k: v["init_s"] for k, v in res.items()},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.workload == "pr":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the PR workload has no reference CPU arm here"}))
            return
        run_pr(args)
        return
    if args.workload == "served":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the served workload has no reference CPU arm"}))
            return
        run_served(args)
        return
    if args.workload == "uneven":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the uneven workload has no reference CPU arm"}))
            return
        run_uneven(args)
        return
    if args.workload not in ("stream", "road"):
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
