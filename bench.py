#!/usr/bin/env python
"""bench.py -- subgraph-matching throughput on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one full query: the GPU root filter plus the persistent DFS launch
over every root edge of the workload's graph, counts read back.  `value` is
matches/s with the graph already resident in HBM (device time, CUDA events on
the library's own stream, max over ranks); `e2e` is the same metric through the
public API with host buffers (graph upload + match + count read-back inside the
timed region).  With N>1 ranks the query's root chunks are sharded across ranks
(rank r takes chunks r, r+N, ...) and the counts are summed with one 8-byte
all-reduce per pattern.

--impl reference times the CPU implementation of the same path (the oracle
port; the reference itself has no CPU implementation of its matcher) on the
host cores, one bounded root sample per step, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import pumatch_b200 as pm  # noqa: E402
from pumatch_b200 import patterns as P  # noqa: E402

# name -> definition.  Graph sizes/seeds follow the configuration each one
# stands in for; the reasons for each stand-in are in DESIGN.md.
WORKLOADS = {
    # Chung-Lu 100K vertices / 1M edges, gamma 2.1, expected degrees capped
    # at 5,000, unlabeled, in HBM; one 7-vertex query: the 7-clique.
    "chunglu100k_k7": dict(graph=dict(kind="chung_lu", n=100_000, m=1_000_000, gamma=2.1, i0=10.0,
                                      max_w=5000.0, seed=1),
                           labeled=False, n_labels=0, patterns=[("K7", P.clique(7))]),
    # the same graph with 16 uniform labels and the 7-cycle (labeled semantics)
    "chunglu100k_c7_lab16": dict(graph=dict(kind="chung_lu", n=100_000, m=1_000_000, gamma=2.1, i0=10.0,
                                            max_w=5000.0, seed=1),
                                 labeled=True, n_labels=16, label_seed=102, pattern_label_seed=202,
                                 patterns=[("C7", P.cycle(7))]),
}
DEFAULT_WORKLOAD = "chunglu100k_k7"


def build_workload(name):
    w = WORKLOADS[name]
    g = w["graph"]
    if g["kind"] == "chung_lu":
        hg = pm.gen_chung_lu(g["n"], g["m"], gamma=g["gamma"], i0=g["i0"], max_w=g["max_w"], seed=g["seed"])
    else:
        hg = pm.gen_rmat(g["n"], g["m"], a=g.get("a", 0.57), b=g.get("b", 0.19), c=g.get("c", 0.19), seed=g["seed"])
    if w["labeled"]:
        hg = pm.HostGraph(hg.rowptr, hg.colidx, pm.gen_labels(hg.n, w["n_labels"], seed=w["label_seed"]))
    texts = []
    for i, (pname, (k, edges)) in enumerate(w["patterns"]):
        labs = P.seeded_labels(k, w["n_labels"], w["pattern_label_seed"] + i) if w["labeled"] else None
        texts.append((pname, P.to_g(k, edges, labs)))
    return w, hg, texts


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profile_traffic(workload):
    """DRAM bytes per launch of the matching kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"match_kernel_{workload}.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch")
    except (OSError, ValueError):
        return None


def cpu_sample_run(hg, texts, labeled, threads, target_s=15.0, seed=5, max_frac=1.0):
    """Times the oracle on a seeded random root sample sized for ~target_s.
    Returns (matches, seconds, roots_in_sample, roots_total)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pm_oracle as orc
    g = orc.Graph(hg.rowptr, hg.colidx, hg.labels if labeled else None)
    rng = np.random.default_rng(seed)
    plans = [(orc.plan(t, labeled)) for _, t in texts]
    roots = [orc.roots(g, p) for p in plans]
    total_roots = sum(len(r) for r in roots)
    frac = 1e-4
    while True:
        samples = []
        for r in roots:
            k = max(1, int(len(r) * frac))
            idx = np.sort(rng.choice(len(r), size=min(k, len(r)), replace=False))
            samples.append(np.ascontiguousarray(r[idx]))
        t0 = time.perf_counter()
        m = 0
        for p, s in zip(plans, samples):
            c, _ = orc.count(g, p, s, threads=threads)
            m += c if labeled else c * p.multiplicity
        dt = time.perf_counter() - t0
        n_s = sum(len(s) for s in samples)
        if dt >= target_s / 4 or frac >= max_frac:
            return m, dt, n_s, total_roots
        frac = min(max_frac, frac * max(2.0, min(50.0, (target_s / 2) / max(dt, 1e-3))))


def run_reference(args, workload):
    """CPU arm: the oracle port of the path, all host threads, bounded samples."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    w, hg, texts = build_workload(workload)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample_run(hg, texts, w["labeled"], threads, target_s=2.0, seed=99)
    tot_m, tot_s, tot_n = 0, 0.0, 0
    total_roots = 0
    for k in range(args.steps):
        m, dt, n_s, total_roots = cpu_sample_run(hg, texts, w["labeled"], threads, target_s=10.0, seed=k + 1)
        tot_m += m
        tot_s += dt
        tot_n += n_s
    value = tot_m / tot_s if tot_s > 0 else 0.0
    sample = f"{tot_n} of {total_roots} root edges per {args.steps} steps (seeded random samples)"
    line = {
        "impl": "reference", "metric": "matches_per_s", "value": value, "unit": "matches/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_s / max(args.steps, 1),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": workload, "graph": w["graph"], "labeled": w["labeled"],
                   "patterns": [p for p, _ in texts], "sample": sample},
        "cpu_baseline": {"value": value, "unit": "matches/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "matches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, workload):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    w, hg, texts = build_workload(workload)
    labeled = w["labeled"]
    plans = [pm.PatternPreprocessor(text=t, labeled=labeled) for _, t in texts]
    ctx = pm.Context(local)
    graph = pm.GraphPreprocessor.from_host(hg, labeled=labeled, device=local)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    shard = dict(shard_rank=rank, shard_count=world) if world > 1 else {}
    run_kw = dict(timeout_ms=args.timeout_s * 1000, high_occupancy=args.high_occupancy, **shard)
    if args.root_limit > 0:
        run_kw.update(root_begin=0, root_end=args.root_limit)

    def one_step():
        counts, st = ctx.match(graph, plans, **run_kw)
        return counts, st

    def reduce_counts(counts):
        if dist is None:
            return counts
        t = torch.tensor(counts, dtype=torch.int64, device="cuda")
        dist.all_reduce(t)
        return [int(x) for x in t.cpu()]

    for _ in range(args.warmup):
        reduce_counts(one_step()[0])
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    dev_ms, kern_ms, alg_bytes, set_ops, launches = [], [], 0, 0, 0
    counts_total = None
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(k & 0xFF)  # evict the graph from L2 between steps
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            counts, st = one_step()
            e1.record(stream)
            e1.synchronize()
            dev_ms.append(e0.elapsed_time(e1))
            kern_ms.append(st["kernel_ms"])
            alg_bytes += st["alg_bytes"]
            set_ops += st["set_ops"]
            launches += 2 * len(plans) + 1
            counts = reduce_counts(counts)
            counts_total = counts
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms = sum(dev_ms)
    if dist:
        t = torch.tensor([total_ms, sum(kern_ms)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t[0])
    matches_per_step = sum(counts_total)
    value = matches_per_step * args.steps / (total_ms / 1000.0)

    # end to end through the public API with host buffers
    e2e_ms = []
    h2d = hg.rowptr.nbytes + hg.colidx.nbytes + (hg.labels.nbytes if labeled else 0)
    d2h = 8 * len(plans)
    for k in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        g2 = pm.GraphPreprocessor.from_host(hg, labeled=labeled, device=local)
        c2, _ = ctx.match(g2, plans, **run_kw)
        g2.close()
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) * 1000.0
        c2 = reduce_counts(c2)
        assert c2 == counts_total, (c2, counts_total)
        e2e_ms.append(dt)
    e2e_total = sum(e2e_ms)
    if dist:
        t = torch.tensor([e2e_total], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t[0])
    e2e_value = matches_per_step * len(e2e_ms) / (e2e_total / 1000.0)

    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        per_launch_bytes = alg_bytes / args.steps
        per_launch_s = (sum(kern_ms) / args.steps) / 1000.0
        achieved = per_launch_bytes / per_launch_s / 1e9 if per_launch_s > 0 else 0.0
        traffic = profile_traffic(workload)
        line = {
            "metric": "matches_per_s", "value": value, "unit": "matches/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic",
            "config": {"workload": workload, "graph": w["graph"], "labeled": w["labeled"],
                       "patterns": [p for p, _ in texts], "counts": counts_total,
                       "kernel_variant": "high_occupancy" if args.high_occupancy else "default",
                       "root_limit": args.root_limit or None,
                       "roots": int(st["n_roots"]), "set_ops_per_step": set_ops // args.steps,
                       "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"roots sharded x{world}" if world > 1 else "1 GPU"},
            "e2e": {"value": e2e_value, "unit": "matches/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_total / len(e2e_ms)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "match_kernel", "peak_source": peak_kind,
                         "alg_bytes_per_launch": int(per_launch_bytes)},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            m, dt, n_s, n_tot = cpu_sample_run(hg, texts, labeled, threads, target_s=15.0)
            line["cpu_baseline"] = {"value": m / dt, "unit": "matches/s", "cores": threads, "kind": "port",
                                    "sample": f"{n_s} of {n_tot} root edges, seeded random sample, "
                                              f"{dt:.1f} s of oracle DFS"}
        print(json.dumps(line), flush=True)
    graph.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--timeout-s", type=int, default=120, help="hard device-side limit per launch")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--high-occupancy", action="store_true", help="kernel variant capped at 64 registers")
    ap.add_argument("--root-limit", type=int, default=0, help="profile a prefix of the root list only")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args, args.workload)
    else:
        run_ours(args, args.workload)


if __name__ == "__main__":
    main()
