#!/usr/bin/env python
"""bench.py -- subgraph-matching throughput on B200 (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one query over the workload's root edges: the GPU root filter plus
the persistent DFS launch, counts read back.  The default workload is the
configured small query -- the 7-cycle, unlabeled, on the Chung-Lu graph of
100K vertices and 1M edges -- whose full root list is out of reach of any
exact enumerator (about 1.4e16 set operations), so a step runs a seeded
sample of its root edges (tests/golden/root_samples.json states the rule);
every sampled root's count is checked against the oracle's exact per-root
count in that fixture, and the run fails on any difference.  Workloads
without a sample run every root edge and are checked per root on the roots
the CPU baseline samples.

`value` is matches/s with the graph already resident in HBM (device time,
CUDA events on the library's own stream, max over ranks); `e2e` is the same
metric through the public API with host buffers (graph upload + match +
count read-back inside the timed region).  With N>1 ranks the root chunks are
sharded across ranks (rank r takes chunks r, r+N, ...) and the counts are
summed with one 8-byte all-reduce per pattern.

The default line (one GPU) also carries the two comparisons the metric
names, measured after the timed steps: `batched_vs_sequential` (twenty
patterns in one persistent launch vs one launch each) and `learned_vs_plain`
(learned residency, order, prefetch and split thresholds vs a cold CLOCK pool
on a paged graph, with the model's prediction error beside a constant
predictor's), both on R-MAT graphs of 2^17 vertices with identical counts
across arms.  Two more follow on the same graphs: `paging_ablation`, the
reference's residency ablations (device partition plus package buffer,
partition only, buffer only, UM only) as pool splits of the paged path,
beside the graph in HBM; and `page_size_tuning`, the autotuner's page-size
axis (16, 64, 256 KB) on the twenty-pattern batch, paged.
--no-comparisons leaves all four out.

--impl reference times the CPU implementation of the same path (the oracle
port; the reference itself has no CPU implementation of its matcher) on all
host cores, one bounded sample of the same roots per step, rank 0 only; it
builds its inputs with the oracle's generators and never loads the product
library.
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

# name -> definition.  Each keeps the graph family, sizes and seeds of the
# configuration it stands in for.  A workload with a "sample" runs the seeded
# root sample of that name in tests/golden/root_samples.json.
_CL100K = dict(kind="chung_lu", n=100_000, m=1_000_000, gamma=2.1, i0=10.0, max_w=5000.0, seed=1)
_RMAT1M = dict(kind="rmat", n=1 << 20, m=16 << 20, a=0.57, b=0.19, c=0.19, seed=2)
_RMAT128K = dict(kind="rmat", n=1 << 17, m=16 << 17, a=0.57, b=0.19, c=0.19, seed=2)
# the configured R-MAT graph: 65M vertices, 1.8e9 undirected edges (3.6e9
# adjacency entries, 14.4 GB), generated on the GPU (same arrays as the host
# generator)
_RMAT65M = dict(kind="rmat", n=65_000_000, m=1_800_000_000, a=0.57, b=0.19, c=0.19, seed=2, device=0)
WORKLOADS = {
    # the configured small query: Chung-Lu 100K vertices / 1M edges, gamma
    # 2.1, expected degrees capped at 5,000, unlabeled, in HBM; the 7-cycle,
    # on a seeded sample of its root edges
    "chunglu100k_c7": dict(graph=_CL100K, labeled=False, n_labels=0, patterns=[("C7", P.cycle(7))],
                           sample="chunglu100k_c7"),
    # the same query over its whole root list: only for --root-begin/--root-limit
    # slices (profiling); the whole list is out of reach
    "chunglu100k_c7_all": dict(graph=_CL100K, labeled=False, n_labels=0, patterns=[("C7", P.cycle(7))]),
    # the same graph, every root edge of the 7-clique
    "chunglu100k_k7": dict(graph=_CL100K, labeled=False, n_labels=0, patterns=[("K7", P.clique(7))]),
    # the same graph with 16 uniform labels and the 7-cycle (labeled semantics)
    "chunglu100k_c7_lab16": dict(graph=_CL100K, labeled=True, n_labels=16, label_seed=102, pattern_label_seed=202,
                                 patterns=[("C7", P.cycle(7))]),
    # the K7 query with the adjacency in host memory: 60% of it in static
    # frames (the reference's device partition: the first 60% of the edges)
    # plus evictable frames for 28% (its 4 GB package buffer against the
    # 14.4 GB adjacency of the configured R-MAT graph)
    "chunglu100k_k7_paged": dict(graph=_CL100K, labeled=False, n_labels=0, patterns=[("K7", P.clique(7))],
                                 paged=dict(frame_fraction=0.88, static_fraction=0.6, page_bytes=16 << 10)),
    # R-MAT (a,b,c = .57,.19,.19) 1M vertices / 16M edges, 32 labels, the
    # 5-cycle plus 2-vertex pendant path, in HBM and paged (the same pool split)
    "rmat1m_c5t2_lab32": dict(graph=_RMAT1M, labeled=True, n_labels=32, label_seed=102, pattern_label_seed=202,
                              patterns=[("C5t2", P.cycle_tail(5, 2))]),
    "rmat1m_c5t2_lab32_paged": dict(graph=_RMAT1M, labeled=True, n_labels=32, label_seed=102,
                                    pattern_label_seed=202, patterns=[("C5t2", P.cycle_tail(5, 2))],
                                    paged=dict(frame_fraction=0.88, static_fraction=0.6, page_bytes=64 << 10)),
    # the configured R-MAT query: 8 uniform labels, the 5-cycle plus a 2-vertex
    # pendant path (labels from the 8), on a seeded root sample; paged through
    # a 4 GB frame pool of 64 KB pages (the whole adjacency stays in pinned
    # host memory), half of it static (the array's first 2 GB: the hubs'
    # lists, measured 1.3x faster than an all-evictable pool), and in HBM for
    # the set-operation roofline
    "rmat65m_c5t2_lab8_paged": dict(graph=_RMAT65M, labeled=True, n_labels=8, label_seed=102, pattern_label_seed=202,
                                    patterns=[("C5t2", P.cycle_tail(5, 2))], sample="rmat65m_c5t2_lab8",
                                    paged=dict(frame_bytes=4 << 30, static_bytes=2 << 30, page_bytes=64 << 10)),
    "rmat65m_c5t2_lab8": dict(graph=_RMAT65M, labeled=True, n_labels=8, label_seed=102, pattern_label_seed=202,
                              patterns=[("C5t2", P.cycle_tail(5, 2))], sample="rmat65m_c5t2_lab8"),
    # the configured batch: twenty seeded 4-7-vertex patterns (8 labels) on the
    # configured R-MAT graph, paged through the 4 GB pool, over a slice of
    # each pattern's root list (--root-frac, --root-limit)
    "rmat65m_batch20_lab8_paged": dict(graph=_RMAT65M, labeled=True, n_labels=8, label_seed=102, batch_seed=303,
                                       paged=dict(frame_bytes=4 << 30, static_bytes=2 << 30, page_bytes=64 << 10)),
    # twenty seeded 4-7-vertex patterns in one persistent launch
    "rmat128k_batch20_lab32": dict(graph=_RMAT128K, labeled=True, n_labels=32, label_seed=102, batch_seed=303),
    # learned-scheduler comparison (--learned): trained on seeds 11, 12, 13;
    # a frame pool of half the adjacency, all of it under CLOCK
    "rmat128k_c5t2_lab32_clock": dict(graph=_RMAT128K, labeled=True, n_labels=32, label_seed=102,
                                      pattern_label_seed=202, patterns=[("C5t2", P.cycle_tail(5, 2))],
                                      paged=dict(frame_fraction=0.5, static_fraction=0.0, page_bytes=16 << 10)),
    # the same graph with the reference's split: 60% of the adjacency in
    # static frames plus 28% evictable
    "rmat128k_c5t2_lab32_paged": dict(graph=_RMAT128K, labeled=True, n_labels=32, label_seed=102,
                                      pattern_label_seed=202, patterns=[("C5t2", P.cycle_tail(5, 2))],
                                      paged=dict(frame_fraction=0.88, static_fraction=0.6, page_bytes=16 << 10)),
}
DEFAULT_WORKLOAD = "chunglu100k_c7"
SAMPLES_PATH = os.path.join(ROOT, "tests", "golden", "root_samples.json")


def _oracle():
    """The CPU oracle (test infrastructure): the checker and the CPU arm."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pm_oracle as orc
    return orc


def make_graph(g, seed=None, via_oracle=False):
    """Host CSR of a workload graph: the product's generator, or (for the CPU
    arm, which must not load the product library) the oracle's restatement of
    it, which a CPU test pins to the same arrays."""
    seed = g["seed"] if seed is None else seed
    if via_oracle:
        orc = _oracle()
        if g["kind"] == "chung_lu":
            rp, ci = orc.gen_chung_lu(g["n"], g["m"], g["gamma"], g["i0"], g["max_w"], seed)
        else:
            rp, ci = orc.gen_rmat(g["n"], g["m"], g["a"], g["b"], g["c"], seed)
        return pm.HostGraph(rp, ci)
    if g["kind"] == "chung_lu":
        return pm.gen_chung_lu(g["n"], g["m"], gamma=g["gamma"], i0=g["i0"], max_w=g["max_w"], seed=seed)
    return pm.gen_rmat(g["n"], g["m"], a=g["a"], b=g["b"], c=g["c"], seed=seed, device=g.get("device"))


def build_workload(name, graph_seed=None, via_oracle=False):
    w = WORKLOADS[name]
    hg = make_graph(w["graph"], graph_seed, via_oracle)
    if w["labeled"]:
        ls = w["label_seed"] if graph_seed is None else w["label_seed"] + 1000 * graph_seed
        labels = _oracle().gen_labels(hg.n, w["n_labels"], ls) if via_oracle else pm.gen_labels(hg.n, w["n_labels"], ls)
        hg = pm.HostGraph(hg.rowptr, hg.colidx, labels)
    if "batch_seed" in w:
        texts = P.batch_of_20(seed=w["batch_seed"], n_labels=w["n_labels"])
    else:
        texts = []
        for i, (pname, (k, edges)) in enumerate(w["patterns"]):
            labs = P.seeded_labels(k, w["n_labels"], w["pattern_label_seed"] + i) if w["labeled"] else None
            texts.append((pname, P.to_g(k, edges, labs)))
    return w, hg, texts


def load_sample(w, hg, path=None):
    """The workload's root sample record, after checking that this graph is
    the one the sample was drawn on (arrays' sha256)."""
    if "sample" not in w:
        return None
    import hashlib
    with open(path or SAMPLES_PATH) as f:
        rec = json.load(f)[w["sample"]]
    h = hashlib.sha256()
    h.update(hg.rowptr.tobytes())
    h.update(hg.colidx.tobytes())
    if h.hexdigest() != rec["graph_sha256"]:
        raise SystemExit(f"the generated graph differs from the one {w['sample']} was drawn on")
    return rec


def sample_config(rec):
    if rec is None:
        return None
    k = len(rec["roots"])
    extra = rec.get("extra_roots") or []
    out = {"rule": rec["rule"], "roots": k + len(extra), "of": rec["n_roots_total"],
           "root_ids": [r["index"] for r in rec["roots"]] + [r["index"] for r in extra],
           "oracle_verified_roots": k, "verified_set_ops": rec["set_ops"],
           "query_set_ops_estimate": rec["query_set_ops_estimate"]}
    if extra:
        out["extra_rule"] = rec.get("extra_rule")
        out["extra_set_ops_estimate"] = sum(r["set_ops_estimate"] for r in extra)
    else:
        out["share_of_query"] = rec["set_ops"] / rec["query_set_ops_estimate"]
    return out


def place_graph(w, hg, device):
    pg = w.get("paged")
    if not pg:
        return pm.GraphPreprocessor.from_host(hg, labeled=w["labeled"], device=device)
    pb = pg["page_bytes"]
    if "frame_bytes" in pg:  # an absolute pool (the configured 4 GB)
        pool, static = pg["frame_bytes"] // pb * pb, pg.get("static_bytes", 0) // pb * pb
    else:  # a share of the adjacency array
        pool = max(pb, int(hg.colidx.nbytes * pg["frame_fraction"]) // pb * pb)
        static = int(hg.colidx.nbytes * pg.get("static_fraction", 0.0)) // pb * pb
    if pg.get("partitioned"):
        # the array cut into slices held in the HBM of this node's GPUs (all
        # on `device` when it is the only one), mapped into one device range
        import torch

        from pumatch_b200 import parts
        k, ndev = pg["partitioned"], max(1, torch.cuda.device_count())
        return parts.place_local(hg, k, device=device, owners=[(device + i) % ndev for i in range(k)],
                                 labeled=w["labeled"], frame_pool_bytes=pool, page_bytes=pb, static_pool_bytes=static)
    return pm.GraphPreprocessor.from_host(hg, labeled=w["labeled"], device=device, paged=True,
                                          page_bytes=pb, frame_pool_bytes=pool, static_pool_bytes=static)


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


def cpu_measure(hg, texts, labeled, threads, sample=None, time_limit_s=15.0, seed=5, per_root=False):
    """Times the oracle on the host cores.

    With a root sample: the sampled roots' DFS pieces (level-1 candidates) in
    a seeded shuffled order, stopped at time_limit_s (inside a piece too);
    the rate is the matches found per second.  Without one: seeded random root samples,
    grown until a run takes about a quarter of time_limit_s; with per_root the
    per-root counts of the last sample are returned for the parity check.
    Returns dict(matches, seconds, sample text[, roots, per_root])."""
    orc = _oracle()
    g = orc.Graph(hg.rowptr, hg.colidx, hg.labels if labeled else None)
    plans = [orc.plan(t, labeled) for _, t in texts]
    mult = [1 if labeled else p.multiplicity for p in plans]
    if sample is not None:
        p = plans[0]
        ids = [r["index"] for r in sample["roots"]] + [r["index"] for r in (sample.get("extra_roots") or [])]
        rts = orc.roots(g, p)[ids]
        t0 = time.perf_counter()
        c, _, done, tot, _ = orc.count_split(g, p, rts, threads=threads, time_limit_s=time_limit_s,
                                             shuffle_seed=seed)
        dt = time.perf_counter() - t0
        return {"matches": c * mult[0], "seconds": dt,
                "sample": f"the {len(rts)} sampled root edges' DFS split into {tot} level-1 pieces, taken in a "
                          f"seeded shuffled order for {dt:.1f} s on {threads} threads ({done} pieces finished)"}
    rng = np.random.default_rng(seed)
    roots = [orc.roots(g, p) for p in plans]
    total_roots = sum(len(r) for r in roots)
    frac = 1e-4
    while True:
        samples = []
        for r in roots:
            k = max(1, int(len(r) * frac))
            idx = np.sort(rng.choice(len(r), size=min(k, len(r)), replace=False))
            samples.append(idx)
        t0 = time.perf_counter()
        m, per = 0, []
        for p, r, idx, mu in zip(plans, roots, samples, mult):
            c, pr, _, _, _ = orc.count_split(g, p, r[idx], threads=threads)
            m += c * mu
            per.append(pr)
        dt = time.perf_counter() - t0
        n_s = sum(len(s) for s in samples)
        if dt >= time_limit_s / 4 or frac >= 1.0:
            out = {"matches": m, "seconds": dt,
                   "sample": f"{n_s} of {total_roots} root edges, seeded random sample, {dt:.1f} s of oracle DFS"}
            if per_root:
                out["roots"] = samples
                out["per_root"] = per
            return out
        frac = min(1.0, frac * max(2.0, min(50.0, (time_limit_s / 2) / max(dt, 1e-3))))


def run_reference(args, workload):
    """CPU arm: the oracle port of the path, all host threads, a bounded
    sample of the same workload per step.  Inputs come from the oracle's own
    generators; the product library is never loaded."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    w, hg, texts = build_workload(workload, via_oracle=True)
    sample = load_sample(w, hg, args.samples)
    threads = os.cpu_count() or 1
    for k in range(args.warmup):
        cpu_measure(hg, texts, w["labeled"], threads, sample, time_limit_s=2.0, seed=99 + k)
    tot_m, tot_s, descr = 0, 0.0, ""
    for k in range(args.steps):
        r = cpu_measure(hg, texts, w["labeled"], threads, sample, time_limit_s=10.0, seed=k + 1)
        tot_m += r["matches"]
        tot_s += r["seconds"]
        descr = r["sample"]
    value = tot_m / tot_s if tot_s > 0 else 0.0
    sample_txt = f"{args.steps} steps, each {descr}"
    line = {
        "impl": "reference", "metric": "matches_per_s", "value": value, "unit": "matches/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_s / max(args.steps, 1),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": workload, "graph": w["graph"], "labeled": w["labeled"],
                   "patterns": [p for p, _ in texts], "root_sample": sample_config(sample)},
        "cpu_baseline": {"value": value, "unit": "matches/s", "cores": threads, "kind": "port",
                         "sample": sample_txt},
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
    if args.static_frac is not None and w.get("paged") and "frame_bytes" in w["paged"]:
        # part of the absolute pool placed once and never evicted (the array's first pages)
        w = dict(w, paged=dict(w["paged"], static_bytes=int(args.static_frac * w["paged"]["frame_bytes"])))
    if args.partitioned and w.get("paged"):
        w = dict(w, paged=dict(w["paged"], partitioned=args.partitioned))
    sample = load_sample(w, hg, args.samples)
    subset = bool(sample and sample.get("extra_roots"))
    if sample is not None and args.sample_roots:
        # profiling a part of the sample: its roots' counts are still checked
        # positions past the verified roots select extra (timed, unverified) roots
        keep = [int(x) for x in args.sample_roots.split(",")]
        nv = len(sample["roots"])
        extra = sample.get("extra_roots") or []
        sample = dict(sample, roots=[sample["roots"][i] for i in keep if i < nv],
                      extra_roots=[extra[i - nv] for i in keep if i >= nv])
        sample["raw_count"] = sum(r["raw_count"] for r in sample["roots"])
        sample["count"] = sum(r["count"] for r in sample["roots"])
        subset = True
    labeled = w["labeled"]
    plans = [pm.PatternPreprocessor(text=t, labeled=labeled) for _, t in texts]
    ctx = pm.Context(local)
    graph = place_graph(w, hg, local)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    shard = dict(shard_rank=rank, shard_count=world) if world > 1 else {}
    run_kw = dict(timeout_ms=args.timeout_s * 1000, high_occupancy=args.high_occupancy,
                  leaf_per_lane=int(args.leaf_per_lane), lane_subtree_max=args.lane_subtree_max,
                  host_page_copy=int(args.host_page_copy), **shard)
    if args.root_limit > 0:
        run_kw.update(root_begin=args.root_begin, root_end=args.root_begin + args.root_limit)
    # per-root counts of plan 0, for the parity check
    n_roots = ctx.count_roots(graph, plans[0])
    root_counts = torch.zeros(max(n_roots, 1), dtype=torch.int64, device="cuda")
    run_kw["root_counts_ptr"] = root_counts.data_ptr()
    order_h = None
    if sample is not None:
        if len(plans) != 1 or args.root_limit > 0:
            raise SystemExit("a sampled workload runs one pattern over its sample")
        roots_all = ctx.roots(graph, plans[0])
        if len(roots_all) != sample["n_roots_total"]:
            raise SystemExit("root list length differs from the sample's")
        for r in sample["roots"] + (sample.get("extra_roots") or []):
            if tuple(roots_all[r["index"]]) != (r["v0"], r["v1"]):
                raise SystemExit(f"root {r['index']} is not the sampled edge")
        del roots_all
        ids = [r["index"] for r in sample["roots"]] + [r["index"] for r in (sample.get("extra_roots") or [])]
        order_h = torch.tensor(ids, dtype=torch.int32).pin_memory()
        order = order_h.to("cuda")
        run_kw.update(root_order_ptr=order.data_ptr(), root_begin=0, root_end=len(order_h))
        if world > 1:
            # a sample of a few roots: one root per chunk, so that the
            # chunk-cyclic shards spread them over the ranks
            run_kw["chunk"] = 1

    def one_step():
        with torch.cuda.stream(stream):
            root_counts.zero_()
        return ctx.match(graph, plans, **run_kw)

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
    per_root_gpu = root_counts.cpu().numpy()
    if dist:
        t = root_counts.clone()
        dist.all_reduce(t)
        per_root_gpu = t.cpu().numpy()

    # end to end through the public API with host buffers
    e2e_ms = []
    h2d = hg.rowptr.nbytes + hg.colidx.nbytes + (hg.labels.nbytes if labeled else 0)
    d2h = 8 * len(plans)
    if order_h is not None:
        h2d += order_h.numel() * 4
    e2e_steps = 1 if hg.colidx.nbytes > (1 << 30) else max(1, min(args.steps, 3))
    for k in range(e2e_steps):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        g2 = place_graph(w, hg, local)
        kw2 = dict(run_kw)
        kw2.pop("root_counts_ptr")
        if order_h is not None:
            o2 = order_h.to("cuda", non_blocking=True)
            kw2["root_order_ptr"] = o2.data_ptr()
        c2, _ = ctx.match(g2, plans, **kw2)
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
        parity = None
        ok = True
        mult = 1 if labeled else plans[0].PatternMultiplicity
        if sample is not None:
            # every sampled root against the oracle's exact per-root count
            bad = [r["index"] for r in sample["roots"] if int(per_root_gpu[r["index"]]) != r["raw_count"]]
            verified = sum(int(per_root_gpu[r["index"]]) for r in sample["roots"]) * mult
            ok = (not bad and verified == sample["count"] and
                  (subset or (counts_total[0] == sample["count"] and set_ops // args.steps == sample["set_ops"] and
                              alg_bytes // args.steps == sample["alg_bytes"])))
            parity = {"roots_checked": len(sample["roots"]), "ok": ok, "mismatched_roots": bad,
                      "roots_not_checked": len(sample.get("extra_roots") or []),
                      "count_checked_roots": verified, "oracle_count": sample["count"],
                      "set_ops_equal": None if subset else set_ops // args.steps == sample["set_ops"],
                      "alg_bytes_equal": None if subset else alg_bytes // args.steps == sample["alg_bytes"],
                      "against": "oracle exact per-root counts, set operations and algorithmic bytes "
                                 "(tests/golden/root_samples.json)"}
        line = {
            "metric": "matches_per_s", "value": value, "unit": "matches/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic",
            "config": {"workload": workload, "graph": w["graph"], "labeled": w["labeled"],
                       "patterns": [p for p, _ in texts], "counts": counts_total,
                       "root_sample": sample_config(sample),
                       "kernel_variant": ["default", "regs64", "regs85", "uncapped"][args.high_occupancy] +
                                         ({0: "", 1: "+leaf_per_lane", 2: "+leaf_strided"}[args.leaf_per_lane]) +
                                         (f"+lane_subtree_max={args.lane_subtree_max}"
                                          if args.lane_subtree_max else ""),
                       "root_limit": args.root_limit or None,
                       "roots": int(st["n_roots"]), "set_ops_per_step": set_ops // args.steps,
                       "donated_ranges_last_step": int(st["splits"]),
                       "page_misses_last_step": int(st["page_misses"]), "pages_loaded_last_step": int(st["pages_loaded"]),
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
            "warp_idle_frac_last_step": st["idle_ns"] / max(1, st["warp_ns"]),
            "phase_cycles_last_step": {k: int(st[k]) for k in ("leaf_cycles", "level_cycles", "prefix_cycles")},
            "arenas": {"bytes": int(st["arena_bytes"]), "borrowed": int(st["borrowed_arenas"]),
                       "pool": int(st["arena_pool"])},
        }
        if achieved > peak:
            line["roofline"]["note"] = (
                "algorithmic bytes charge each set operation its whole operand lists, as the reference's "
                "merge scans them; this kernel reads one label's group of a label-grouped list and searches "
                "a long operand rather than scanning it, so frac above 1 is that difference, not bandwidth")
        if w.get("paged"):
            info = graph.info()
            link = st["h2d_page_bytes"] + st["zero_copy_bytes"]
            line["host_link"] = {
                "pages": int(info["n_pages"]), "frames": int(info["n_frames"]),
                "static_frames": int(info["n_static_frames"]), "page_bytes": w["paged"]["page_bytes"],
                "page_hits_last_step": int(st["page_hits"]), "h2d_page_bytes_last_step": int(st["h2d_page_bytes"]),
                "page_requests_last_step": int(st["page_requests"]), "page_dropped_last_step": int(st["page_dropped"]),
                "evictions_last_step": int(st["evictions"]),
                "device_page_loads_last_step": int(st["device_page_loads"]),
                "page_loads": "host service thread only" if args.host_page_copy else
                              "warps copy pages of one-page lists; the rest through the host service thread",
                "zero_copy_bytes_last_step": int(st["zero_copy_bytes"]),
                "achieved_gbs": link / (st["kernel_ms"] / 1000.0) / 1e9 if st["kernel_ms"] > 0 else 0.0,
                "nominal_gbs": 64.0, "nominal": "PCIe Gen5 x16, one direction"}
            if w["paged"].get("partitioned"):
                line["host_link"].update(
                    source=f"array partitioned into {w['paged']['partitioned']} slices of device memory",
                    nominal_gbs=900.0, nominal="NVLink 5, one direction (peer slices; local slices read from HBM)")
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            cm = cpu_measure(hg, texts, labeled, threads, sample, time_limit_s=15.0, per_root=sample is None)
            line["cpu_baseline"] = {"value": cm["matches"] / cm["seconds"], "unit": "matches/s", "cores": threads,
                                    "kind": "port", "sample": cm["sample"]}
            if sample is None and args.root_limit == 0 and world == 1:
                # per-root parity on the roots the CPU baseline sampled (plan 0)
                idx = cm["roots"][0]
                gpu = per_root_gpu[idx].astype(np.uint64)
                bad = [int(i) for i, a, b in zip(idx, gpu, cm["per_root"][0]) if a != b]
                ok = not bad
                parity = {"roots_checked": int(len(idx)), "ok": ok, "mismatched_roots": bad[:16],
                          "against": "oracle per-root counts on the CPU baseline's seeded root sample"}
        line["parity"] = parity
        if (world == 1 and workload == DEFAULT_WORKLOAD and not args.no_comparisons and not args.sample_roots
                and args.root_limit == 0):
            line.update(comparisons(args))
        print(json.dumps(line), flush=True)
        if not ok:
            sys.exit(1)
    graph.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def learned_compare(args, workload):
    """Plain vs learned on the workload's paged graph, the model trained on
    plain runs over three other seeds of the same generator.

    plain: the frame pool starts cold (only static frames) and pages in on
    demand under CLOCK, roots in reference order.  learned: the pool starts
    with the pages the model predicts hottest, roots heaviest-first, and each
    root chunk's predicted pages are posted to the copy ring a few chunks
    ahead during the run.  Counts must be identical."""
    import torch

    from pumatch_b200 import learn
    torch.cuda.set_device(0)
    ctx = pm.Context(0)
    w, hg, texts = build_workload(workload)
    if len(texts) != 1 or not w.get("paged"):
        raise SystemExit("--learned needs a single-pattern paged workload")
    labeled = w["labeled"]
    xs, ts = [], []
    t0 = time.time()
    for seed in (11, 12, 13):
        _, hgs, _ = build_workload(workload, graph_seed=seed)
        gs = pm.GraphPreprocessor.from_host(hgs, labeled=labeled)
        ps = pm.PatternPreprocessor(text=texts[0][1], labeled=labeled)
        _, _, cost, reads = learn.plain_costs(ctx, gs, ps, timeout_ms=args.timeout_s * 1000)
        xs.append(learn.root_features(ctx, gs, ps))
        ts.append(learn.targets(cost, reads))
        gs.close()
    x, t = torch.cat(xs), torch.cat(ts)
    model = learn.CostModel(0, seed=1)
    hist = model.fit(x, t, epochs=args.learn_epochs, batch=4096, lr=3e-3)
    train_s = time.time() - t0
    p = pm.PatternPreprocessor(text=texts[0][1], labeled=labeled)
    g = place_graph(w, hg, 0)
    xe = learn.root_features(ctx, g, p)
    pred = model.predict(xe)
    # the evaluation graph's own per-root costs, from a plain run, judge the prediction
    hb = pm.GraphPreprocessor.from_host(hg, labeled=labeled)
    count, st0, cost, reads = learn.plain_costs(ctx, hb, p, timeout_ms=args.timeout_s * 1000)
    hb.close()
    te = learn.targets(cost, reads)
    mae = (pred - te).abs().mean(0).tolist()
    base = (te - t.mean(0)).abs().mean(0).tolist()
    order = learn.heavy_first_order(pred)
    info = g.info()
    roots = ctx.roots(g, p)
    pred_reads = torch.expm1(pred[:, 1].clamp_min(0)).cpu().numpy()
    page_ints = w["paged"]["page_bytes"] // 4
    score = learn.page_scores(hg.rowptr, roots, pred_reads, page_ints, info["n_pages"])
    chunk = 16
    pf_off, pf_pages = learn.prefetch_lists(hg.rowptr, hg.colidx, roots, order.cpu().numpy(), pred_reads, page_ints,
                                            chunk, per_chunk=args.prefetch_pages)
    split = learn.split_thresholds(pred)
    pf_off_d = torch.from_numpy(pf_off).cuda()
    pf_pages_d = torch.from_numpy(pf_pages if len(pf_pages) else np.zeros(1, dtype=np.int32)).cuda()
    kw = dict(timeout_ms=args.timeout_s * 1000, chunk=chunk)
    arms = {
        "plain": dict(cold_cache=1),
        "learned_residency_order": dict(root_order_ptr=order.data_ptr()),
        "learned": dict(root_order_ptr=order.data_ptr(), prefetch_off_ptr=pf_off_d.data_ptr(),
                        prefetch_pages_ptr=pf_pages_d.data_ptr(), prefetch_chunks=len(pf_off) - 1,
                        root_split_ptr=split.data_ptr()),
    }
    hot = np.argsort(-score)[:info["n_frames"] - info["n_static_frames"]]
    res = {}
    print(f"learned: trained in {train_s:.1f} s on {int(x.shape[0])} roots; evaluating", file=sys.stderr, flush=True)
    for mode, extra in arms.items():
        g.set_resident_pages(hot if mode != "plain" else np.zeros(0, dtype=np.int64))
        times, stats = [], None
        for k in range(args.warmup + args.steps):
            c, stt = ctx.match(g, [p], **kw, **extra)
            assert c[0] == count, (mode, c, count)
            print(f"  {mode} run {k}: {stt['kernel_ms']:.1f} ms, {stt['page_misses']} misses", file=sys.stderr,
                  flush=True)
            if k >= args.warmup:
                times.append(stt["kernel_ms"])
                stats = stt
        res[mode] = {"kernel_ms": statistics.median(times), "page_hits": stats["page_hits"],
                     "page_misses": stats["page_misses"], "pages_loaded": stats["pages_loaded"],
                     "zero_copy_bytes": stats["zero_copy_bytes"], "h2d_page_bytes": stats["h2d_page_bytes"],
                     "prefetch_requests": stats["prefetch_requests"], "page_requests": stats["page_requests"],
                     "page_dropped": stats["page_dropped"], "evictions": stats["evictions"],
                     "device_page_loads": stats["device_page_loads"],
                     "phase_cycles": {k: int(stats[k]) for k in ("leaf_cycles", "level_cycles", "prefix_cycles")},
                     "splits": stats["splits"]}
    line = {"metric": "query_ms_learned_vs_plain", "workload": workload, "count": count,
            "arms": res, "speedup": res["plain"]["kernel_ms"] / res["learned"]["kernel_ms"],
            "plain": "cold frame pool, CLOCK, reference root order",
            "learned": "predicted-hot pages resident, heaviest-first roots, predicted pages prefetched per chunk, "
                       "finer donation for roots predicted heavy",
            "prediction_mae_log": mae, "constant_predictor_mae_log": base, "train_loss": [hist[0], hist[-1]],
            "train_s": train_s, "train_roots": int(x.shape[0]), "eval_roots": int(xe.shape[0]),
            "frames": int(info["n_frames"]), "pages": int(info["n_pages"]),
            "prefetch_pages_listed": int(len(pf_pages))}
    g.close()
    model.close()
    ctx.close()
    return line


def run_batch_compare(args, workload, emit=True):
    """One batched persistent launch (and its CUDA-graph replay) vs the same
    patterns launched one by one, over the same roots; optional autotuner
    sweep.  With --root-frac/--root-limit every pattern runs the root
    positions [f * L, f * L + limit) of its list, L the shortest list."""
    import torch
    torch.cuda.set_device(0)
    ctx = pm.Context(0)
    w, hg, texts = build_workload(workload)
    labeled = w["labeled"]
    g = place_graph(w, hg, 0)
    plans = [pm.PatternPreprocessor(text=t, labeled=labeled) for _, t in texts]
    kw = dict(timeout_ms=args.timeout_s * 1000)
    rng = None
    if args.root_limit > 0:
        shortest = min(ctx.count_roots(g, p) for p in plans)
        b = int(args.root_frac * shortest)
        rng = (b, b + args.root_limit)
        kw.update(root_begin=rng[0], root_end=rng[1])
    for _ in range(args.warmup):
        ctx.match(g, plans, **kw)
    batched = []
    for _ in range(args.steps):
        c, st = ctx.match(g, plans, **kw)
        batched.append(st["kernel_ms"] + st["roots_ms"])
    q = ctx.prepare(g, plans, **kw)
    replay = []
    for _ in range(args.steps):
        cq, sq = q.run()
        assert cq == c
        replay.append(sq["kernel_ms"])
    q.close()
    seq = []
    for _ in range(args.steps):
        tot, cs = 0.0, []
        for p in plans:
            c1, s1 = ctx.match(g, [p], **kw)
            tot += s1["kernel_ms"] + s1["roots_ms"]
            cs.append(c1[0])
        assert cs == c
        seq.append(tot)
    line = {"metric": "batched_vs_sequential_ms", "workload": workload, "patterns": [n for n, _ in texts],
            "counts": c, "root_range": rng, "batched_ms": statistics.median(batched),
            "graph_replay_kernel_ms": statistics.median(replay), "sequential_ms": statistics.median(seq),
            "speedup": statistics.median(seq) / statistics.median(batched),
            "counts_equal": "batched, graph replay and sequential"}
    if w.get("paged"):
        line["paged"] = w["paged"]
    if not emit:
        g.close()
        ctx.close()
        return line
    print(json.dumps(line), flush=True)
    if args.autotune:
        from pumatch_b200 import autotune
        limit = max(10.0, 3.0 * statistics.median(batched) / 1000.0)  # a config 3x slower is not a candidate
        extra = {k: v for k, v in kw.items() if k != "timeout_ms"}
        rows = autotune.sweep(ctx, g, plans, warps=(4, 8, 16), chunks=(16, 64, 256, 2048), splits=(16, 64),
                              timeout_ms=int(limit * 1000), extra=extra)
        done = [r for r in rows if r["kernel_ms"] is not None]
        best = min(done, key=lambda r: r["kernel_ms"]) if done else None
        tuned = {"metric": "autotune_batched_ms", "workload": workload, "best": best,
                 "default": rows[0], "configs": len(rows), "results": rows}
        print(json.dumps(tuned), flush=True)
    g.close()
    ctx.close()
    return line


def paging_ablation(args, workload="rmat128k_c5t2_lab32_paged", root_share=16, um_timeout_ms=8000):
    """The reference's residency ablations (plot/plot_fig11.sh:139-166) on one
    paged workload, as pool splits of the same paged path: the device
    partition plus the package buffer (the workload's split), the partition
    only (the whole pool static), the buffer only (the whole pool
    evictable), and UM only (a pool of one page: every list read over the
    host link); the graph in HBM beside them.  Every arm starts cold and runs
    the first 1/root_share of the root list; counts must be equal.  The UM arm
    has a shorter device deadline: past it, it is reported as timed out."""
    import torch
    torch.cuda.set_device(0)
    ctx = pm.Context(0)
    w, hg, texts = build_workload(workload)
    labeled = w["labeled"]
    p = pm.PatternPreprocessor(text=texts[0][1], labeled=labeled)
    pg = w["paged"]
    pb = pg["page_bytes"]
    pool = max(pb, int(hg.colidx.nbytes * pg["frame_fraction"]) // pb * pb)
    static = int(hg.colidx.nbytes * pg.get("static_fraction", 0.0)) // pb * pb
    arms = {"hbm": None,
            "partition_and_buffer": (pool, static),
            "partition_only": (static, static),
            "buffer_only": (pool, 0),
            "um_only": (pb, 0)}
    rows, want, rng = {}, None, None
    for name, split in arms.items():
        if split is None:
            g = pm.GraphPreprocessor.from_host(hg, labeled=labeled, device=0)
        else:
            g = pm.GraphPreprocessor.from_host(hg, labeled=labeled, device=0, paged=True, page_bytes=pb,
                                               frame_pool_bytes=split[0], static_pool_bytes=split[1])
        try:
            if rng is None:
                rng = (0, max(1, ctx.count_roots(g, p) // root_share))
            kw = dict(root_begin=rng[0], root_end=rng[1],
                      timeout_ms=um_timeout_ms if name == "um_only" else args.timeout_s * 1000)
            if split is not None:
                kw["cold_cache"] = 1
            times, st = [], None
            try:
                for k in range(1 + args.steps):
                    c, st = ctx.match(g, [p], **kw)
                    if want is None:
                        want = c[0]
                    if c[0] != want:
                        raise RuntimeError(f"{name}: count {c[0]} differs from {want}")
                    if k >= 1:
                        times.append(st["kernel_ms"])
            except pm.PmError as e:
                if e.status != pm.PM_ERR_TIMEOUT:
                    raise
                rows[name] = {"timed_out_ms": kw["timeout_ms"]}
                continue
            info = g.info()
            row = {"kernel_ms": statistics.median(times)}
            if split is not None:
                row.update(frames=int(info["n_frames"]), static_frames=int(info["n_static_frames"]),
                           pages=int(info["n_pages"]), page_hits=st["page_hits"], page_misses=st["page_misses"],
                           pages_loaded=st["pages_loaded"] + st["device_page_loads"],
                           zero_copy_bytes=st["zero_copy_bytes"], h2d_page_bytes=st["h2d_page_bytes"])
            rows[name] = row
        finally:
            g.close()
    ctx.close()
    return {"workload": workload, "root_range": list(rng), "page_bytes": pb, "count": want, "counts_equal": True,
            "arms": rows}


def page_size_tuning(args, workload="rmat128k_batch20_lab32", root_share=8):
    """The autotuner's page-size axis on the batched query, paged: the twenty
    patterns in one launch through a frame pool of half the adjacency (all
    evictable), every run cold, at pages of 16, 64 and 256 KB with the
    default launch configuration, over the first 1/root_share of the
    shortest root list.  The tuner refuses a page size that changes a count."""
    import torch

    from pumatch_b200 import autotune
    torch.cuda.set_device(0)
    ctx = pm.Context(0)
    w, hg, texts = build_workload(workload)
    labeled = w["labeled"]
    plans = [pm.PatternPreprocessor(text=t, labeled=labeled) for _, t in texts]
    g0 = pm.GraphPreprocessor.from_host(hg, labeled=labeled, device=0)
    shortest = min(ctx.count_roots(g0, p) for p in plans)
    g0.close()
    rng = dict(root_begin=0, root_end=max(1, shortest // root_share))
    pool = hg.colidx.nbytes // 2
    out = autotune.autotune(ctx, hg, plans, labeled=labeled, paged=True, frame_pool_bytes=pool,
                            page_kb=autotune.PAGE_KB, warps=(8,), chunks=(16,), splits=(64,), variants=(),
                            reps=2, extra=rng, timeout_ms=args.timeout_s * 1000)
    ctx.close()
    return {"workload": workload, "patterns": len(plans), "root_range": [rng["root_begin"], rng["root_end"]],
            "frame_pool_bytes": pool, "best_page_kb": out["best"]["page_kb"],
            "kernel_ms_by_page_kb": {str(r["page_kb"]): r["kernel_ms"] for r in out["results"]},
            "counts_equal": True}


def comparisons(args):
    """The two comparisons the metric names, for the default line: the
    20-pattern batch in one launch vs one launch per pattern, and learned vs
    plain scheduling on a paged graph (stand-ins of the configured batch and
    learned queries at 2^17 vertices; the standalone --compare-sequential and
    --learned runs print the full records).  A failure is reported in the
    line, not raised: the default line's own measurement stands."""
    import copy
    sub = copy.copy(args)
    sub.steps, sub.warmup, sub.root_limit, sub.autotune = 2, 1, 0, False
    out = {}
    try:
        b = run_batch_compare(sub, "rmat128k_batch20_lab32", emit=False)
        out["batched_vs_sequential"] = {k: b[k] for k in ("workload", "batched_ms", "graph_replay_kernel_ms",
                                                           "sequential_ms", "speedup")}
        out["batched_vs_sequential"].update(patterns=len(b["patterns"]), counts_equal=True)
    except Exception as e:  # noqa: BLE001 -- reported in the line
        out["batched_vs_sequential"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    try:
        sub.steps, sub.warmup = 3, 1
        ln = learned_compare(sub, "rmat128k_c5t2_lab32_clock")
        arms = ln["arms"]
        out["learned_vs_plain"] = {
            "workload": ln["workload"], "plain_ms": arms["plain"]["kernel_ms"],
            "learned_residency_order_ms": arms["learned_residency_order"]["kernel_ms"],
            "learned_ms": arms["learned"]["kernel_ms"],
            "speedup_residency_order": arms["plain"]["kernel_ms"] / arms["learned_residency_order"]["kernel_ms"],
            "speedup": ln["speedup"],
            "page_misses": {k: v["page_misses"] for k, v in arms.items()},
            "prediction_mae_log": ln["prediction_mae_log"],
            "constant_predictor_mae_log": ln["constant_predictor_mae_log"],
            "counts_equal": True, "plain": ln["plain"], "learned": ln["learned"]}
    except Exception as e:  # noqa: BLE001
        out["learned_vs_plain"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    try:
        sub.steps = 2
        out["paging_ablation"] = paging_ablation(sub)
    except Exception as e:  # noqa: BLE001
        out["paging_ablation"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    try:
        out["page_size_tuning"] = page_size_tuning(sub)
    except Exception as e:  # noqa: BLE001
        out["page_size_tuning"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    return out


def run_ref_gpu_table(args):
    """This build's kernel ms beside the reference GPU binary's, on every
    (graph, pattern, truncation) of tests/golden/ref_gpu_counts.json (the
    reference's own counts and kernel ms, as shipped: -G device code); the
    counts must be the reference's."""
    import torch
    torch.cuda.set_device(0)
    gold = os.path.join(ROOT, "tests", "golden")
    recs = json.load(open(os.path.join(gold, "ref_gpu_counts.json")))
    pats = json.load(open(os.path.join(gold, "patterns.json")))
    ctx = pm.Context(0)
    graphs, rows = {}, []
    for r in recs:
        key = (r["graph"], r["labeled"])
        if key not in graphs:
            hg = pm.HostGraph.read(os.path.join(gold, "graphs", r["graph"]), labeled=r["labeled"])
            graphs[key] = pm.GraphPreprocessor.from_host(hg, labeled=r["labeled"])
        p = pm.PatternPreprocessor(text=pats[r["pattern"]], labeled=r["labeled"])
        times = []
        for k in range(args.warmup + args.steps):
            c, st = ctx.match(graphs[key], [p], truncate=r["truncate"])
            if k >= args.warmup:
                times.append(st["kernel_ms"])
        rows.append({"graph": r["graph"], "pattern": r["pattern"], "labeled": r["labeled"], "truncate": r["truncate"],
                     "count": c[0], "ref_count": r["count"], "equal": c[0] == r["count"],
                     "ref_kernel_ms": r["ms"], "kernel_ms": statistics.median(times)})
    for g in graphs.values():
        g.close()
    ctx.close()
    line = {"metric": "reference_gpu_vs_ours_kernel_ms", "rows": rows,
            "all_counts_equal": all(x["equal"] for x in rows),
            "note": "reference: its own GPU binary built from its sources as shipped (-G device code), times from "
                    "tests/golden/ref_gpu_counts.json; ours: median device time of this build's launch"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--timeout-s", type=int, default=120, help="hard device-side limit per launch")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--high-occupancy", type=int, default=0,
                    help="kernel variant: 0 default, 1 capped at 64 registers, 2 capped at 85, 3 uncapped")
    ap.add_argument("--static-frac", type=float, default=None,
                    help="paged workloads with an absolute pool: this share of it static (never evicted)")
    ap.add_argument("--partitioned", type=int, default=0,
                    help="paged workloads: take pages from the array cut into this many slices of device memory "
                         "(one per GPU of the node, round robin) instead of pinned host memory")
    ap.add_argument("--host-page-copy", action="store_true",
                    help="paged: every page load through the host service thread (no warp-side copies)")
    ap.add_argument("--leaf-per-lane", type=int, default=0,
                    help="last level: 0 work-balanced in lane-contiguous parts (default), 1 one candidate per "
                         "lane, 2 work-balanced strided")
    ap.add_argument("--lane-subtree-max", type=int, default=0,
                    help="clique-like plans: last two levels one candidate per lane up to this parent size "
                         "(0 default, -1 never)")
    ap.add_argument("--root-limit", type=int, default=0, help="profile this many roots only (from --root-begin)")
    ap.add_argument("--root-begin", type=int, default=0)
    ap.add_argument("--root-frac", type=float, default=0.0,
                    help="with --compare-sequential: start the root slice at this fraction of the shortest list")
    ap.add_argument("--samples", default=None, help="root-sample fixture file (default tests/golden/root_samples.json)")
    ap.add_argument("--sample-roots", default="",
                    help="sampled workloads: run only these positions of the sample (comma-separated; profiling)")
    ap.add_argument("--learned", action="store_true", help="plain vs learned scheduling on the workload")
    ap.add_argument("--learn-epochs", type=int, default=20)
    ap.add_argument("--prefetch-pages", type=int, default=64, help="learned: pages listed per root chunk")
    ap.add_argument("--compare-sequential", action="store_true", help="batched vs one launch per pattern")
    ap.add_argument("--autotune", action="store_true", help="with --compare-sequential: sweep launch configs")
    ap.add_argument("--no-comparisons", action="store_true",
                    help="default line without the batched and learned comparisons")
    ap.add_argument("--ref-gpu-table", action="store_true",
                    help="this build's kernel ms beside the reference GPU binary's on its golden cases")
    args = ap.parse_args()
    if args.ref_gpu_table:
        run_ref_gpu_table(args)
    elif args.learned:
        print(json.dumps(learned_compare(args, args.workload)), flush=True)
    elif args.compare_sequential:
        run_batch_compare(args, args.workload)
    elif args.impl == "reference":
        run_reference(args, args.workload)
    else:
        run_ours(args, args.workload)


if __name__ == "__main__":
    main()
