"""Writes tests/golden/root_samples.json: seeded root samples of the configured
queries whose whole root lists no exact enumerator can finish, with the
oracle's exact per-root counts.

    python tests/golden/make_root_samples.py [--threads N] [--only NAME]

A sample walks a seeded permutation of the query's root list (reference
order, the positions the library's root ids use) and keeps each root whose
Knuth estimate of set operations is at most `budget`, until the kept roots'
estimates sum to `budget`: a fixed-size unit of work per bench step, drawn at
random from all roots but the ones heavier than a whole step.  Every kept
root is then counted exactly by the oracle (each root's DFS divided over
threads at level 1, the same DFS per piece), giving the raw count, the final
count (x |Aut| when unlabeled) and the set operations, which the GPU's
per-root counts and launch statistics must equal.

The graph is built by the oracle's generator (the workload definition the
product's generator implements; a CPU test pins the two equal) -- or, for a
graph too large to sort on a host, by the product's device generator, which a
GPU test pins to the host generator -- and its arrays' sha256 is stored so a
run on another machine can check it has the same graph.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import pm_oracle as orc  # noqa: E402
from pumatch_b200 import patterns as P  # noqa: E402

# the configured C1 query: Chung-Lu 100K vertices / 1M edges (gamma 2.1,
# i0 10, expected degrees capped at 5,000, seed 1), unlabeled 7-cycle
SAMPLES = {
    "chunglu100k_c7": dict(graph=dict(kind="chung_lu", n=100_000, m=1_000_000, gamma=2.1, i0=10.0, max_w=5000.0,
                                      seed=1),
                           labeled=False, pattern=P.to_g(*P.cycle(7)), perm_seed=7, budget=5e9,
                           budget_kind="set_ops", est_probes=400, est_seed=11, max_looked=20000,
                           query_probes=20000),
    # the configured R-MAT query: 65M vertices, 1.8e9 undirected edges (a, b, c
    # = .57, .19, .19, seed 2), 8 uniform labels (seed 102), the 5-cycle plus a
    # 2-vertex pendant path with labels drawn from the 8 (seed 202).  Its
    # graph is built on a GPU (the device generator returns the host
    # generator's arrays) in a machine with ~100 GB of free RAM.  The oracle
    # scans whole hub lists (1.5M entries), so its budget is in algorithmic
    # bytes and covers the cheap roots only; `extra` roots of the same
    # permutation, budgeted in set operations, are timed on the GPU without
    # an oracle count (per-root parity on a subsample).
    "rmat65m_c5t2_lab8": dict(graph=dict(kind="rmat", n=65_000_000, m=1_800_000_000, a=0.57, b=0.19, c=0.19,
                                         seed=2, device=0),
                              labeled=True, n_labels=8, label_seed=102,
                              pattern=P.to_g(*P.cycle_tail(5, 2), P.seeded_labels(7, 8, 202)), perm_seed=7,
                              budget=4e11, budget_kind="alg_bytes", est_probes=20, est_seed=11, max_looked=300,
                              max_kept=6, query_probes=300, extra_budget=5e9, extra_cap=3e9, max_extra=6,
                              verify_s=40.0),
}


def build_graph(gd):
    if gd["kind"] == "chung_lu":
        return orc.gen_chung_lu(gd["n"], gd["m"], gd["gamma"], gd["i0"], gd["max_w"], gd["seed"])
    if "device" in gd:  # too large for a host sort: the product's device generator (same arrays)
        import pumatch_b200 as pm
        hg = pm.gen_rmat(gd["n"], gd["m"], a=gd["a"], b=gd["b"], c=gd["c"], seed=gd["seed"], device=gd["device"])
        return hg.rowptr, hg.colidx
    return orc.gen_rmat(gd["n"], gd["m"], gd["a"], gd["b"], gd["c"], gd["seed"])


def graph_digest(rowptr: np.ndarray, colidx: np.ndarray) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rowptr, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(colidx, dtype=np.int32).tobytes())
    return h.hexdigest()


def choose(g, p, roots, spec):
    """Walks the seeded permutation: roots within the oracle budget are kept
    (verified); with an extra budget, roots within it in set operations are
    kept as extra (timed, not counted by the oracle)."""
    perm = np.random.default_rng(spec["perm_seed"]).permutation(len(roots))
    kept, extra, total, xtotal, looked = [], [], 0.0, 0.0, 0
    by_bytes = spec.get("budget_kind") == "alg_bytes"
    xb = spec.get("extra_budget", 0.0)
    t0 = time.time()
    for i in perm:
        looked += 1
        if looked > spec["max_looked"]:
            break
        if looked % 25 == 0:
            print(f"  examined {looked} roots, kept {len(kept)}, extra {len(extra)}, {time.time() - t0:.0f} s",
                  flush=True)
        so, by, _ = orc.estimate(g, p, roots[i:i + 1], probes=spec["est_probes"], seed=spec["est_seed"])
        cost = by if by_bytes else so
        max_kept, max_extra = spec.get("max_kept", 1 << 30), spec.get("max_extra", 1 << 30)
        if total < spec["budget"] and cost <= spec["budget"] and len(kept) < max_kept:
            kept.append((int(i), so))
            total += cost
        elif xtotal < xb and so <= spec["extra_cap"] and len(extra) < max_extra:
            extra.append((int(i), so, by))
            xtotal += so
        kept_done = total >= spec["budget"] or len(kept) >= max_kept
        extra_done = xtotal >= xb or len(extra) >= max_extra
        if kept_done and extra_done:
            break
    return kept, extra, looked


def make(name, threads):
    spec = SAMPLES[name]
    t0 = time.time()
    rp, ci = build_graph(spec["graph"])
    labels = orc.gen_labels(len(rp) - 1, spec["n_labels"], spec["label_seed"]) if spec["labeled"] else None
    g = orc.Graph(rp, ci, labels)
    p = orc.plan(spec["pattern"], spec["labeled"])
    print(f"{name}: graph {time.time() - t0:.0f} s", flush=True)
    roots = orc.roots(g, p)
    print(f"{name}: {len(roots)} roots, {time.time() - t0:.0f} s", flush=True)
    kept, extra, looked = choose(g, p, roots, spec)
    print(f"{name}: {len(kept)} kept, {len(extra)} extra of {looked} examined, {time.time() - t0:.0f} s", flush=True)
    t1 = time.time()
    if spec.get("verify_s"):
        # exact counts within a time limit per root (a run whose pieces all
        # finish is exact); a root the oracle cannot finish in time is timed
        # on the GPU without a count
        ok, counts = [], []
        st = {"set_ops": 0, "alg_bytes": 0}
        for i, so in kept:
            c, _, done, pieces, s1 = orc.count_split(g, p, roots[i:i + 1], threads=threads,
                                                     time_limit_s=spec["verify_s"])
            if done == pieces:
                ok.append((i, so))
                counts.append(c)
                st["set_ops"] += s1["set_ops"]
                st["alg_bytes"] += s1["alg_bytes"]
            else:
                extra.append((i, so, float("nan")))
            print(f"  root {i}: {'counted' if done == pieces else 'too slow for the oracle'}, "
                  f"{time.time() - t0:.0f} s", flush=True)
        kept = ok
        per_root = np.array(counts, dtype=np.uint64)
        total = int(per_root.sum())
    else:
        idx = np.array([i for i, _ in kept], dtype=np.int64)
        total, per_root, done, pieces, st = orc.count_split(g, p, roots[idx], threads=threads)
        assert done == pieces
    mult = 1 if spec["labeled"] else p.multiplicity
    so_total, _, _ = orc.estimate(g, p, roots, probes=spec["query_probes"], seed=spec["est_seed"])
    rec = {
        "graph": spec["graph"], "graph_sha256": graph_digest(rp, ci), "n_adj": int(len(ci)),
        "labeled": spec["labeled"], "pattern": spec["pattern"], "multiplicity": int(mult),
        "rule": (f"seeded permutation (numpy default_rng({spec['perm_seed']})) of the {len(roots)} root edges; "
                 f"keep roots whose Knuth estimate ({spec['est_probes']} probes, seed {spec['est_seed']}) is at "
                 f"most {spec['budget']:.0e} {spec.get('budget_kind', 'set_ops').replace('_', ' ')} until the "
                 f"kept estimates sum to {spec['budget']:.0e}"),
        "n_labels": spec.get("n_labels", 0), "label_seed": spec.get("label_seed"),
        "n_roots_total": int(len(roots)), "roots_examined": looked,
        "max_kept": spec.get("max_kept"), "max_extra": spec.get("max_extra"),
        "query_set_ops_estimate": so_total,
        "roots": [{"index": int(i), "v0": int(roots[i][0]), "v1": int(roots[i][1]), "raw_count": int(c),
                   "count": int(c) * mult, "set_ops_estimate": so}
                  for (i, so), c in zip(kept, per_root)],
        "extra_roots": [{"index": int(i), "v0": int(roots[i][0]), "v1": int(roots[i][1]), "set_ops_estimate": so,
                         "alg_bytes_estimate": None if by != by else by} for i, so, by in extra],
        "extra_rule": (f"the same permutation's roots whose estimate is at most {spec['extra_cap']:.0e} set "
                       f"operations, until they sum to {spec['extra_budget']:.0e}, and candidates the oracle could "
                       f"not count within {spec.get('verify_s')} s; timed on the GPU, not counted by the oracle")
                      if extra else None,
        "raw_count": int(total), "count": int(total) * mult, "set_ops": int(st["set_ops"]),
        "alg_bytes": int(st["alg_bytes"]), "oracle_s": round(time.time() - t1, 1), "oracle_threads": threads,
    }
    return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", default=None)
    ap.add_argument("--out", default=os.path.join(HERE, "root_samples.json"))
    args = ap.parse_args()
    out = {}
    if os.path.exists(args.out):
        with open(args.out) as f:
            out = json.load(f)
    for name in SAMPLES:
        if args.only and name != args.only:
            continue
        out[name] = make(name, args.threads)
        print(name, len(out[name]["roots"]), "roots", out[name]["count"], out[name]["set_ops"],
              out[name]["oracle_s"], "s", flush=True)
        with open(args.out, "w") as f:
            json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
