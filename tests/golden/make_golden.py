"""Generates the golden fixtures under tests/golden/ from the REFERENCE itself.

Run in a container that has the reference sources (the recipe oracle/Makefile
`make ref` compiles the reference's own, untouched host headers into
oracle/_ref/):

    PM_REF_DIR=<reference checkout> make -C oracle ref && python tests/golden/make_golden.py

Writes
  graphs/<name>.{meta.txt,vertex.bin,edge.bin,label.bin}  seeded small graphs
                                                          (the product's own
                                                          generators)
  patterns.json    {name: .g text} -- generated shapes and random patterns
  plans.jsonl      the reference PatternPreprocessor's plan per (pattern, mode)
  roots.json       the reference JobQueuePreprocessor's root list per
                   (graph, pattern, mode): count, sha256 of the pairs, first 16
The reference's GPU counts on the same inputs are produced on a GPU machine by
tests/golden/make_ref_gpu_counts.py (ref_gpu_counts.json).
"""
from __future__ import annotations

import json
import os
import random
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import pumatch_b200 as pm  # noqa: E402
from pumatch_b200 import patterns as P  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")


def golden_graphs():
    """name -> (HostGraph, labels or None).  Small enough to keep in git."""
    out = {}
    hg = pm.gen_chung_lu(400, 2000, gamma=2.1, i0=1.0, max_w=0, seed=11)
    out["cl400"] = (hg, pm.gen_labels(hg.n, 3, seed=111))
    hg = pm.gen_rmat(512, 3000, seed=12)
    out["rmat512"] = (hg, pm.gen_labels(hg.n, 4, seed=112))
    hg = pm.gen_chung_lu(60, 900, gamma=2.5, i0=5.0, max_w=0, seed=13)
    out["dense60"] = (hg, pm.gen_labels(hg.n, 2, seed=113))
    hg = pm.gen_chung_lu(3000, 6000, gamma=2.1, i0=1.0, max_w=0, seed=14)
    out["cl3000"] = (hg, pm.gen_labels(hg.n, 2, seed=114))
    return out


def golden_patterns():
    pats = {}
    for k in range(3, 8):
        for shape in ("clique", "cycle", "star", "path"):
            n, e = P.SHAPES[shape](k)
            pats[f"{shape}{k}"] = P.to_g(n, e)
    pats["house"] = P.to_g(*P.house())
    pats["house_tail1"] = P.to_g(*P.house_tail(1))
    pats["house_tail2"] = P.to_g(*P.house_tail(2))
    pats["cycle5_tail2"] = P.to_g(*P.cycle_tail(5, 2))
    r = random.Random(2026)
    for t in range(40):
        k = r.randint(3, 7)
        edges = [(0, 1)] + [(r.randrange(i), i) for i in range(2, k)]
        edges += [(i, j) for i in range(k) for j in range(i + 1, k) if (i, j) not in edges and r.random() < 0.3]
        pats[f"rand{t:02d}"] = P.to_g(k, edges, [r.randrange(3) for _ in range(k)])
    # labeled variants of the shapes (labels over 3 values)
    for name in ("cycle5", "clique4", "path5", "star5", "house", "cycle5_tail2"):
        n = int(pats[name].count("\nv ") + 1)
        labs = [r.randrange(3) for _ in range(n)]
        lines = pats[name].splitlines()
        vl = [f"v {i} {labs[i]}" for i in range(n)]
        pats[name + "_lab"] = "\n".join(vl + lines[n:]) + "\n"
    return pats


def pairs_digest(pairs) -> str:
    """sha256 over the int32 little-endian (r, c) pairs, in list order."""
    import hashlib
    import struct
    h = hashlib.sha256()
    for r, c in pairs:
        h.update(struct.pack("<ii", r, c))
    return h.hexdigest()


def main():
    graphs = golden_graphs()
    gdir = os.path.join(HERE, "graphs")
    os.makedirs(gdir, exist_ok=True)
    for name, (hg, labels) in graphs.items():
        pm.HostGraph(hg.rowptr, hg.colidx, labels).write(os.path.join(gdir, name))
    pats = golden_patterns()
    with open(os.path.join(HERE, "patterns.json"), "w") as f:
        json.dump(pats, f, indent=0, sort_keys=True)
    tmp = tempfile.mkdtemp()
    plans = []
    for name, text in sorted(pats.items()):
        path = os.path.join(tmp, name + ".g")
        open(path, "w").write(text)
        for mode in ("labeled", "unlabeled"):
            out = subprocess.run([os.path.join(REF, f"ref_plan_dump_{mode}"), path], check=True,
                                 capture_output=True, text=True).stdout
            rec = json.loads(out)
            rec["pattern"] = name
            plans.append(rec)
    with open(os.path.join(HERE, "plans.jsonl"), "w") as f:
        for rec in plans:
            f.write(json.dumps(rec, sort_keys=True) + "\n")
    roots = {}
    pick = ["cycle5", "clique4", "path4", "star4", "house", "rand03", "rand07", "cycle5_lab", "path5_lab",
            "house_lab", "cycle5_tail2_lab", "clique4_lab"]
    for gname in graphs:
        for pname in pick:
            path = os.path.join(tmp, pname + ".g")
            for mode in ("labeled", "unlabeled"):
                out = subprocess.run([os.path.join(REF, f"ref_roots_dump_{mode}"), os.path.join(gdir, gname), path],
                                     check=True, capture_output=True, text=True).stdout.split("\n")
                cnt = int(out[0])
                pairs = [[int(x) for x in line.split()] for line in out[1:1 + cnt]]
                roots[f"{gname}|{pname}|{mode}"] = {"count": cnt, "sha256": pairs_digest(pairs),
                                                    "head": pairs[:16]}
    with open(os.path.join(HERE, "roots.json"), "w") as f:
        json.dump(roots, f, separators=(",", ":"), sort_keys=True)
    print(f"wrote {len(graphs)} graphs, {len(pats)} patterns, {len(plans)} plans, {len(roots)} root lists")


if __name__ == "__main__":
    main()
