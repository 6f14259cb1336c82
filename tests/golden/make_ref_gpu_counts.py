"""Runs the REFERENCE's own GPU `test` binary on the golden graphs and records
its counts (tests/golden/ref_gpu_counts.json).

Needs a GPU and the binaries built by `make -C oracle ref` (oracle/_ref/
ref_test_{labeled,unlabeled}[_t16]: the reference's untouched sources with
LABELED / GRAPH_DEGREE selected by -include shims, device code built with -G
as the reference's Makefile does).  Reads only files under
this repository.

    python tests/golden/make_ref_gpu_counts.py --out ref_gpu_counts.json

Each record: graph, pattern, labeled, truncate (the binary's GRAPH_DEGREE),
count (last stdout line of the binary), ms.  The committed fixture is the
union of two runs (--graphs cl400,dense60, then --graphs rmat512,cl3000);
cases whose binary crashed twice on the host (SIGSEGV in the reference's
helper threads, no GPU fault) are absent.  Unlabeled patterns whose last
vertex is a fresh neighbour set are skipped: there the reference diffs a slot
it never wrote (src/gpu_match.cu:292 vs 534-568), so its count depends on
stale device memory.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
import pumatch_b200 as pm  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref")
VARIANTS = [("ref_test_labeled", True, 4096), ("ref_test_unlabeled", False, 4096),
            ("ref_test_labeled_t16", True, 16), ("ref_test_unlabeled_t16", False, 16)]
GRAPHS = ["cl400", "rmat512", "dense60", "cl3000"]
PATTERNS_LAB = ["cycle5_lab", "house_lab", "clique4_lab", "path5_lab", "cycle5_tail2_lab", "star5_lab"]
PATTERNS_UNL = ["cycle4", "cycle5", "clique4", "house", "star4", "rand03"]


def last_fresh(text: str) -> bool:
    d = pm.PatternPreprocessor(text=text, labeled=False).describe()
    return bool(d["set_ops"][d["nslots"] - 1] & 0x20)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--graphs", default=",".join(GRAPHS))
    ap.add_argument("--timeout", type=float, default=120)
    args = ap.parse_args()
    pats = json.load(open(os.path.join(HERE, "patterns.json")))
    tmp = tempfile.mkdtemp()
    recs = []
    for binary, labeled, T in VARIANTS:
        exe = os.path.join(REF, binary)
        for gname in args.graphs.split(","):
            for pname in (PATTERNS_LAB if labeled else PATTERNS_UNL):
                if not labeled and last_fresh(pats[pname]):
                    continue
                pfile = os.path.join(tmp, pname + ".g")
                open(pfile, "w").write(pats[pname])
                t0 = time.time()
                for attempt in range(2):  # the reference's host threads crash now and then (SIGSEGV)
                    r = subprocess.run([exe, os.path.join(HERE, "graphs", gname), pfile], capture_output=True,
                                       text=True, cwd=tmp, timeout=args.timeout)
                    if r.returncode == 0:
                        break
                if r.returncode != 0:
                    print(f"FAILED {binary} {gname} {pname}: rc={r.returncode}\n{r.stderr[-2000:]}", flush=True)
                    continue
                ms, count = r.stdout.strip().splitlines()[-1].split()
                recs.append({"graph": gname, "pattern": pname, "labeled": labeled, "truncate": T,
                             "count": int(count), "ms": float(ms), "binary": binary})
                print(binary, gname, pname, count, ms, f"{time.time() - t0:.1f}s", flush=True)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    with open(args.out, "w") as f:
        json.dump(recs, f, indent=1)
    print(f"wrote {len(recs)} records to {args.out}")


if __name__ == "__main__":
    main()
