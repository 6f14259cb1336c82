"""Autotuner for the batched persistent launch.

Sweeps warps per block, root chunk size, donation threshold and -- for
paged graphs -- page size, timing each configuration with the device time the
library reports, and keeps the fastest per (graph, pattern set).  Every
configuration must return the same counts; a mismatch is an error, never a
faster answer.  The result is a JSON file the CLI and the bench can reuse.

The reference has no tuner: its knobs are compile-time constants edited by
`sed` (src/config.h:19-25, plot/plot_fig11.sh:89-97).
"""
from __future__ import annotations

import itertools
import json
import time
from typing import Callable, Dict, Iterable, List, Optional, Sequence

from . import PM_ERR_TIMEOUT, Context, GraphPreprocessor, HostGraph, PatternPreprocessor, PmError

WARPS = (4, 8, 16)
CHUNKS = (16, 32, 64, 128, 256, 512, 1024, 2048, 4096)
SPLITS = (16, 64, 256)
VARIANTS = (2, 3)  # kernel register caps: 85 (three 256-thread blocks per SM), uncapped
PAGE_KB = (16, 64, 256)
# the library's own defaults (pm_run_opts zeroed): always a candidate, so the
# tuned configuration is never slower than the untuned one
DEFAULT = {"warps_per_block": 8, "chunk": 16, "split_level1": 64, "high_occupancy": 0}


def _valid(w: int, v: int) -> bool:
    return v == 3 or w <= 8  # 16-warp blocks need the uncapped variant


def sweep(ctx: Context, graph: GraphPreprocessor, plans: Sequence[PatternPreprocessor], *,
          warps: Iterable[int] = WARPS, chunks: Iterable[int] = CHUNKS, splits: Iterable[int] = SPLITS,
          variants: Iterable[int] = VARIANTS, reps: int = 1, timeout_ms: int = 60000,
          extra: Optional[dict] = None) -> List[dict]:
    """Times the default configuration, then every valid (warps, chunk,
    split, kernel variant), on one placed graph.  A configuration that hits
    timeout_ms is dropped (kernel_ms None); one that changes a count is an
    error."""
    extra = extra or {}
    configs = [dict(DEFAULT, default=True)]
    for w, c, s, v in itertools.product(warps, chunks, splits, variants):
        if _valid(w, v):
            configs.append({"warps_per_block": w, "chunk": c, "split_level1": s, "high_occupancy": v})
    rows = []
    want = None
    for cfg in configs:
        kw = {k: cfg[k] for k in ("warps_per_block", "chunk", "split_level1", "high_occupancy")}
        best = None
        for _ in range(reps):
            try:
                counts, st = ctx.match(graph, list(plans), timeout_ms=timeout_ms, **kw, **extra)
            except PmError as e:
                if e.status != PM_ERR_TIMEOUT:
                    raise
                break  # slower than the limit: not a candidate (kernel_ms stays None)
            if want is None:
                want = counts
            if counts != want:
                raise RuntimeError(f"config {kw} changed the counts")
            ms = st["kernel_ms"]
            best = ms if best is None else min(best, ms)
        rows.append(dict(cfg, kernel_ms=best))
    return rows


def autotune(ctx: Context, hg: HostGraph, plans: Sequence[PatternPreprocessor], *, labeled: bool,
             paged: bool = False, frame_pool_bytes: int = 4 << 30, page_kb: Iterable[int] = PAGE_KB,
             out_json: Optional[str] = None, extra: Optional[dict] = None, **kw) -> dict:
    """Full sweep (page sizes too when paged); returns and optionally writes
    the best config.  extra: run options every configuration shares (a root
    range, say); paged sweeps start each run cold."""
    results = []
    for pk in (page_kb if paged else (None,)):
        g = GraphPreprocessor.from_host(hg, labeled=labeled, device=ctx.device, paged=paged,
                                        frame_pool_bytes=frame_pool_bytes,
                                        page_bytes=(pk << 10) if pk else 64 << 10)
        try:
            shared = dict(extra or {})
            if paged:
                shared["cold_cache"] = True
            for r in sweep(ctx, g, plans, extra=shared, **kw):
                r["page_kb"] = pk
                results.append(r)
        finally:
            g.close()
    done = [r for r in results if r["kernel_ms"] is not None]
    if not done:
        raise RuntimeError("every configuration hit the time limit")
    best = min(done, key=lambda r: r["kernel_ms"])
    out = {"best": best, "results": results, "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
    if out_json:
        with open(out_json, "w") as f:
            json.dump(out, f, indent=1)
    return out
