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
CHUNKS = (32, 64, 128, 256, 512, 1024, 2048, 4096)
SPLITS = (16, 64, 256)
PAGE_KB = (16, 64, 256)


def sweep(ctx: Context, graph: GraphPreprocessor, plans: Sequence[PatternPreprocessor], *,
          warps: Iterable[int] = WARPS, chunks: Iterable[int] = CHUNKS, splits: Iterable[int] = SPLITS,
          reps: int = 1, timeout_ms: int = 60000, extra: Optional[dict] = None) -> List[dict]:
    """Times every (warps, chunk, split) on one placed graph."""
    extra = extra or {}
    rows = []
    want = None
    for w, c, s in itertools.product(warps, chunks, splits):
        best = None
        for _ in range(reps):
            try:
                counts, st = ctx.match(graph, list(plans), warps_per_block=w, chunk=c, split_level1=s,
                                       timeout_ms=timeout_ms, **extra)
            except PmError as e:
                if e.status != PM_ERR_TIMEOUT:
                    raise
                break  # slower than the limit: not a candidate (kernel_ms stays None)
            if want is None:
                want = counts
            if counts != want:
                raise RuntimeError(f"config warps={w} chunk={c} split={s} changed the counts")
            ms = st["kernel_ms"]
            best = ms if best is None else min(best, ms)
        rows.append({"warps_per_block": w, "chunk": c, "split_level1": s, "kernel_ms": best})
    return rows


def autotune(ctx: Context, hg: HostGraph, plans: Sequence[PatternPreprocessor], *, labeled: bool,
             paged: bool = False, frame_pool_bytes: int = 4 << 30, page_kb: Iterable[int] = PAGE_KB,
             out_json: Optional[str] = None, **kw) -> dict:
    """Full sweep (page sizes too when paged); returns and optionally writes the best config."""
    results = []
    for pk in (page_kb if paged else (None,)):
        g = GraphPreprocessor.from_host(hg, labeled=labeled, device=ctx.device, paged=paged,
                                        frame_pool_bytes=frame_pool_bytes,
                                        page_bytes=(pk << 10) if pk else 64 << 10)
        try:
            extra = {"cold_cache": True} if paged else {}
            for r in sweep(ctx, g, plans, extra=extra, **kw):
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
