"""Resumable long runs.

A match is a sum over root edges, so a long run (an out-of-HBM graph, a
batch of heavy patterns) can be cut into root ranges whose partial counts
are saved after each range: an interrupted run resumes at the next range
instead of starting over.  The reference's persistent-interval job queue
(src/gpu_match.cu:321-384, test_mpi.cu:116-170) could restart from a job
index but never writes one down.

The state file is JSON, replaced atomically after every range:
{"key": ..., "n_roots": N, "n_patterns": P, "next": r, "counts": [...]}.
A state file written for another job (different key or sizes) is an error,
never silently reused or overwritten.
"""
from __future__ import annotations

import hashlib
import json
import os
from typing import Callable, List, Sequence


def _load(path: str):
    with open(path) as f:
        return json.load(f)


def _save(path: str, state: dict) -> None:
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(state, f)
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)


def run_resumable(run_range: Callable[[int, int], Sequence[int]], n_roots: int, n_patterns: int,
                  state_path: str, key: str, chunk_roots: int = 65536) -> List[int]:
    """Runs root positions [0, n_roots) in ranges of chunk_roots through
    run_range(b, e) -> per-pattern counts, saving the running sums and the
    next position to state_path after each range; continues from a state
    file of the same job.  Returns the per-pattern totals (the state file is
    left in place, complete, for the caller to remove)."""
    if chunk_roots <= 0 or n_roots < 0 or n_patterns <= 0:
        raise ValueError("bad chunk_roots, n_roots or n_patterns")
    if os.path.exists(state_path):
        state = _load(state_path)
        if (state.get("key") != key or state.get("n_roots") != n_roots
                or state.get("n_patterns") != n_patterns):
            raise ValueError(f"{state_path} belongs to another job")
    else:
        state = {"key": key, "n_roots": n_roots, "n_patterns": n_patterns, "next": 0, "counts": [0] * n_patterns}
        _save(state_path, state)
    while state["next"] < n_roots:
        b = state["next"]
        e = min(n_roots, b + chunk_roots)
        c = list(run_range(b, e))
        if len(c) != n_patterns:
            raise ValueError("run_range returned the wrong number of counts")
        state["counts"] = [int(x) + int(y) for x, y in zip(state["counts"], c)]
        state["next"] = e
        _save(state_path, state)
    return [int(x) for x in state["counts"]]


def job_key(graph_info: dict, plan_descs: Sequence[dict], options: dict, content: Sequence[str] = ()) -> str:
    """A digest naming a job: the placed graph's shape, the compiled plans,
    the run options that change counts, and digests of what the shape does
    not pin (each plan's root list -- the graph's edges and labels as the
    query sees them -- and a root order)."""
    blob = json.dumps({"graph": graph_info, "plans": list(plan_descs), "options": options,
                       "content": list(content)}, sort_keys=True, default=str)
    return hashlib.sha256(blob.encode()).hexdigest()


def roots_digest(ctx, graph, plan) -> str:
    """sha256 of a plan's root list on a placed graph (reference order)."""
    return hashlib.sha256(ctx.roots(graph, plan).tobytes()).hexdigest()


def match_resumable(ctx, graph, plans, state_path: str, chunk_roots: int = 65536, root_order=None,
                    **run_kw) -> List[int]:
    """Context.match over all root edges, one launch per range of chunk_roots
    root positions, resumable from state_path.  Counts equal one full
    launch's.  root_order (single plan): a host int32 array of root ids, the
    order positions are taken in; it is part of the job's key."""
    if "root_order_ptr" in run_kw or "root_begin" in run_kw or "root_end" in run_kw:
        raise ValueError("pass root_order as a host array; root ranges are this function's to choose")
    n_roots = max(ctx.count_roots(graph, p) for p in plans)
    info = {k: v for k, v in graph.info().items() if k in ("n_vertices", "n_adj", "max_degree", "labeled", "n_labels")}
    content = [roots_digest(ctx, graph, p) for p in plans]
    order_dev = None
    if root_order is not None:
        import numpy as np
        import torch
        order = np.ascontiguousarray(root_order, dtype=np.int32)
        if len(plans) != 1 or len(order) != n_roots:
            raise ValueError("root_order needs one plan and one entry per root")
        content.append("order:" + hashlib.sha256(order.tobytes()).hexdigest())
        order_dev = torch.from_numpy(order).to(f"cuda:{ctx.device}")
        run_kw["root_order_ptr"] = order_dev.data_ptr()
    key = job_key(info, [p.describe() for p in plans], {"truncate": run_kw.get("truncate", 0)}, content)

    def run_range(b, e):
        counts, _ = ctx.match(graph, list(plans), root_begin=b, root_end=e, **run_kw)
        return counts

    return run_resumable(run_range, n_roots, len(plans), state_path, key, chunk_roots)
