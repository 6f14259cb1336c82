"""Multi-GPU plumbing: one process per GPU, roots sharded across ranks.

The count is a sum over root edges, so the only exchange is one all-reduce of
per-pattern counts at the end (the reference's MPI driver does the same with
MPI_Reduce, test_mpi.cu:608).  Rank r takes root chunks r, r+W, r+2W, ...
(chunk-cyclic, the rule the kernel applies with shard_rank/shard_count), so
skewed root costs spread over all ranks.  `run_sharded` is the alternative
the reference's MPI driver uses: cost-balanced static ranges, then a dynamic
tail claimed from a shared counter.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple


def shard_ranges(n_roots: int, chunk: int, rank: int, world: int) -> List[Tuple[int, int]]:
    """Root index ranges [begin, end) owned by `rank` (chunk-cyclic)."""
    out = []
    c = rank
    while c * chunk < n_roots:
        out.append((c * chunk, min(n_roots, (c + 1) * chunk)))
        c += world
    return out


def reduce_counts(counts: Sequence[int], device=None) -> List[int]:
    """Sums per-pattern counts over all ranks (8 bytes per pattern)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [int(c) for c in counts]
    t = torch.tensor([int(c) for c in counts], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [int(x) for x in t.cpu()]


def max_over_ranks(values: Sequence[float], device=None) -> List[float]:
    """Element-wise max over ranks (device times are reported as the max)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def cost_split(pred_cost: Sequence[float], world: int, static_frac: float = 0.8) -> Tuple[List[Tuple[int, int]], int]:
    """Static part of a cost-balanced split (the reference's MPI driver: static
    slices, then dynamic claims; test_mpi.cu:317-349, 78-114).

    pred_cost holds the predicted cost of each root in queue order.  The
    shortest prefix holding static_frac of the total cost is cut into `world`
    contiguous ranges of about equal predicted cost; the returned tail start is
    where dynamic claims begin.
    """
    import numpy as np
    c = np.maximum(np.asarray(pred_cost, dtype=np.float64), 0.0)
    n = len(c)
    if n == 0 or world <= 0:
        return [(0, 0)] * max(world, 0), 0
    cum = np.cumsum(c)
    total = float(cum[-1])
    if total <= 0.0:
        tail = int(n * static_frac)
        cuts = [tail * r // world for r in range(world + 1)]
        return [(cuts[r], cuts[r + 1]) for r in range(world)], tail
    tail = int(np.searchsorted(cum, static_frac * total, side="left")) + 1
    tail = min(max(tail, 0), n)
    base = float(cum[tail - 1]) if tail > 0 else 0.0
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum[:tail], base * r / world, side="left")) + 1)
    cuts.append(tail)
    cuts = [min(max(x, 0), tail) for x in cuts]
    for r in range(1, len(cuts)):
        cuts[r] = max(cuts[r], cuts[r - 1])
    return [(cuts[r], cuts[r + 1]) for r in range(world)], tail


class DynamicClaims:
    """Claims [b, e) chunks of the tail [begin, end) from a shared counter in a
    torch.distributed store (atomic add), so the first rank to finish its
    static range takes the next chunk.  The counter key must be fresh per run."""

    def __init__(self, store, key: str, begin: int, end: int, chunk: int):
        self.store, self.key, self.begin, self.end, self.chunk = store, key, begin, end, max(1, chunk)

    def next(self):
        k = int(self.store.add(self.key, 1)) - 1
        b = self.begin + k * self.chunk
        if b >= self.end:
            return None
        return b, min(self.end, b + self.chunk)


def run_sharded(run_range: Callable[[int, int], Sequence[int]], n_patterns: int, n_roots: int, rank: int,
                world: int, store, key: str, pred_cost: Optional[Sequence[float]] = None,
                static_frac: float = 0.8, tail_chunk: int = 4096) -> List[int]:
    """This rank's share of a match over roots [0, n_roots): its static range
    (cost-balanced when pred_cost is given, else equal-sized), then tail chunks
    claimed dynamically.  run_range(b, e) returns per-pattern counts for root
    positions [b, e) (e.g. Context.match with root_begin/root_end and the
    root_order the costs were predicted in).  Returns the local sums; reduce
    them with reduce_counts."""
    if pred_cost is None:
        pred_cost = [1.0] * n_roots
    if len(pred_cost) != n_roots:
        raise ValueError("pred_cost must hold one cost per root")
    ranges, tail = cost_split(pred_cost, world, static_frac)
    total = [0] * n_patterns

    def add(c):
        nonlocal total
        if len(c) != n_patterns:
            raise ValueError("run_range returned the wrong number of counts")
        total = [int(a) + int(b) for a, b in zip(total, c)]

    b, e = ranges[rank]
    if e > b:
        add(run_range(b, e))
    claims = DynamicClaims(store, key, tail, n_roots, tail_chunk)
    while True:
        r = claims.next()
        if r is None:
            break
        add(run_range(*r))
    return total
