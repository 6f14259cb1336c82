"""Multi-GPU plumbing: one process per GPU, roots sharded across ranks.

The count is a sum over root edges, so the only exchange is one all-reduce of
per-pattern counts at the end (the reference's MPI driver does the same with
MPI_Reduce, test_mpi.cu:608).  Rank r takes root chunks r, r+W, r+2W, ...
(chunk-cyclic, the rule the kernel applies with shard_rank/shard_count), so
skewed root costs spread over all ranks.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


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
