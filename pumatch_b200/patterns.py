"""Pattern (.g) generation for synthetic workloads.

Writes the reference's gSpan-like format (pattern/*.g): ``v <id> <label>``
lines, then ``e <a> <b> 1`` lines listing each edge in both directions, as the
reference's own pattern files do.  Shapes: cliques, cycles, stars, paths,
house, house+tail and the cycle-with-pendant-path of the labeled workloads.
"""
from __future__ import annotations

import random
from typing import List, Optional, Sequence, Tuple

Edge = Tuple[int, int]


def clique(k: int) -> Tuple[int, List[Edge]]:
    return k, [(i, j) for i in range(k) for j in range(i + 1, k)]


def cycle(k: int) -> Tuple[int, List[Edge]]:
    return k, [(i, (i + 1) % k) for i in range(k)]


def star(k: int) -> Tuple[int, List[Edge]]:
    """k vertices: centre 0 and k-1 leaves."""
    return k, [(0, i) for i in range(1, k)]


def path(k: int) -> Tuple[int, List[Edge]]:
    return k, [(i, i + 1) for i in range(k - 1)]


def house() -> Tuple[int, List[Edge]]:
    """Square 0-1-2-3 with roof vertex 4 on the edge 0-1."""
    return 5, [(0, 1), (1, 2), (2, 3), (3, 0), (4, 0), (4, 1)]


def house_tail(tail: int = 1) -> Tuple[int, List[Edge]]:
    """House plus a pendant path of `tail` vertices hanging off vertex 4."""
    n, e = house()
    prev = 4
    for t in range(tail):
        e.append((prev, n + t))
        prev = n + t
    return n + tail, e


def cycle_tail(k: int = 5, tail: int = 2) -> Tuple[int, List[Edge]]:
    """k-cycle 0..k-1 plus a pendant path of `tail` vertices from vertex k-1."""
    n, e = cycle(k)
    prev = k - 1
    for t in range(tail):
        e.append((prev, n + t))
        prev = n + t
    return n + tail, e


SHAPES = {
    "clique": clique, "cycle": cycle, "star": star, "path": path,
}


def to_g(n: int, edges: Sequence[Edge], labels: Optional[Sequence[int]] = None) -> str:
    labels = list(labels) if labels is not None else [1] * n
    lines = [f"v {i} {labels[i]}" for i in range(n)]
    for a, b in edges:
        lines.append(f"e {a} {b} 1")
        lines.append(f"e {b} {a} 1")
    return "\n".join(lines) + "\n"


def seeded_labels(n: int, n_labels: int, seed: int) -> List[int]:
    r = random.Random(seed)
    return [r.randrange(n_labels) for _ in range(n)]


def batch_of_20(seed: int = 303, n_labels: int = 8) -> List[Tuple[str, str]]:
    """Twenty seeded 4-7-vertex shapes (cliques K4-K6, cycles C4-C7, stars,
    paths P4-P7, house, house+tail, plus extra cycles/houses), labels uniform
    over n_labels.  Returns (name, .g text) pairs."""
    shapes = [("K4", clique(4)), ("K5", clique(5)), ("K6", clique(6)),
              ("C4", cycle(4)), ("C5", cycle(5)), ("C6", cycle(6)), ("C7", cycle(7)),
              ("S4", star(4)), ("S5", star(5)), ("S6", star(6)),
              ("P4", path(4)), ("P5", path(5)), ("P6", path(6)), ("P7", path(7)),
              ("house", house()), ("house_tail1", house_tail(1)), ("house_tail2", house_tail(2)),
              ("C5_tail2", cycle_tail(5, 2)), ("C4_tail2", cycle_tail(4, 2)), ("C6_tail1", cycle_tail(6, 1))]
    r = random.Random(seed)
    out = []
    for name, (n, e) in shapes:
        labs = [r.randrange(n_labels) for _ in range(n)]
        out.append((name, to_g(n, e, labs)))
    return out
