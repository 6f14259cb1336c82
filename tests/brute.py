"""Brute-force enumerators for tiny graphs -- independent of the plan machinery.

Used by the oracle tests: the oracle (a restatement of the reference's slot
plan) must agree with these direct definitions of what the reference counts.

  labeled   : label-preserving homomorphisms v0..v{k-1} whose root edge
              (v0, v1) passes the reference's root filter (src/job_queue.h:39-64);
              pattern vertices that are not adjacent may share a data vertex
              (no diff step when LABELED, src/gpu_match.cu:534, 730).
  unlabeled : injective homomorphisms (embeddings, automorphisms included),
              i.e. the reference's count after x |Aut| (test.cu:198).
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple


def parse_g(text: str):
    labels, edges = [], []
    for line in text.splitlines():
        t = line.split()
        if not t or t[0].startswith("#"):
            continue
        if t[0] == "v":
            labels.append(int(t[2]))
        elif t[0] == "e" and int(t[3]) != 0:
            a, b = int(t[1]), int(t[2])
            if (b, a) not in edges and (a, b) not in edges:
                edges.append((a, b))
    return len(labels), labels, edges


def adjacency(rowptr, colidx):
    n = len(rowptr) - 1
    return [set(int(x) for x in colidx[rowptr[v]:rowptr[v + 1]]) for v in range(n)]


def count_labeled(rowptr, colidx, glabels, gtext: str) -> int:
    k, plab, pedges = parse_g(gtext)
    adj = adjacency(rowptr, colidx)
    n = len(adj)
    deg = [len(a) for a in adj]
    pdeg = [sum(1 for e in pedges if i in e) for i in range(k)]
    need = [[j for j in range(i) if (i, j) in pedges or (j, i) in pedges] for i in range(k)]
    total = 0

    def rec(path: List[int]):
        nonlocal total
        i = len(path)
        if i == k:
            total += 1
            return
        for v in (adj[path[need[i][0]]] if need[i] else range(n)):
            if glabels[v] != plab[i]:
                continue
            if all(v in adj[path[j]] for j in need[i]):
                rec(path + [v])

    for r in range(n):
        if glabels[r] != plab[0] or deg[r] < pdeg[0]:
            continue
        for c in sorted(adj[r]):
            if glabels[c] != plab[1] or deg[c] < pdeg[1]:
                continue
            if not any(deg[d] >= pdeg[2] for d in adj[c]):
                continue
            rec([r, c])
    return total


def count_injective(rowptr, colidx, gtext: str) -> int:
    k, _, pedges = parse_g(gtext)
    adj = adjacency(rowptr, colidx)
    n = len(adj)
    need = [[j for j in range(i) if (i, j) in pedges or (j, i) in pedges] for i in range(k)]
    total = 0

    def rec(path: List[int]):
        nonlocal total
        i = len(path)
        if i == k:
            total += 1
            return
        cands = adj[path[need[i][0]]] if need[i] else range(n)
        for v in cands:
            if v in path:
                continue
            if all(v in adj[path[j]] for j in need[i]):
                rec(path + [v])

    for r in range(n):
        for c in adj[r]:
            rec([r, c])
    return total
