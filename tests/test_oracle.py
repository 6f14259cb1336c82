"""The CPU oracle against the reference's own root filter (golden fixtures),
against brute-force enumeration, and against closed forms."""
import hashlib
import json
import math
import os
import random
import struct

import numpy as np
import pytest

import brute
import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import patterns as P

GOLD = os.path.join(os.path.dirname(__file__), "golden")
PATTERNS = json.load(open(os.path.join(GOLD, "patterns.json")))
ROOTS = json.load(open(os.path.join(GOLD, "roots.json")))


def golden_graph(name, labeled):
    return pm.HostGraph.read(os.path.join(GOLD, "graphs", name), labeled=labeled)


def digest(pairs):
    h = hashlib.sha256()
    for r, c in pairs:
        h.update(struct.pack("<ii", int(r), int(c)))
    return h.hexdigest()


@pytest.mark.parametrize("key", sorted(ROOTS))
def test_oracle_roots_match_reference(key):
    gname, pname, mode = key.split("|")
    labeled = mode == "labeled"
    hg = golden_graph(gname, labeled)
    g = orc.Graph(hg.rowptr, hg.colidx, hg.labels)
    r = orc.roots(g, orc.plan(PATTERNS[pname], labeled))
    want = ROOTS[key]
    assert len(r) == want["count"]
    assert [list(map(int, x)) for x in r[:16]] == want["head"]
    assert digest(r) == want["sha256"]


def connected_prefix_pattern(r, k, nlab):
    edges = [(0, 1)] + [(r.randrange(i), i) for i in range(2, k)]
    edges += [(i, j) for i in range(k) for j in range(i + 1, k) if (i, j) not in edges and r.random() < 0.35]
    return P.to_g(k, edges, [r.randrange(nlab) for _ in range(k)])


@pytest.mark.parametrize("trial", range(60))
def test_oracle_vs_brute_force(trial):
    r = random.Random(1000 + trial)
    n = r.randint(6, 14)
    m = r.randint(n, min(n * (n - 1) // 2, 4 * n))
    hg = pm.gen_chung_lu(n, m, gamma=2.1, i0=1.0, max_w=0, seed=trial + 1)
    labs = pm.gen_labels(n, 2, seed=trial)
    text = connected_prefix_pattern(r, r.randint(3, 6), 2)
    gl = orc.Graph(hg.rowptr, hg.colidx, labs)
    gu = orc.Graph(hg.rowptr, hg.colidx, None)
    assert orc.total(gl, text, True) == brute.count_labeled(hg.rowptr, hg.colidx, labs, text)
    assert orc.total(gu, text, False) == brute.count_injective(hg.rowptr, hg.colidx, text)


def complete_graph(n):
    nb = [[j for j in range(n) if j != i] for i in range(n)]
    rowptr = np.zeros(n + 1, dtype=np.uint64)
    rowptr[1:] = np.cumsum([len(x) for x in nb])
    return rowptr, np.array([x for l in nb for x in l], dtype=np.int32)


def cycle_graph(n):
    nb = [sorted({(i - 1) % n, (i + 1) % n}) for i in range(n)]
    rowptr = np.zeros(n + 1, dtype=np.uint64)
    rowptr[1:] = np.cumsum([len(x) for x in nb])
    return rowptr, np.array([x for l in nb for x in l], dtype=np.int32)


@pytest.mark.parametrize("n,k", [(5, 3), (6, 4), (7, 5), (8, 6), (8, 7)])
def test_closed_form_cliques(n, k):
    rp, ci = complete_graph(n)
    g = orc.Graph(rp, ci, None)
    assert orc.total(g, P.to_g(*P.clique(k)), False) == math.factorial(n) // math.factorial(n - k)
    # cycles in K_n: n!/(n-k)! embeddings as well (every injective map works)
    assert orc.total(g, P.to_g(*P.cycle(k)), False) == math.factorial(n) // math.factorial(n - k)


@pytest.mark.parametrize("k", [3, 4, 5, 6, 7])
def test_closed_form_cycle_in_cycle(k):
    rp, ci = cycle_graph(k)
    g = orc.Graph(rp, ci, None)
    assert orc.total(g, P.to_g(*P.cycle(k)), False) == 2 * k
    rp, ci = cycle_graph(2 * k + 1)
    g = orc.Graph(rp, ci, None)
    # a path of k vertices in a long cycle C_m: 2m embeddings
    assert orc.total(g, P.to_g(*P.path(k)), False) == 2 * (2 * k + 1)


def test_truncation_is_identity_above_max_degree():
    hg = golden_graph("cl400", True)
    g = orc.Graph(hg.rowptr, hg.colidx, hg.labels)
    md = hg.max_degree
    for name in ("cycle5_lab", "house_lab", "path5_lab"):
        p = orc.plan(PATTERNS[name], True)
        r = orc.roots(g, p)
        exact, _ = orc.count(g, p, r)
        trunc, _ = orc.count(g, p, r, truncate=md)
        low, _ = orc.count(g, p, r, truncate=2)
        assert exact == trunc
        assert low <= exact


def test_per_root_counts_and_bytes_add_up():
    hg = golden_graph("rmat512", False)
    g = orc.Graph(hg.rowptr, hg.colidx, None)
    p = orc.plan(PATTERNS["cycle5"], False)
    r = orc.roots(g, p)
    c, st, per = orc.count(g, p, r, per_root=True)
    assert int(per.sum()) == c
    c2, st2 = orc.count(g, p, r, threads=3)
    assert c2 == c and st2["alg_bytes"] == st["alg_bytes"] and st2["set_ops"] == st["set_ops"]
    half = len(r) // 2
    a, sa = orc.count(g, p, r, 0, half)
    b, sb = orc.count(g, p, r, half, len(r))
    assert a + b == c and sa["alg_bytes"] + sb["alg_bytes"] == st["alg_bytes"]


def test_estimator_is_unbiased_enough():
    hg = golden_graph("cl400", False)
    g = orc.Graph(hg.rowptr, hg.colidx, None)
    p = orc.plan(PATTERNS["cycle4"], False)
    r = orc.roots(g, p)
    exact, st = orc.count(g, p, r)
    so, by, ct = orc.estimate(g, p, r, probes=20000, seed=3)
    assert abs(ct - exact) / max(exact, 1) < 0.25
    assert abs(so - st["set_ops"]) / st["set_ops"] < 0.25
