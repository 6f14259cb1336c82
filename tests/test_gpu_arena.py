"""Candidate storage that scales with hub degrees: warps whose candidate sets
or copied lists outgrow their own arena borrow a worst-case arena from a pool
for the rest of the root.  Forced here with tiny own arenas (and a pool of one
arena, so warps queue for it) and with a hub whose list exceeds a warp's own
gather space under paging; every count must equal the oracle's, and the
launch must report that it borrowed.
"""
import os

import numpy as np
import pytest

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import patterns as P

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _oracle(hg, text, labeled, begin=0, end=None):
    g = orc.Graph(hg.rowptr, hg.colidx, hg.labels if labeled else None)
    p = orc.plan(text, labeled)
    r = orc.roots(g, p)
    end = len(r) if end is None else min(end, len(r))
    c, _, _, _, st = orc.count_split(g, p, r[begin:end], threads=os.cpu_count())
    return (c if labeled else c * p.multiplicity), st


CASES = [
    ("cl3000", False, P.to_g(*P.clique(4))),
    ("cl3000", False, P.to_g(*P.cycle(6))),
    ("cl3000", True, P.to_g(*P.cycle(5), [0, 0, 1, 1, 0])),
    ("rmat512", True, P.to_g(*P.cycle_tail(4, 2), [0, 1, 0, 1, 2, 0])),
    ("rmat512", False, P.to_g(*P.house())),
]


@pytest.mark.parametrize("paged", [False, True], ids=["hbm", "paged"])
@pytest.mark.parametrize("name,labeled,text", CASES)
def test_tiny_own_arenas_borrow_and_keep_counts(ctx, name, labeled, text, paged):
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", name), labeled=labeled)
    kw = dict(labeled=labeled)
    rng = {}
    if paged:
        # a pool of a few pages: most lists are read over the host link, so a
        # bounded range of roots
        kw.update(paged=True, page_bytes=4096, frame_pool_bytes=max(4096, hg.colidx.nbytes // 4 // 4096 * 4096))
        rng = dict(root_begin=0, root_end=150)
    want, ost = _oracle(hg, text, labeled, 0, rng.get("root_end"))
    g = pm.GraphPreprocessor.from_host(hg, **kw)
    p = pm.PatternPreprocessor(text=text, labeled=labeled)
    try:
        for own in (48, 200):
            got, st = ctx.match(g, [p], own_arena_words=own, timeout_ms=120000, **rng)
            assert got[0] == want, own
            assert st["set_ops"] == ost["set_ops"]
            assert st["arena_pool"] >= 1  # the own arena is below the plans' worst case
            if text == P.to_g(*P.cycle(6)) and not paged and own == 48:
                assert st["borrowed_arenas"] > 0  # its level-1 sets reach 537 words
        # a pool of one arena: warps queue for it (every root needs it, so
        # the roots run one at a time -- a small range of them)
        k = 100 if paged else 300
        want_k, ost_k = _oracle(hg, text, labeled, 0, k)
        got, st = ctx.match(g, [p], own_arena_words=48, max_borrowed=1, root_begin=0, root_end=k,
                            warps_per_block=4, blocks_per_sm=1, timeout_ms=120000)
        assert got[0] == want_k
        assert st["set_ops"] == ost_k["set_ops"] and st["arena_pool"] == 1
    finally:
        g.close()


def test_hub_lists_beyond_the_own_gather_space(ctx):
    """Paged lists longer than a warp's own gather half (16,384 words) are
    gathered into a borrowed arena."""
    hg = pm.gen_chung_lu(200_000, 2_000_000, gamma=2.0, i0=10.0, max_w=60_000.0, seed=21)
    assert hg.max_degree > 20_000
    # one label: a labeled slot's label group is the whole list, so the hub's
    # group exceeds the gather half too
    hg = pm.HostGraph(hg.rowptr, hg.colidx, pm.gen_labels(hg.n, 1, seed=22))
    cases = [(False, P.to_g(*P.clique(4)), 0, 3000), (True, P.to_g(*P.cycle(4), [0, 0, 0, 0]), 0, 150)]
    for labeled, text, b, e in cases:
        want, ost = _oracle(hg, text, labeled, b, e)
        g = pm.GraphPreprocessor.from_host(hg, labeled=labeled, paged=True, page_bytes=64 << 10,
                                           frame_pool_bytes=hg.colidx.nbytes // 2 // (64 << 10) * (64 << 10))
        p = pm.PatternPreprocessor(text=text, labeled=labeled)
        try:
            got, st = ctx.match(g, [p], root_begin=b, root_end=e, timeout_ms=300000)
            assert got[0] == want
            assert st["set_ops"] == ost["set_ops"]
            assert st["borrowed_arenas"] > 0
            hb = pm.GraphPreprocessor.from_host(hg, labeled=labeled)
            got2, _ = ctx.match(hb, [p], root_begin=b, root_end=e, own_arena_words=1000, timeout_ms=300000)
            hb.close()
            assert got2[0] == want
        finally:
            g.close()
