"""Launches that overlap on one device: two contexts on their own streams,
driven from two host threads, each running a different pattern at the same
time (and a prepared query replaying beside a plain launch).  Every launch
carries its own plans, so each count must equal the oracle's.
"""
import os
import threading

import pytest

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import patterns as P

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _oracle(hg, text, labeled):
    g = orc.Graph(hg.rowptr, hg.colidx, hg.labels if labeled else None)
    p = orc.plan(text, labeled)
    c, _ = orc.count(g, p, orc.roots(g, p), threads=os.cpu_count())
    return c if labeled else c * p.multiplicity


def _run_pair(jobs, reps=4):
    """Runs each job(rep) in its own thread, all reps at once; returns results."""
    out = [[None] * reps for _ in jobs]
    errs = []
    barrier = threading.Barrier(len(jobs))

    def worker(j, fn):
        try:
            for r in range(reps):
                barrier.wait(timeout=60)
                out[j][r] = fn()
        except Exception as e:  # surfaced below
            errs.append(e)
            barrier.abort()

    th = [threading.Thread(target=worker, args=(j, fn)) for j, fn in enumerate(jobs)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    assert not errs, errs
    return out


def test_two_contexts_different_patterns_at_once():
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", "cl3000"), labeled=False)
    texts = [P.to_g(*P.clique(5)), P.to_g(*P.cycle(6))]
    want = [_oracle(hg, t, False) for t in texts]
    ctxs = [pm.Context(0), pm.Context(0)]
    g = pm.GraphPreprocessor.from_host(hg, labeled=False)
    plans = [pm.PatternPreprocessor(text=t, labeled=False) for t in texts]
    try:
        res = _run_pair([lambda i=i: ctxs[i].match(g, [plans[i]], timeout_ms=120000)[0][0] for i in range(2)])
        for i in range(2):
            assert res[i] == [want[i]] * len(res[i]), (texts[i], res[i], want[i])
    finally:
        g.close()
        for c in ctxs:
            c.close()


def test_prepared_query_beside_plain_launch():
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", "cl3000"), labeled=True)
    t_lab = P.to_g(*P.cycle(5), [0, 0, 1, 1, 0])
    t_other = P.to_g(*P.cycle(4), [1, 0, 1, 0])
    want = [_oracle(hg, t_lab, True), _oracle(hg, t_other, True)]
    ctxs = [pm.Context(0), pm.Context(0)]
    g = pm.GraphPreprocessor.from_host(hg, labeled=True)
    p0 = pm.PatternPreprocessor(text=t_lab, labeled=True)
    p1 = pm.PatternPreprocessor(text=t_other, labeled=True)
    q = ctxs[0].prepare(g, [p0], timeout_ms=120000)
    try:
        res = _run_pair([lambda: q.run()[0][0], lambda: ctxs[1].match(g, [p1], timeout_ms=120000)[0][0]])
        assert res[0] == [want[0]] * len(res[0])
        assert res[1] == [want[1]] * len(res[1])
    finally:
        q.close()
        g.close()
        for c in ctxs:
            c.close()
