"""The configured queries' seeded root samples (tests/golden/root_samples.json)
and the generators they rest on.

CPU: the oracle's generators (used by the CPU measurement arm, which must not
load the product library) produce the product generators' arrays; the
fixture's graph digest and sampled root edges are reproduced; the oracle's
split runner gives orc_count's per-root counts.
GPU: the library's per-root counts on the sampled roots equal the fixture's
exact counts, and on cheap roots of the same query equal a live oracle run.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import patterns as P

GOLD = os.path.join(os.path.dirname(__file__), "golden")
_PATH = os.path.join(GOLD, "root_samples.json")
SAMPLES = json.load(open(_PATH)) if os.path.exists(_PATH) else {}
needs_sample = pytest.mark.skipif("chunglu100k_c7" not in SAMPLES, reason="root sample fixture not generated")


def _digest(rp, ci):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(rp, dtype=np.uint64).tobytes())
    h.update(np.ascontiguousarray(ci, dtype=np.int32).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("seed", [1, 9])
def test_oracle_generators_equal_product_generators(seed):
    a = pm.gen_chung_lu(20000, 90000, gamma=2.1, i0=10.0, max_w=500.0, seed=seed)
    rp, ci = orc.gen_chung_lu(20000, 90000, 2.1, 10.0, 500.0, seed)
    assert np.array_equal(a.rowptr, rp) and np.array_equal(a.colidx, ci)
    b = pm.gen_rmat(1 << 14, 12 << 14, a=0.57, b=0.19, c=0.19, seed=seed)
    rp, ci = orc.gen_rmat(1 << 14, 12 << 14, 0.57, 0.19, 0.19, seed)
    assert np.array_equal(b.rowptr, rp) and np.array_equal(b.colidx, ci)
    assert np.array_equal(pm.gen_labels(70000, 8, seed), orc.gen_labels(70000, 8, seed))


# the R-MAT record's graph (3.6e9 adjacency entries) is regenerated on the
# device by the bench that uses it, which checks its digest there
@pytest.mark.parametrize("name", sorted(k for k, v in SAMPLES.items() if v["graph"]["kind"] == "chung_lu"))
def test_sample_fixture_reproduces(name):
    rec = SAMPLES[name]
    gd = rec["graph"]
    rp, ci = orc.gen_chung_lu(gd["n"], gd["m"], gd["gamma"], gd["i0"], gd["max_w"], gd["seed"])
    assert _digest(rp, ci) == rec["graph_sha256"]
    hg = pm.gen_chung_lu(gd["n"], gd["m"], gamma=gd["gamma"], i0=gd["i0"], max_w=gd["max_w"], seed=gd["seed"])
    assert _digest(hg.rowptr, hg.colidx) == rec["graph_sha256"]
    g = orc.Graph(rp, ci, None)
    p = orc.plan(rec["pattern"], rec["labeled"])
    r = orc.roots(g, p)
    assert len(r) == rec["n_roots_total"]
    for s in rec["roots"]:
        assert tuple(r[s["index"]]) == (s["v0"], s["v1"])
        assert s["count"] == s["raw_count"] * rec["multiplicity"]
    assert sum(s["raw_count"] for s in rec["roots"]) == rec["raw_count"]


def test_split_runner_equals_plain_dfs():
    rp, ci = orc.gen_chung_lu(5000, 30000, 2.1, 10.0, 300.0, 3)
    g = orc.Graph(rp, ci, None)
    for text in (P.to_g(*P.cycle(6)), P.to_g(*P.clique(4)), P.to_g(*P.path(3))):
        p = orc.plan(text, False)
        r = orc.roots(g, p)[::7]
        c0, st0, pr0 = orc.count(g, p, r, per_root=True)
        c1, pr1, done, tot, st1 = orc.count_split(g, p, r, threads=4, shuffle_seed=5)
        assert c0 == c1 and done == tot
        assert np.array_equal(pr0, pr1)
        assert st0 == st1


@pytest.mark.gpu
@needs_sample
def test_gpu_sampled_roots_equal_fixture():
    import torch
    rec = SAMPLES["chunglu100k_c7"]
    gd = rec["graph"]
    hg = pm.gen_chung_lu(gd["n"], gd["m"], gamma=gd["gamma"], i0=gd["i0"], max_w=gd["max_w"], seed=gd["seed"])
    ctx = pm.Context(0)
    g = pm.GraphPreprocessor.from_host(hg, labeled=False)
    p = pm.PatternPreprocessor(text=rec["pattern"], labeled=False)
    idx = [s["index"] for s in rec["roots"]]
    order = torch.tensor(idx, dtype=torch.int32, device="cuda")
    rc = torch.zeros(rec["n_roots_total"], dtype=torch.int64, device="cuda")
    counts, st = ctx.match(g, [p], root_order_ptr=order.data_ptr(), root_begin=0, root_end=len(idx),
                           root_counts_ptr=rc.data_ptr(), timeout_ms=300000)
    got = rc.cpu().numpy()
    assert [int(got[i]) for i in idx] == [s["raw_count"] for s in rec["roots"]]
    assert counts[0] == rec["count"]
    assert st["set_ops"] == rec["set_ops"] and st["alg_bytes"] == rec["alg_bytes"]
    g.close()
    ctx.close()


@pytest.mark.gpu
def test_gpu_cheap_c7_roots_equal_live_oracle():
    """The configured 7-cycle on the configured graph: the first root edges in
    reference order (v0 is the cycle's largest id, so they are the cheap
    ones), per root, against the oracle."""
    import torch
    hg = pm.gen_chung_lu(100_000, 1_000_000, gamma=2.1, i0=10.0, max_w=5000.0, seed=1)
    text = P.to_g(*P.cycle(7))
    og = orc.Graph(hg.rowptr, hg.colidx, None)
    op = orc.plan(text, False)
    roots = orc.roots(og, op)
    k = 400
    want_total, want, _, _, ost = orc.count_split(og, op, roots[:k], threads=os.cpu_count())
    ctx = pm.Context(0)
    g = pm.GraphPreprocessor.from_host(hg, labeled=False)
    p = pm.PatternPreprocessor(text=text, labeled=False)
    rc = torch.zeros(len(roots), dtype=torch.int64, device="cuda")
    counts, st = ctx.match(g, [p], root_begin=0, root_end=k, root_counts_ptr=rc.data_ptr(), timeout_ms=300000)
    assert np.array_equal(rc.cpu().numpy()[:k].astype(np.uint64), want)
    assert counts[0] == want_total * op.multiplicity
    assert st["set_ops"] == ost["set_ops"]
    g.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("n,m,seed", [(1 << 14, 12 << 14, 2), (50_000, 400_000, 7), (1 << 10, 100_000, 3),
                                      (1 << 17, 16 << 17, 2)])
def test_device_rmat_generator_equals_host_generator(n, m, seed):
    """The device generator returns the host generator's arrays (the same draw
    sequence, the first m distinct edges), including when its first pass draws
    too few distinct edges (the dense 1,024-vertex case)."""
    a = pm.gen_rmat(n, m, a=0.57, b=0.19, c=0.19, seed=seed)
    b = pm.gen_rmat(n, m, a=0.57, b=0.19, c=0.19, seed=seed, device=0)
    assert np.array_equal(a.rowptr, b.rowptr)
    assert np.array_equal(a.colidx, b.colidx)
