"""CUDA path vs the oracle (and the reference's own outputs), through the C-ABI.

Bar: bit-exact counts (integer work), identical root lists, identical
set-operation counts and algorithmic bytes (the kernel executes the same set
operations as the reference's DFS).
"""
import hashlib
import json
import os
import random
import struct
import subprocess

import numpy as np
import pytest
import torch

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import patterns as P

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
PATTERNS = json.load(open(os.path.join(GOLD, "patterns.json")))
ROOTS = json.load(open(os.path.join(GOLD, "roots.json")))
GRAPHS = ("cl400", "rmat512", "dense60", "cl3000")
_cache = {}


def host_graph(name, labeled):
    key = (name, labeled)
    if key not in _cache:
        _cache[key] = pm.HostGraph.read(os.path.join(GOLD, "graphs", name), labeled=labeled)
    return _cache[key]


def dev_graph(name, labeled):
    key = ("dev", name, labeled)
    if key not in _cache:
        _cache[key] = pm.GraphPreprocessor.from_host(host_graph(name, labeled), labeled=labeled)
    return _cache[key]


def oracle_count(hg, text, labeled, truncate=0, threads=os.cpu_count()):
    key = ("oracle", id(hg), text, labeled, truncate)
    if key not in _cache:
        g = orc.Graph(hg.rowptr, hg.colidx, hg.labels if labeled else None)
        p = orc.plan(text, labeled)
        r = orc.roots(g, p)
        c, st = orc.count(g, p, r, truncate=truncate, threads=threads)
        _cache[key] = ((c if labeled else c * p.multiplicity), st)
    return _cache[key]


def digest(pairs):
    h = hashlib.sha256()
    for r, c in pairs:
        h.update(struct.pack("<ii", int(r), int(c)))
    return h.hexdigest()


@pytest.mark.parametrize("key", sorted(ROOTS))
def test_gpu_roots_match_reference(ctx, key):
    gname, pname, mode = key.split("|")
    labeled = mode == "labeled"
    r = ctx.roots(dev_graph(gname, labeled), pm.PatternPreprocessor(text=PATTERNS[pname], labeled=labeled))
    want = ROOTS[key]
    assert len(r) == want["count"]
    assert digest(r) == want["sha256"]


COUNT_PATTERNS = ["cycle4", "cycle5", "clique4", "clique5", "path4", "path5", "star4", "star5", "house",
                  "house_tail1", "cycle5_tail2", "rand03", "rand07", "rand11", "rand19", "cycle5_lab",
                  "path5_lab", "house_lab", "cycle5_tail2_lab", "clique4_lab", "star5_lab"]


MODES = {"default": {}, "perlane": {"leaf_per_lane": 1}, "nosubtree": {"lane_subtree_max": -1},
         "subtree512": {"lane_subtree_max": 512}}


@pytest.mark.parametrize("gname", GRAPHS)
@pytest.mark.parametrize("labeled", [True, False], ids=["lab", "unl"])
@pytest.mark.parametrize("mode", sorted(MODES))
def test_gpu_counts_match_oracle(ctx, gname, labeled, mode):
    """Every last-level scheme (work-balanced across the warp, one candidate
    per lane, the last two levels one candidate per lane for clique-like
    plans at any parent size or never) gives the oracle's counts, set
    operations and bytes."""
    if labeled and mode in ("nosubtree", "subtree512"):
        pytest.skip("the two-level lane scheme is for unlabeled plans only")
    hg = host_graph(gname, labeled)
    g = dev_graph(gname, labeled)
    names = COUNT_PATTERNS + ([] if labeled else ["clique6", "clique7"])
    for pname in names:
        if not labeled and pname.startswith("cycle5_tail2"):
            continue  # minutes of oracle time unlabeled; covered labeled and on the small graphs
        text = PATTERNS[pname]
        want, st = oracle_count(hg, text, labeled)
        got, gst = ctx.match(g, [pm.PatternPreprocessor(text=text, labeled=labeled)], **MODES[mode])
        assert got[0] == want, (gname, pname)
        assert gst["set_ops"] == st["set_ops"], (gname, pname)
        assert gst["alg_bytes"] == st["alg_bytes"], (gname, pname)
        assert gst["device_status"] == 0


@pytest.mark.parametrize("T", [4, 16, 40])
@pytest.mark.parametrize("labeled", [True, False], ids=["lab", "unl"])
def test_gpu_truncation_emulation(ctx, T, labeled):
    hg = host_graph("cl3000", labeled)
    g = dev_graph("cl3000", labeled)
    for pname in ("cycle4", "path4", "star4", "house", "cycle5_lab", "house_lab"):
        text = PATTERNS[pname]
        want, _ = oracle_count(hg, text, labeled, truncate=T)
        got, _ = ctx.match(g, [pm.PatternPreprocessor(text=text, labeled=labeled)], truncate=T)
        assert got[0] == want, (pname, T)


def test_gpu_per_root_counts(ctx):
    hg = host_graph("rmat512", False)
    g = dev_graph("rmat512", False)
    text = PATTERNS["cycle5"]
    og = orc.Graph(hg.rowptr, hg.colidx, None)
    p = orc.plan(text, False)
    r = orc.roots(og, p)
    c, st, per = orc.count(og, p, r, per_root=True)
    buf = torch.zeros(len(r), dtype=torch.int64, device="cuda")
    cost = torch.zeros(len(r), dtype=torch.float32, device="cuda")
    got, _ = ctx.match(g, [pm.PatternPreprocessor(text=text, labeled=False)], root_counts_ptr=buf.data_ptr(),
                       root_cost_ptr=cost.data_ptr())
    assert got[0] == c * p.multiplicity
    assert np.array_equal(buf.cpu().numpy().astype(np.uint64), per)
    assert abs(float(cost.sum()) - st["alg_bytes"]) / st["alg_bytes"] < 1e-3


def test_gpu_batched_launch(ctx):
    hg = host_graph("cl3000", True)
    g = dev_graph("cl3000", True)
    batch = P.batch_of_20(seed=303, n_labels=2)
    plans = [pm.PatternPreprocessor(text=t, labeled=True) for _, t in batch]
    got, st = ctx.match(g, plans)
    for (name, text), c in zip(batch, got):
        want, _ = oracle_count(hg, text, True)
        assert c == want, name
    single = [ctx.match(g, [p])[0][0] for p in plans]
    assert single == got


@pytest.mark.parametrize("wpb", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("chunk", [1, 7, 64])
def test_gpu_launch_shapes(ctx, wpb, chunk):
    hg = host_graph("cl400", False)
    g = dev_graph("cl400", False)
    for pname in ("house", "clique5", "path5", "star5"):
        text = PATTERNS[pname]
        want, st = oracle_count(hg, text, False)
        for split in (-1, 1, 8):
            for high in ((0, 3) if wpb == 16 else (0, 1, 2, 3)):
                got, gst = ctx.match(g, [pm.PatternPreprocessor(text=text, labeled=False)], warps_per_block=wpb,
                                     chunk=chunk, split_level1=split, high_occupancy=high)
                assert got[0] == want, (pname, wpb, chunk, split, high)
                assert gst["set_ops"] == st["set_ops"] and gst["alg_bytes"] == st["alg_bytes"]


def test_gpu_shards_and_root_ranges(ctx):
    hg = host_graph("cl3000", False)
    g = dev_graph("cl3000", False)
    p = pm.PatternPreprocessor(text=PATTERNS["cycle5"], labeled=False)
    total = ctx.match(g, [p])[0][0]
    for k in (2, 3, 5):
        parts = [ctx.match(g, [p], shard_rank=i, shard_count=k, chunk=4)[0][0] for i in range(k)]
        assert sum(parts) == total
    n = ctx.count_roots(g, p)
    cut = n // 3
    a = ctx.match(g, [p], root_begin=0, root_end=cut)[0][0]
    b = ctx.match(g, [p], root_begin=cut, root_end=n)[0][0]
    assert a + b == total
    # per-root counts are indexed by root id whatever the range, and a range
    # with an order covers those positions of the order
    full = torch.zeros(n, dtype=torch.int64, device="cuda")
    ctx.match(g, [p], root_counts_ptr=full.data_ptr())
    parts = torch.zeros(n, dtype=torch.int64, device="cuda")
    ctx.match(g, [p], root_begin=0, root_end=cut, root_counts_ptr=parts.data_ptr())
    ctx.match(g, [p], root_begin=cut, root_end=n, root_counts_ptr=parts.data_ptr())
    assert torch.equal(parts, full)
    order = torch.from_numpy(np.random.default_rng(5).permutation(n).astype(np.int32)).cuda()
    byorder = torch.zeros(n, dtype=torch.int64, device="cuda")
    got = [ctx.match(g, [p], root_order_ptr=order.data_ptr(), root_begin=lo, root_end=hi,
                     root_counts_ptr=byorder.data_ptr())[0][0] for lo, hi in ((0, cut), (cut, 2 * cut), (2 * cut, n))]
    assert sum(got) == total and torch.equal(byorder, full)
    first = order[:cut].long()
    assert got[0] == int(full[first].sum()) * p.PatternMultiplicity


def small_graph(edges, n):
    nb = [[] for _ in range(n)]
    for a, b in edges:
        nb[a].append(b)
        nb[b].append(a)
    nb = [sorted(set(x)) for x in nb]
    rowptr = np.zeros(n + 1, dtype=np.uint64)
    rowptr[1:] = np.cumsum([len(x) for x in nb])
    colidx = np.array([x for l in nb for x in l], dtype=np.int32)
    return pm.HostGraph(rowptr, colidx, np.zeros(n, dtype=np.uint32))


def test_gpu_edge_cases(ctx):
    # no edges at all
    hg = small_graph([], 5)
    g = pm.GraphPreprocessor.from_host(hg, labeled=False)
    assert ctx.match(g, [pm.PatternPreprocessor(text=P.to_g(*P.cycle(4)), labeled=False)])[0] == [0]
    # isolated vertices around a triangle; 3-vertex patterns (last level = level 1)
    hg = small_graph([(1, 2), (2, 3), (1, 3)], 6)
    g = pm.GraphPreprocessor.from_host(hg, labeled=False)
    assert ctx.match(g, [pm.PatternPreprocessor(text=P.to_g(*P.clique(3)), labeled=False)])[0] == [6]
    assert ctx.match(g, [pm.PatternPreprocessor(text=P.to_g(*P.path(3)), labeled=False)])[0] == [6]
    # labeled pattern whose labels do not occur: no roots, count 0
    gl = pm.GraphPreprocessor.from_host(hg, labeled=True)
    txt = P.to_g(3, [(0, 1), (1, 2)], [5, 5, 5])
    assert ctx.count_roots(gl, pm.PatternPreprocessor(text=txt, labeled=True)) == 0
    assert ctx.match(gl, [pm.PatternPreprocessor(text=txt, labeled=True)])[0] == [0]
    # labeled plan on an unlabeled graph is an error, not a silent zero
    with pytest.raises(pm.PmError) as e:
        ctx.match(g, [pm.PatternPreprocessor(text=txt, labeled=True)])
    assert e.value.status == pm.PM_ERR_INVALID


def test_gpu_larger_random_graph(ctx):
    hg = pm.gen_chung_lu(20000, 100000, gamma=2.1, i0=10.0, max_w=300.0, seed=21)
    lab = pm.gen_labels(hg.n, 4, seed=22)
    hgl = pm.HostGraph(hg.rowptr, hg.colidx, lab)
    g = pm.GraphPreprocessor.from_host(hgl, labeled=True)
    for name in ("cycle5_lab", "house_lab", "cycle5_tail2_lab", "clique4_lab"):
        text = PATTERNS[name]
        want, _ = oracle_count(hgl, text, True, threads=8)
        got, st = ctx.match(g, [pm.PatternPreprocessor(text=text, labeled=True)])
        assert got[0] == want, name
    gu = pm.GraphPreprocessor.from_host(hg, labeled=False)
    for name in ("cycle4", "clique4", "house"):
        want, _ = oracle_count(hg, PATTERNS[name], False, threads=8)
        assert ctx.match(gu, [pm.PatternPreprocessor(text=PATTERNS[name], labeled=False)])[0][0] == want


def test_gpu_graph_from_device(ctx):
    hg = host_graph("rmat512", True)
    rp = torch.from_numpy(hg.rowptr.astype(np.int64)).cuda()
    ci = torch.from_numpy(hg.colidx).cuda()
    lb = torch.from_numpy(hg.labels.astype(np.uint8)).cuda()
    g = pm.GraphPreprocessor.from_device(hg.n, hg.n_adj, hg.max_degree, rp.data_ptr(), ci.data_ptr(),
                                         lb.data_ptr())
    p = pm.PatternPreprocessor(text=PATTERNS["house_lab"], labeled=True)
    assert ctx.match(g, [p])[0] == ctx.match(dev_graph("rmat512", True), [p])[0]


def test_gpu_cli_output(tmp_path):
    pat = tmp_path / "c5.g"
    pat.write_text(PATTERNS["cycle5_lab"])
    prefix = os.path.join(GOLD, "graphs", "cl400")
    r = subprocess.run([pm.CLI_PATH, prefix, str(pat)], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    ms, count = r.stdout.strip().splitlines()[-1].split()
    float(ms)
    want, _ = oracle_count(host_graph("cl400", True), PATTERNS["cycle5_lab"], True)
    assert int(count) == want
    rec = (tmp_path / "result.txt").read_text().strip().split("\t")
    assert rec[0] == prefix and rec[1] == str(pat) and int(rec[3]) == want
    # the JSON sidecar carries the same count and the launch's counters
    side = tmp_path / "stats.json"
    r = subprocess.run([pm.CLI_PATH, prefix, str(pat), "--json=" + str(side)], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    d = json.loads(side.read_text())
    assert d["counts"] == [want] and d["set_ops"] > 0 and d["device_status"] == 0
    r = subprocess.run([pm.CLI_PATH, prefix, str(pat), "--labeled=0", "--truncate=8"], capture_output=True,
                       text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    want, _ = oracle_count(host_graph("cl400", False), PATTERNS["cycle5_lab"], False, truncate=8)
    assert int(r.stdout.strip().splitlines()[-1].split()[1]) == want
    # launch configuration from an autotuner record, then overridden by a flag
    tuned = tmp_path / "tuned.json"
    tuned.write_text('{"best": {"warps_per_block": 16, "chunk": 32, "split_level1": 16, "high_occupancy": 3, '
                     '"page_kb": null, "kernel_ms": 1.0}, "results": []}')
    r = subprocess.run([pm.CLI_PATH, prefix, str(pat), "--tuned=" + str(tuned), "--chunk=8"], capture_output=True,
                       text=True, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    want, _ = oracle_count(host_graph("cl400", True), PATTERNS["cycle5_lab"], True)
    assert int(r.stdout.strip().splitlines()[-1].split()[1]) == want


REF_COUNTS = os.path.join(GOLD, "ref_gpu_counts.json")


@pytest.mark.skipif(not os.path.exists(REF_COUNTS), reason="reference GPU counts not generated")
def test_gpu_counts_match_reference_gpu_output(ctx):
    """Counts printed by the reference's own `test` binary (built from its
    untouched sources) on the golden graphs."""
    recs = json.load(open(REF_COUNTS))
    assert recs
    for rec in recs:
        labeled = rec["labeled"]
        g = dev_graph(rec["graph"], labeled)
        p = pm.PatternPreprocessor(text=PATTERNS[rec["pattern"]], labeled=labeled)
        got = ctx.match(g, [p], truncate=rec["truncate"])[0][0]
        assert got == rec["count"], rec


def test_gpu_prepared_query_replays(ctx):
    """A batched launch captured in a CUDA graph gives the same counts on
    every replay as the direct call."""
    g = dev_graph("cl3000", True)
    batch = P.batch_of_20(seed=303, n_labels=2)
    plans = [pm.PatternPreprocessor(text=t, labeled=True) for _, t in batch]
    want = ctx.match(g, plans)[0]
    q = ctx.prepare(g, plans)
    for _ in range(3):
        got, st = q.run()
        assert got == want and st["device_status"] == 0
    q.close()
    gu = dev_graph("rmat512", False)
    p = pm.PatternPreprocessor(text=PATTERNS["cycle5"], labeled=False)
    q = ctx.prepare(gu, [p], warps_per_block=16, chunk=3)
    assert q.run()[0] == ctx.match(gu, [p])[0]


def test_gpu_degree_order_keeps_counts(ctx):
    """Renumbering by degree (the reference's relabel step) changes the
    search, not the answer: every count is the same on the GPU and equals
    the oracle's on the original graph."""
    from pumatch_b200 import patterns as P
    cases = {("cl3000", False): [PATTERNS["clique5"], PATTERNS["clique6"], PATTERNS["house"], PATTERNS["cycle5"]],
             ("rmat512", True): [P.to_g(*P.house(), [0, 1, 0, 1, 0]), P.to_g(*P.cycle(5), [0, 0, 1, 1, 0]),
                                 P.to_g(*P.star(5), [1, 0, 0, 1, 2])]}
    for (name, labeled), texts in cases.items():
        hg = host_graph(name, labeled)
        rg, _ = pm.reorder_by_degree(hg)
        g0 = pm.GraphPreprocessor.from_host(hg, labeled=labeled)
        g1 = pm.GraphPreprocessor.from_host(rg, labeled=labeled)
        try:
            for text in texts:
                p = pm.PatternPreprocessor(text=text, labeled=labeled)
                want, _ = oracle_count(hg, text, labeled)
                a, _ = ctx.match(g0, [p])
                b, _ = ctx.match(g1, [p])
                assert a[0] == want and b[0] == want, (name, text)
        finally:
            g0.close()
            g1.close()


def test_gpu_deadline_returns_timeout_and_context_stays_usable(ctx):
    """A launch that runs past its deadline stops on its own (every wait and
    every warp checks the clock), reports PM_ERR_TIMEOUT, and leaves the
    context usable: the next launch gives the full count."""
    from pumatch_b200 import patterns as P
    hg = pm.gen_chung_lu(20000, 200000, gamma=2.1, i0=5.0, max_w=2000.0, seed=7)
    g = pm.GraphPreprocessor.from_host(hg)
    try:
        p = pm.PatternPreprocessor(text=P.to_g(*P.clique(6)), labeled=False)
        full, st = ctx.match(g, [p])
        if st["kernel_ms"] < 20:
            pytest.skip(f"the launch takes {st['kernel_ms']:.1f} ms: too quick to cut short")
        with pytest.raises(pm.PmError) as e:
            ctx.match(g, [p], timeout_ms=1)
        assert e.value.status == pm.PM_ERR_TIMEOUT
        again, st2 = ctx.match(g, [p])
        assert again == full and st2["device_status"] == 0
    finally:
        g.close()
