"""Paged residency (adjacency in pinned host memory, capped device frame pool)
against the oracle and the HBM path: counts must stay bit-exact whatever the
frame pool size, page size, cache temperature or eviction pressure."""
import pytest

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import patterns as P

pytestmark = pytest.mark.gpu

_cache = {}


def workload():
    if "w" not in _cache:
        # hubs well above one 4 KiB page (1024 ids) so multi-page lists occur
        hg = pm.gen_chung_lu(8000, 40000, gamma=2.1, i0=3.0, max_w=2500.0, seed=41)
        lab = pm.gen_labels(hg.n, 4, seed=42)
        _cache["w"] = pm.HostGraph(hg.rowptr, hg.colidx, lab)
    return _cache["w"]


TEXTS = {
    "C5_lab": (P.to_g(*P.cycle(5), [0, 1, 2, 3, 1]), True),
    "house_lab": (P.to_g(*P.house(), [1, 2, 0, 3, 2]), True),
    "K4": (P.to_g(*P.clique(4)), False),
    "C4": (P.to_g(*P.cycle(4)), False),
}


def oracle(hg, name):
    if name not in _cache:
        text, labeled = TEXTS[name]
        g = orc.Graph(hg.rowptr, hg.colidx, hg.labels if labeled else None)
        p = orc.plan(text, labeled)
        c, st = orc.count(g, p, orc.roots(g, p), threads=8)
        _cache[name] = (c if labeled else c * p.multiplicity, st)
    return _cache[name]


@pytest.mark.parametrize("page_kb,frames", [(4, 1), (4, 16), (4, 200), (16, 8), (64, 4), (64, 10000)])
def test_paged_counts_exact(ctx, page_kb, frames):
    hg = workload()
    pb = page_kb << 10
    for labeled in (True, False):
        g = pm.GraphPreprocessor.from_host(hg, labeled=labeled, paged=True, page_bytes=pb,
                                           frame_pool_bytes=frames * pb)
        info = g.info()
        assert info["residency"] == pm.PM_RESIDENT_PAGED
        assert info["n_frames"] == min(frames, info["n_pages"])
        for name, (text, lab) in TEXTS.items():
            if lab != labeled:
                continue
            want, ost = oracle(hg, name)
            p = pm.PatternPreprocessor(text=text, labeled=labeled)
            for cold in (True, False):
                got, st = ctx.match(g, [p], cold_cache=cold, timeout_ms=120000)
                assert got[0] == want, (name, page_kb, frames, cold)
                assert st["set_ops"] == ost["set_ops"]
                assert st["device_status"] == 0
                if cold and frames < info["n_pages"]:
                    assert st["page_misses"] > 0
        g.close()


@pytest.mark.parametrize("page_kb,frames,static", [(4, 16, 8), (4, 200, 150), (16, 8, 8), (4, 64, 1), (64, 10000, 10000)])
def test_paged_static_frames_exact(ctx, page_kb, frames, static):
    """Part of the pool placed once and never evicted (the reference's device
    partition): counts stay exact warm and cold, with and without spare frames."""
    hg = workload()
    pb = page_kb << 10
    for labeled in (True, False):
        g = pm.GraphPreprocessor.from_host(hg, labeled=labeled, paged=True, page_bytes=pb,
                                           frame_pool_bytes=frames * pb, static_pool_bytes=static * pb)
        info = g.info()
        assert info["n_static_frames"] == min(static, info["n_frames"])
        for name, (text, lab) in TEXTS.items():
            if lab != labeled:
                continue
            want, ost = oracle(hg, name)
            p = pm.PatternPreprocessor(text=text, labeled=labeled)
            for cold in (True, False, True):
                got, st = ctx.match(g, [p], cold_cache=cold, timeout_ms=120000)
                assert got[0] == want, (name, page_kb, frames, static, cold)
                assert st["set_ops"] == ost["set_ops"]
                assert st["device_status"] == 0
        if info["n_pages"] > 2:
            # learned-style residency: a scattered page set, static part sorted
            pages = list(range(info["n_pages"] - 1, -1, -3))
            g.set_resident_pages(pages)
            assert g.info()["n_static_frames"] == min(static, info["n_frames"], len(pages))
            for name, (text, lab) in TEXTS.items():
                if lab == labeled:
                    got, _ = ctx.match(g, [pm.PatternPreprocessor(text=text, labeled=labeled)])
                    assert got[0] == oracle(hg, name)[0]
        g.close()


@pytest.mark.parametrize("host_copy", [0, 1], ids=["warp-copies", "host-copies"])
def test_paged_pressure_evicts_and_loads(ctx, host_copy):
    """Under eviction pressure, with pages loaded by the missing warps
    themselves (default) or all through the host service thread."""
    hg = workload()
    g = pm.GraphPreprocessor.from_host(hg, labeled=True, paged=True, page_bytes=4096, frame_pool_bytes=32 * 4096)
    text, _ = TEXTS["C5_lab"]
    want, _ = oracle(hg, "C5_lab")
    got, st = ctx.match(g, [pm.PatternPreprocessor(text=text, labeled=True)], cold_cache=True,
                        host_page_copy=host_copy)
    assert got[0] == want
    assert st["pages_loaded"] > 0 and st["evictions"] > 0
    assert st["h2d_page_bytes"] <= st["pages_loaded"] * 4096
    assert st["page_hits"] + st["page_misses"] > 0
    if host_copy:
        assert st["device_page_loads"] == 0
    else:
        assert st["device_page_loads"] > 0
    g.close()


@pytest.mark.parametrize("page_kb,frames", [(4, 16), (64, 4), (16, 8)])
def test_paged_host_copies_exact(ctx, page_kb, frames):
    """Every page load through the host service thread: the same counts."""
    hg = workload()
    pb = page_kb << 10
    for labeled in (True, False):
        g = pm.GraphPreprocessor.from_host(hg, labeled=labeled, paged=True, page_bytes=pb,
                                           frame_pool_bytes=frames * pb)
        for name, (text, lab) in TEXTS.items():
            if lab != labeled:
                continue
            want, ost = oracle(hg, name)
            got, st = ctx.match(g, [pm.PatternPreprocessor(text=text, labeled=labeled)], cold_cache=True,
                                host_page_copy=1, timeout_ms=120000)
            assert got[0] == want and st["set_ops"] == ost["set_ops"], (name, page_kb, frames)
            assert st["device_page_loads"] == 0
        g.close()


def test_paged_full_pool_matches_hbm(ctx):
    hg = workload()
    text, _ = TEXTS["house_lab"]
    p = pm.PatternPreprocessor(text=text, labeled=True)
    gh = pm.GraphPreprocessor.from_host(hg, labeled=True)
    gp = pm.GraphPreprocessor.from_host(hg, labeled=True, paged=True, frame_pool_bytes=1 << 30)
    a, sa = ctx.match(gh, [p])
    b, sb = ctx.match(gp, [p])
    assert a == b and sa["alg_bytes"] == sb["alg_bytes"]
    assert sb["page_misses"] == 0  # everything was prefilled
    # batched patterns over a paged graph
    batch = P.batch_of_20(seed=9, n_labels=4)
    plans = [pm.PatternPreprocessor(text=t, labeled=True) for _, t in batch[:8]]
    assert ctx.match(gh, plans)[0] == ctx.match(gp, plans, cold_cache=True)[0]
