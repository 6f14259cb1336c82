"""The batched launch's autotuner: its sweep always contains the library's
default configuration (so the tuned configuration is never slower than the
untuned one), covers the kernel variants, and every configuration returns
the same counts (checked against the oracle here)."""
import os

import pytest

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import autotune
from pumatch_b200 import patterns as P

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_sweep_contains_default_and_keeps_counts(ctx, tmp_path):
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", "cl3000"), labeled=True)
    texts = [P.to_g(*P.cycle(4), [0, 1, 0, 1]), P.to_g(*P.house(), [1, 1, 0, 2, 2]), P.to_g(*P.clique(4))]
    og = orc.Graph(hg.rowptr, hg.colidx, hg.labels)
    want = []
    for t in texts:
        p = orc.plan(t, True)
        want.append(orc.count(og, p, orc.roots(og, p))[0])
    g = pm.GraphPreprocessor.from_host(hg, labeled=True)
    plans = [pm.PatternPreprocessor(text=t, labeled=True) for t in texts]
    try:
        rows = autotune.sweep(ctx, g, plans, warps=(4, 8, 16), chunks=(16, 256), splits=(64,), timeout_ms=60000)
        assert rows[0].get("default") and rows[0]["kernel_ms"] is not None
        assert {r["high_occupancy"] for r in rows[1:]} == set(autotune.VARIANTS)
        assert all(r["warps_per_block"] <= 8 or r["high_occupancy"] == 3 for r in rows)
        done = [r for r in rows if r["kernel_ms"] is not None]
        best = min(done, key=lambda r: r["kernel_ms"])
        assert best["kernel_ms"] <= rows[0]["kernel_ms"]
        counts, _ = ctx.match(g, plans, **{k: best[k] for k in ("warps_per_block", "chunk", "split_level1",
                                                                  "high_occupancy")})
        assert counts == want
        # paged: page sizes are part of the search
        out = autotune.autotune(ctx, hg, plans, labeled=True, paged=True, frame_pool_bytes=1 << 20,
                                page_kb=(16, 64), warps=(8,), chunks=(16,), splits=(64,), variants=(2,),
                                out_json=str(tmp_path / "tuned.json"))
        assert {r["page_kb"] for r in out["results"]} == {16, 64}
        assert os.path.exists(tmp_path / "tuned.json")
    finally:
        g.close()
