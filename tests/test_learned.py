"""The learned scheduler: hand-written MLP kernels against the float64 CPU
reference (oracle/mlp_ref.py), training that beats a constant predictor, and
learned root order / page residency that leave every count unchanged."""
import numpy as np
import pytest

import mlp_ref

gpu = pytest.mark.gpu


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    w = rng.normal(0, 0.3, mlp_ref.NPARAM).astype(np.float32)
    w = mlp_ref.to_bf16(w)  # keep parameters on the bf16 grid
    x = rng.normal(0, 1, (12, 16))
    t = rng.normal(0, 1, (12, 2))
    loss, g = mlp_ref.loss_and_grad(w, x, t)

    # finite differences on the unrounded float64 function
    def f(flat):
        p = mlp_ref.unpack(flat)
        h1 = np.maximum(x @ p["W1"] + p["b1"], 0)
        h2 = np.maximum(h1 @ p["W2"] + p["b2"], 0)
        return float((((h2 @ p["W3"] + p["b3"]) - t) ** 2).mean())
    for i in rng.choice(mlp_ref.NPARAM, 40, replace=False):
        e = np.zeros(mlp_ref.NPARAM)
        e[i] = 1e-6
        fd = (f(w + e) - f(w - e)) / 2e-6
        assert abs(fd - g[i]) < 1e-5 + 1e-4 * abs(fd)
    assert abs(loss - f(w)) < 1e-12


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.001953125, -3.14159, 65504.0], dtype=np.float32)
    r = mlp_ref.to_bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0078125 or r[1] == 1.0  # ties to even
    assert abs(r[3] + 3.140625) < 1e-9
    import torch
    assert np.allclose(r, torch.tensor(v).to(torch.bfloat16).float().numpy())


def test_page_scores():
    from pumatch_b200 import learn
    rowptr = np.array([0, 3, 10, 12], dtype=np.uint64)
    roots = np.array([[0, 1], [2, 1]], dtype=np.int32)
    s = learn.page_scores(rowptr, roots, np.array([1.0, 2.0]), page_ints=4, n_pages=3)
    # root 0: v0 list [0,3) -> page 0 (twice), v1 list [3,10) -> pages 0 and 2
    # root 1: v0 list [10,12) -> page 2 (twice), v1 -> pages 0 and 2
    assert s.tolist() == [1 + 1 + 1 + 2, 0, 1 + 2 + 2 + 2]


@gpu
def test_gpu_mlp_forward_and_gradient_match_reference():
    import torch

    from pumatch_b200 import learn
    m = learn.CostModel(0, seed=3)
    w = m.weights()
    rng = np.random.default_rng(1)
    x = rng.normal(0, 1, (1000, 16)).astype(np.float32)
    t = rng.normal(0, 1, (1000, 2)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    td = torch.from_numpy(t).cuda()
    y = m.forward_raw(xd).cpu().numpy()
    yr = mlp_ref.forward(w, x)
    assert np.allclose(y, yr, rtol=1e-4, atol=1e-4)
    loss, g = m.gradient(xd, td)
    lr, gr = mlp_ref.loss_and_grad(w, x, t)
    assert abs(loss - lr) < 1e-4 * max(1.0, abs(lr))
    # FP32 accumulation vs FP64: relative tolerance on the gradient vector
    assert np.linalg.norm(g - gr) <= 1e-4 * np.linalg.norm(gr) + 1e-7
    m.close()


@gpu
def test_gpu_training_beats_constant_predictor():
    import torch

    from pumatch_b200 import learn
    rng = np.random.default_rng(2)
    x = rng.normal(0, 1, (20000, 16)).astype(np.float32)
    wt = rng.normal(0, 1, (16, 2))
    t = (np.tanh(x @ wt) + 0.5 * (x[:, :2] ** 2)).astype(np.float32)
    m = learn.CostModel(0, seed=5)
    xd = torch.from_numpy(x).cuda()
    td = torch.from_numpy(t).cuda()
    hist = m.fit(xd, td, epochs=15, batch=1024, lr=3e-3)
    assert hist[-1] < 0.5 * hist[0]
    pred = m.predict(xd).cpu().numpy()
    mse = ((pred - t) ** 2).mean()
    base = ((t - t.mean(0)) ** 2).mean()
    assert mse < 0.2 * base
    m.close()


@gpu
def test_gpu_learned_order_and_residency_keep_counts(ctx):
    import os

    import torch

    import pumatch_b200 as pm
    from pumatch_b200 import learn
    from pumatch_b200 import patterns as P
    hg = pm.gen_rmat(1 << 14, 12 << 14, seed=11)
    lab = pm.gen_labels(hg.n, 4, seed=12)
    hgl = pm.HostGraph(hg.rowptr, hg.colidx, lab)
    g = pm.GraphPreprocessor.from_host(hgl, labeled=True)
    p = pm.PatternPreprocessor(text=P.to_g(*P.house(), [0, 1, 2, 1, 3]), labeled=True)
    count, st, cost, reads = learn.plain_costs(ctx, g, p)
    x = learn.root_features(ctx, g, p)
    assert x.shape == (st["n_roots"], 16) and torch.isfinite(x).all()
    t = learn.targets(cost, reads)
    m = learn.CostModel(0, seed=1)
    hist = m.fit(x, t, epochs=20, batch=2048)
    pred = m.predict(x)
    err = (pred - t).abs().mean().item()
    base = (t - t.mean(0)).abs().mean().item()
    assert err < base, (err, base)  # the model explains part of the cost
    order = learn.heavy_first_order(pred)
    assert sorted(order.cpu().tolist()) == list(range(st["n_roots"]))
    c2, st2 = ctx.match(g, [p], root_order_ptr=order.data_ptr())
    assert c2[0] == count and st2["set_ops"] == st["set_ops"]
    # paged graph with learned residency
    gp = pm.GraphPreprocessor.from_host(hgl, labeled=True, paged=True, page_bytes=4096,
                                        frame_pool_bytes=16 * 4096)
    info = gp.info()
    roots = ctx.roots(gp, p)
    score = learn.page_scores(hgl.rowptr, roots, np.expm1(pred[:, 1].clamp_min(0).cpu().numpy()), 1024,
                              info["n_pages"])
    gp.set_resident_pages(np.argsort(-score)[:info["n_frames"]])
    c3, st3 = ctx.match(gp, [p], root_order_ptr=order.data_ptr())
    assert c3[0] == count
    m.close()


@gpu
def test_gpu_learned_scheduling_keeps_counts_and_predicts_cost(ctx):
    """The learned scheduler end to end on a fixed seed: a paged R-MAT graph
    whose frame pool holds half of the adjacency, all under CLOCK.  The
    model, trained on three other seeds, predicts the held-out seed's
    per-root log cost and page touches better than a constant predictor;
    the plain run (cold pool, reference order), predicted residency with
    heavy-first order, and the full learned run (plus prefetch lists and
    per-root split thresholds) all return the same count.  Whether the
    learned runs are faster is measured by the bench (`learned_vs_plain`):
    on this small graph the misses and times of single runs vary with the
    warps' races by more than the learned choices change them, so no gain
    is asserted here."""

    import torch

    import pumatch_b200 as pm
    from pumatch_b200 import learn
    from pumatch_b200 import patterns as P
    text = P.to_g(*P.cycle_tail(5, 2), P.seeded_labels(7, 32, 202))

    def graph(seed):
        hg = pm.gen_rmat(1 << 15, 16 << 15, seed=seed)
        return pm.HostGraph(hg.rowptr, hg.colidx, pm.gen_labels(hg.n, 32, seed=102 + 1000 * seed))

    xs, ts = [], []
    for seed in (11, 12, 13):
        gs = pm.GraphPreprocessor.from_host(graph(seed), labeled=True)
        ps = pm.PatternPreprocessor(text=text, labeled=True)
        _, _, cost, reads = learn.plain_costs(ctx, gs, ps)
        xs.append(learn.root_features(ctx, gs, ps))
        ts.append(learn.targets(cost, reads))
        gs.close()
    x, t = torch.cat(xs), torch.cat(ts)
    m = learn.CostModel(0, seed=1)
    m.fit(x, t, epochs=20, batch=4096)
    hg = graph(2)
    pb = 16 << 10
    g = pm.GraphPreprocessor.from_host(hg, labeled=True, paged=True, page_bytes=pb,
                                       frame_pool_bytes=max(pb, hg.colidx.nbytes // 2 // pb * pb))
    p = pm.PatternPreprocessor(text=text, labeled=True)
    pred = m.predict(learn.root_features(ctx, g, p))
    # the prediction beats a constant one on the held-out seed
    hb = pm.GraphPreprocessor.from_host(hg, labeled=True)
    count, _, cost, reads = learn.plain_costs(ctx, hb, p)
    hb.close()
    te = learn.targets(cost, reads)
    assert (pred - te).abs().mean().item() < (te - t.mean(0)).abs().mean().item()
    info = g.info()
    roots = ctx.roots(g, p)
    pred_reads = torch.expm1(pred[:, 1].clamp_min(0)).cpu().numpy()
    order = learn.heavy_first_order(pred)
    score = learn.page_scores(hg.rowptr, roots, pred_reads, pb // 4, info["n_pages"])
    off, pages = learn.prefetch_lists(hg.rowptr, hg.colidx, roots, order.cpu().numpy(), pred_reads, pb // 4, 16)
    split = learn.split_thresholds(pred)
    off_d = torch.from_numpy(off).cuda()
    pages_d = torch.from_numpy(pages if len(pages) else np.zeros(1, dtype=np.int32)).cuda()
    res = {}
    for mode in ("plain", "learned_residency_order", "learned"):
        if mode == "plain":
            g.set_resident_pages(np.zeros(0, dtype=np.int64))
            kw = dict(cold_cache=1)
        else:
            g.set_resident_pages(np.argsort(-score)[:info["n_frames"]])
            kw = dict(root_order_ptr=order.data_ptr())
            if mode == "learned":
                kw.update(prefetch_off_ptr=off_d.data_ptr(), prefetch_pages_ptr=pages_d.data_ptr(),
                          prefetch_chunks=len(off) - 1, root_split_ptr=split.data_ptr())
        ms, misses = [], []
        for _ in range(3):
            c, st = ctx.match(g, [p], chunk=16, **kw)
            assert c[0] == count, mode
            ms.append(st["kernel_ms"])
            misses.append(st["page_misses"])
        res[mode] = (min(ms), min(misses))
    assert all(v[1] > 0 for v in res.values()), res  # the pool is half the adjacency: every arm misses
    g.close()
    m.close()
