"""Learned scheduler: a per-root cost model driving root order and page residency.

The model (pm_mlp_*, hand-written CUDA in csrc/pm_learn.cu) maps 16 features of
a root edge to [log(1 + DFS bytes), log(1 + adjacency reads)] of its subtree.
It is trained on what the plain method logs about itself (per-root cost and
reads from an ordinary run) and then used three ways, none of which can
change a count:
  * root binning: roots are processed heaviest-first (longest-processing-time
    order), so the tail of a launch is made of cheap roots;
  * page residency (paged graphs): pages are scored by the predicted reads of
    the roots whose first two vertices' lists live in them, and the frame pool
    starts with the highest-scoring pages instead of starting cold;
  * prefetch during the run (paged graphs): each root chunk gets a list of the
    pages its predicted-heaviest roots will read first, which the kernel posts
    to the copy ring a few chunks ahead (prefetch_lists).
The plain path is the fallback (no model) and the baseline that prediction
error and speed are measured against.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Tuple

import numpy as np

from . import Context, GraphPreprocessor, PatternPreprocessor, _check, lib

NIN, NOUT = 16, 2
NPARAM = 16 * 64 + 64 + 64 * 64 + 64 + 64 * 2 + 2


def root_features(ctx: Context, g: GraphPreprocessor, p: PatternPreprocessor):
    """(n_roots, 16) float32 device tensor of root features, in root order."""
    import torch
    n = C.c_int64()
    _check(lib().pm_root_features(ctx._h, g._h, p._h, None, 0, C.byref(n)))
    x = torch.zeros((max(n.value, 1), NIN), dtype=torch.float32, device=f"cuda:{ctx.device}")
    _check(lib().pm_root_features(ctx._h, g._h, p._h, C.c_void_p(x.data_ptr()), x.shape[0], C.byref(n)))
    return x[: n.value]


def plain_costs(ctx: Context, g: GraphPreprocessor, p: PatternPreprocessor, **kw):
    """Runs the plain method once, logging per-root bytes and reads.
    Returns (count, stats, cost_bytes tensor, reads tensor)."""
    import torch
    n = ctx.count_roots(g, p)
    dev = f"cuda:{ctx.device}"
    cost = torch.zeros(max(n, 1), dtype=torch.float32, device=dev)
    reads = torch.zeros(max(n, 1), dtype=torch.float32, device=dev)
    counts, st = ctx.match(g, [p], root_cost_ptr=cost.data_ptr(), root_reads_ptr=reads.data_ptr(), **kw)
    return counts[0], st, cost[:n], reads[:n]


def targets(cost, reads):
    import torch
    return torch.stack([torch.log1p(cost), torch.log1p(reads)], dim=1).contiguous()


class CostModel:
    """pm_mlp handle: BF16 weights, FP32 master copy, Adam."""

    def __init__(self, device: int = 0, seed: int = 1):
        h = C.c_void_p()
        _check(lib().pm_mlp_create(device, seed, C.byref(h)))
        self._h = h
        self.device = device
        self.mu = np.zeros(NIN, dtype=np.float32)
        self.sd = np.ones(NIN, dtype=np.float32)
        # targets are fitted standardised (log costs sit near 15 while the
        # output layer starts near 0), and predictions scaled back
        self.tmu = np.zeros(NOUT, dtype=np.float32)
        self.tsd = np.ones(NOUT, dtype=np.float32)

    def close(self):
        if self._h:
            lib().pm_mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self) -> np.ndarray:
        w = np.zeros(NPARAM, dtype=np.float32)
        _check(lib().pm_mlp_get_weights(self._h, w.ctypes.data_as(C.c_void_p)))
        return w

    def set_weights(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().pm_mlp_set_weights(self._h, w.ctypes.data_as(C.c_void_p)))

    def gradient(self, x, t) -> Tuple[float, np.ndarray]:
        g = np.zeros(NPARAM, dtype=np.float32)
        loss = C.c_float()
        _check(lib().pm_mlp_gradient(self._h, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()), x.shape[0],
                                     g.ctypes.data_as(C.c_void_p), C.byref(loss)))
        return loss.value, g

    def forward_raw(self, x):
        import torch
        y = torch.zeros((x.shape[0], NOUT), dtype=torch.float32, device=x.device)
        _check(lib().pm_mlp_forward(self._h, C.c_void_p(x.data_ptr()), x.shape[0], C.c_void_p(y.data_ptr())))
        return y

    def normalise(self, x):
        import torch
        mu = torch.as_tensor(self.mu, device=x.device)
        sd = torch.as_tensor(self.sd, device=x.device)
        return ((x - mu) / sd).contiguous()

    def fit(self, x, t, epochs: int = 30, batch: int = 8192, lr: float = 3e-3, seed: int = 0) -> list:
        """Adam on minibatches of (x, t); returns the per-epoch mean loss."""
        import torch
        xs = x.double()
        self.mu = xs.mean(0).float().cpu().numpy()
        self.sd = (xs.std(0).float().clamp_min(1e-3)).cpu().numpy()
        xn = self.normalise(x)
        ts = t.double()
        self.tmu = ts.mean(0).float().cpu().numpy()
        self.tsd = (ts.std(0).float().clamp_min(1e-3)).cpu().numpy()
        t = ((t - torch.as_tensor(self.tmu, device=t.device)) / torch.as_tensor(self.tsd, device=t.device))
        t = t.float().contiguous()
        gen = torch.Generator(device="cpu").manual_seed(seed)
        hist = []
        n = xn.shape[0]
        for _ in range(epochs):
            perm = torch.randperm(n, generator=gen).to(xn.device)
            tot, k = 0.0, 0
            for b in range(0, n, batch):
                idx = perm[b:b + batch]
                xb = xn[idx].contiguous()
                tb = t[idx].contiguous()
                loss = C.c_float()
                _check(lib().pm_mlp_train_step(self._h, C.c_void_p(xb.data_ptr()), C.c_void_p(tb.data_ptr()),
                                               xb.shape[0], lr, C.byref(loss)))
                tot += loss.value
                k += 1
            hist.append(tot / max(k, 1))
        return hist

    def predict(self, x):
        import torch
        y = self.forward_raw(self.normalise(x))
        return y * torch.as_tensor(self.tsd, device=y.device) + torch.as_tensor(self.tmu, device=y.device)


def heavy_first_order(pred):
    """Root order for the kernel (int32 device tensor): predicted cost, descending."""
    import torch
    return torch.argsort(pred[:, 0], descending=True).to(torch.int32).contiguous()


def split_thresholds(pred, base: int = 64, heavy_q: float = 0.9, light_q: float = 0.5):
    """Per-root donation thresholds (int32 device tensor, root order) from the
    predicted log cost: roots above the heavy quantile hand out their
    last-but-one-level ranges from base/4 candidates on, roots below the light
    quantile only from 2*base, the rest from base."""
    import torch
    c = pred[:, 0]
    hi, lo = torch.quantile(c, heavy_q), torch.quantile(c, light_q)
    out = torch.full_like(c, float(base))
    out[c >= hi] = max(2, base // 4)
    out[c < lo] = 2 * base
    return out.to(torch.int32).contiguous()


def page_scores(rowptr: np.ndarray, roots: np.ndarray, pred_reads: np.ndarray, page_ints: int, n_pages: int):
    """Predicted demand per adjacency page: each root adds its predicted reads
    to the pages holding its two vertices' lists."""
    score = np.zeros(n_pages, dtype=np.float64)
    for col in (0, 1):
        v = roots[:, col].astype(np.int64)
        first = (rowptr[v] // page_ints).astype(np.int64)
        last = (np.maximum(rowptr[v + 1], rowptr[v] + 1) - 1) // page_ints
        np.add.at(score, first, pred_reads)
        np.add.at(score, last.astype(np.int64), pred_reads)
    return score


def prefetch_lists(rowptr: np.ndarray, colidx: np.ndarray, roots: np.ndarray, order: np.ndarray,
                   pred_reads: np.ndarray, page_ints: int, chunk: int, per_chunk: int = 64,
                   cand_filter=None) -> Tuple[np.ndarray, np.ndarray]:
    """Pages to request ahead of each root chunk (the kernel posts chunk c's
    list when a warp claims chunk c - prefetch_ahead), as CSR (off, pages).

    Roots are taken in processing order (`order`, root ids), `chunk` per
    chunk.  Within a chunk, roots are ranked by their predicted page touches
    (`pred_reads`, per root id); each adds the pages of its two vertices'
    lists, then the pages of the lists of its level-1 candidates (v1's
    neighbours passing `cand_filter(v1, neighbours)`, default all), until the
    chunk holds per_chunk distinct pages.  Chunks whose roots are predicted to
    touch nothing get none."""
    n_chunks = (len(order) + chunk - 1) // chunk
    off = np.zeros(n_chunks + 1, dtype=np.int32)
    pages = []

    def list_pages(v):
        b, e = int(rowptr[v]), int(rowptr[v + 1])
        if e <= b:
            return range(0)
        return range(b // page_ints, (e - 1) // page_ints + 1)

    for k in range(n_chunks):
        ids = order[k * chunk:(k + 1) * chunk]
        ranked = ids[np.argsort(-pred_reads[ids], kind="stable")]
        got = []
        seen = set()

        def add(rng):
            for pg in rng:
                if pg not in seen:
                    seen.add(pg)
                    got.append(pg)
                    if len(got) >= per_chunk:
                        return True
            return False

        full = False
        for r in ranked:
            if pred_reads[r] <= 0:
                break
            v0, v1 = int(roots[r, 0]), int(roots[r, 1])
            if add(list_pages(v0)) or add(list_pages(v1)):
                full = True
                break
        if not full:
            for r in ranked:
                if pred_reads[r] <= 0:
                    break
                v1 = int(roots[r, 1])
                nb = colidx[int(rowptr[v1]):int(rowptr[v1 + 1])]
                if cand_filter is not None:
                    nb = cand_filter(v1, nb)
                for u in nb[:per_chunk]:
                    if add(list_pages(int(u))):
                        full = True
                        break
                if full:
                    break
        pages.extend(got)
        off[k + 1] = len(pages)
    return off, np.asarray(pages, dtype=np.int32)
