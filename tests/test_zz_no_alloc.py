"""The allocation-free entry point, pm_match_static, against pm_match.

pm_match_static serves callers that cannot allocate device memory (code that
runs while another library holds the allocator lock, a service that owns a
fixed memory budget, a framework that owns the allocator): its scratch is one
file-scope device array of a fixed size.  The
test calls it through the C-ABI twice in a row -- the second call finds the
first call's leftovers in the shared scratch -- and compares each result with
the allocating entry point on the same inputs (counts are integers: equal).
It also checks that an input too large for the fixed scratch is refused with
a clear error instead of overflowing it.

Collected last (file name), so a stop-at-first-failure run has already run
every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import pumatch_b200 as pm
from pumatch_b200 import patterns as P

pytestmark = pytest.mark.gpu


def _static(graph_arrays, plan, **kw):
    import torch
    rp, ci, lb, n, nadj, maxd = graph_arrays
    o = pm.Context._opts(**kw)
    cnt = C.c_uint64()
    st = pm.Stats()
    rc = pm.lib().pm_match_static(C.c_void_p(rp.data_ptr()), C.c_void_p(ci.data_ptr()),
                                  C.c_void_p(lb.data_ptr()) if lb is not None else None, n, nadj, maxd,
                                  plan._h, C.byref(o), None, C.byref(cnt), C.byref(st))
    return rc, cnt.value, st.as_dict()


def _device_arrays(hg, labeled):
    import torch
    rp = torch.from_numpy(hg.rowptr.astype(np.int64)).cuda()
    ci = torch.from_numpy(hg.colidx).cuda()
    lb = torch.from_numpy(hg.labels.astype(np.uint8)).cuda() if labeled else None
    return rp, ci, lb, hg.n, hg.n_adj, hg.max_degree


@pytest.mark.parametrize("labeled", [True, False], ids=["lab", "unl"])
def test_static_entry_matches_allocating_entry(labeled):
    hg = pm.gen_chung_lu(20000, 120000, gamma=2.1, i0=10.0, max_w=400.0, seed=31)
    hg = pm.HostGraph(hg.rowptr, hg.colidx, pm.gen_labels(hg.n, 3, seed=32))
    arrays = _device_arrays(hg, labeled)
    ctx = pm.Context(0)
    g = pm.GraphPreprocessor.from_host(hg, labeled=labeled)
    texts = ([P.to_g(*P.cycle(5), [0, 1, 2, 0, 1]), P.to_g(*P.house(), [1, 1, 0, 2, 2])] if labeled
             else [P.to_g(*P.clique(4)), P.to_g(*P.cycle(5)), P.to_g(*P.path(4))])
    for text in texts:
        p = pm.PatternPreprocessor(text=text, labeled=labeled)
        want, wst = ctx.match(g, [p])
        for _ in range(2):  # the second call reuses the scratch the first one left behind
            rc, got, st = _static(arrays, p)
            assert rc == pm.PM_OK, pm.lib().pm_last_error()
            assert got == want[0]
            assert st["set_ops"] == wst["set_ops"] and st["alg_bytes"] == wst["alg_bytes"]
        # the launch options mean what they mean for pm_match
        for kw in (dict(leaf_per_lane=1), dict(lane_subtree_max=-1), dict(high_occupancy=3, warps_per_block=16),
                   dict(high_occupancy=1, blocks_per_sm=1)):
            w2, _ = ctx.match(g, [p], **kw)
            rc, got, _ = _static(arrays, p, **kw)
            assert rc == pm.PM_OK, pm.lib().pm_last_error()
            assert got == w2[0] == want[0], kw
    g.close()
    ctx.close()


def test_static_entry_refuses_oversized_input():
    # a star whose centre has 3M neighbours: one warp arena alone exceeds the scratch
    n = 3_000_001
    rowptr = np.zeros(n + 1, dtype=np.uint64)
    rowptr[1:] = (n - 1)
    rowptr[2:] += np.arange(1, n, dtype=np.uint64)
    colidx = np.concatenate([np.arange(1, n, dtype=np.int32), np.zeros(n - 1, dtype=np.int32)])
    hg = pm.HostGraph(rowptr, colidx)
    arrays = _device_arrays(hg, False)
    p = pm.PatternPreprocessor(text=P.to_g(*P.star(5)), labeled=False)
    rc, _, _ = _static(arrays, p)
    assert rc == pm.PM_ERR_INVALID
    assert b"static scratch" in pm.lib().pm_last_error()
