"""File layout (reference src/graph.h:228-254) and the seeded generators."""
import os

import numpy as np
import pytest

import pumatch_b200 as pm

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def check_csr(hg, n, m):
    assert hg.n == n and hg.n_adj == 2 * m
    rp, ci = hg.rowptr.astype(np.int64), hg.colidx
    assert rp[0] == 0 and rp[-1] == len(ci) and np.all(np.diff(rp) >= 0)
    src = np.repeat(np.arange(n), np.diff(rp))
    assert np.all(ci >= 0) and np.all(ci < n)
    assert not np.any(src == ci), "self-loop"
    for v in range(0, n, max(1, n // 200)):
        lst = ci[rp[v]:rp[v + 1]]
        assert np.all(np.diff(lst) > 0), "unsorted or duplicate"
    # symmetric: the multiset of (u, v) equals that of (v, u)
    a = np.sort(src.astype(np.int64) * n + ci)
    b = np.sort(ci.astype(np.int64) * n + src)
    assert np.array_equal(a, b)


def test_chung_lu_exact_and_deterministic():
    a = pm.gen_chung_lu(5000, 30000, gamma=2.1, i0=10, max_w=500, seed=7)
    b = pm.gen_chung_lu(5000, 30000, gamma=2.1, i0=10, max_w=500, seed=7)
    c = pm.gen_chung_lu(5000, 30000, gamma=2.1, i0=10, max_w=500, seed=8)
    check_csr(a, 5000, 30000)
    assert np.array_equal(a.colidx, b.colidx) and np.array_equal(a.rowptr, b.rowptr)
    assert not np.array_equal(a.colidx, c.colidx)
    deg = a.degrees()
    assert deg[:10].mean() > 5 * deg.mean()  # power law: low ids are hubs


def test_rmat_exact_and_deterministic():
    a = pm.gen_rmat(3000, 20000, seed=2)
    b = pm.gen_rmat(3000, 20000, seed=2)
    check_csr(a, 3000, 20000)
    assert np.array_equal(a.colidx, b.colidx)
    assert a.max_degree > 10 * (2 * 20000 / 3000)


def test_labels_uniform():
    lab = pm.gen_labels(80000, 8, seed=102)
    assert lab.min() == 0 and lab.max() == 7
    counts = np.bincount(lab)
    assert counts.min() > 0.9 * counts.mean()
    assert np.array_equal(lab, pm.gen_labels(80000, 8, seed=102))


def test_write_read_roundtrip(tmp_path):
    hg = pm.gen_chung_lu(1000, 4000, seed=3)
    lab = pm.gen_labels(1000, 5, seed=4)
    pre = str(tmp_path / "g")
    pm.HostGraph(hg.rowptr, hg.colidx, lab).write(pre)
    meta = open(pre + ".meta.txt").read().split()
    assert meta == ["1000", str(hg.n_adj), "4", str(hg.max_degree)]
    assert os.path.getsize(pre + ".vertex.bin") == 8 * 1001
    assert os.path.getsize(pre + ".edge.bin") == 4 * hg.n_adj
    assert os.path.getsize(pre + ".label.bin") == 4 * 1000
    back = pm.HostGraph.read(pre, labeled=True)
    assert np.array_equal(back.rowptr, hg.rowptr) and np.array_equal(back.colidx, hg.colidx)
    assert np.array_equal(back.labels, lab)
    unl = pm.HostGraph.read(pre, labeled=False)
    assert unl.labels is None


def test_read_errors(tmp_path):
    with pytest.raises(pm.PmError) as e:
        pm.HostGraph.read(str(tmp_path / "missing"), labeled=False)
    assert e.value.status == pm.PM_ERR_IO
    pre = str(tmp_path / "bad")
    open(pre + ".meta.txt", "w").write("10\n20\n8\n3\n")  # vid_size 8 unsupported
    with pytest.raises(pm.PmError) as e:
        pm.HostGraph.read(pre, labeled=False)
    assert e.value.status == pm.PM_ERR_FORMAT
    hg = pm.gen_chung_lu(50, 100, seed=1)
    pm.HostGraph(hg.rowptr, hg.colidx).write(pre)
    ci = hg.colidx.copy()
    ci[0], ci[1] = ci[1], ci[0]  # unsort one list
    ci.tofile(pre + ".edge.bin")
    with pytest.raises(pm.PmError) as e:
        pm.HostGraph.read(pre, labeled=False)
    assert e.value.status == pm.PM_ERR_FORMAT
    with open(pre + ".edge.bin", "wb") as f:
        f.write(b"\0" * 8)  # truncated file
    with pytest.raises(pm.PmError):
        pm.HostGraph.read(pre, labeled=False)


def test_golden_graphs_load():
    for name in ("cl400", "rmat512", "dense60", "cl3000"):
        hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", name), labeled=True)
        assert hg.labels is not None and hg.labels.max() < 32
