"""SNAP text -> CSR files, the reference's converter pipeline
(graph_converter/convert.sh: snapToBin, makeLists, compactify, labelize)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import pumatch_b200 as pm

SNAP = """# Directed graph (each unordered pair of nodes is saved once)
# FromNodeId\tToNodeId
100\t7
7\t100
7\t42
42\t42

100 9000
9000\t7
42\t100
"""


def test_convert_ids_lists_and_labels(tmp_path):
    path = str(tmp_path / "snap.txt")
    open(path, "w").write(SNAP)
    n, nadj = pm.convert_snap(path, n_labels=10)
    # first-seen order: 100->0, 7->1, 42->2, 9000->3
    assert n == 4
    hg = pm.HostGraph.read(path, labeled=True)
    lists = [sorted(hg.colidx[hg.rowptr[v]:hg.rowptr[v + 1]].tolist()) for v in range(n)]
    assert lists == [[1, 2, 3], [0, 2, 3], [0, 1], [0, 1]]
    assert nadj == 10 and hg.n_adj == 10
    meta = open(path + ".meta.txt").read().split()
    assert meta == ["4", "10", "4", "3"]
    # labels: rand() % 10 after srand(0), vertex by vertex (glibc)
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(0)
    assert hg.labels.tolist() == [libc.rand() % 10 for _ in range(n)]


def test_convert_keeps_self_loops_on_request(tmp_path):
    path = str(tmp_path / "s.txt")
    open(path, "w").write(SNAP)
    n, nadj = pm.convert_snap(path, n_labels=0, keep_self_loops=True)
    hg = pm.HostGraph.read(path, labeled=False)
    assert hg.colidx[hg.rowptr[2]:hg.rowptr[3]].tolist() == [0, 1, 2]  # 42 lists itself once, in order
    assert not os.path.exists(path + ".label.bin")


def test_convert_cli_and_errors(tmp_path):
    path = str(tmp_path / "c.txt")
    open(path, "w").write("1 2\n2 3\n3 1\n")
    cli = os.path.join(os.path.dirname(pm.CLI_PATH), "convert")
    r = subprocess.run([cli, path, "--labels=4"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    hg = pm.HostGraph.read(path, labeled=True)
    assert hg.n == 3 and hg.n_adj == 6 and hg.labels.max() < 4
    bad = str(tmp_path / "bad.txt")
    open(bad, "w").write("1 x\n")
    r = subprocess.run([cli, bad], capture_output=True, text=True)
    assert r.returncode == 1 and "expected two vertex ids" in r.stderr
    try:
        pm.convert_snap(str(tmp_path / "missing.txt"))
        raise AssertionError("expected an error")
    except pm.PmError as e:
        assert e.status == pm.PM_ERR_IO


GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref")


def _copy_graph(name, dst_prefix, labeled):
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", name), labeled=labeled)
    hg.write(dst_prefix)
    return hg


def test_reorder_keeps_every_count_and_orders_by_degree():
    """Renumbering by degree is a relabelling of the same graph: the oracle's
    counts do not change, labeled or not."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(GOLD), "..", "oracle"))
    import pm_oracle as orc
    from pumatch_b200 import patterns as P
    for name in ("cl400", "rmat512"):
        hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", name), labeled=True)
        rg, nid = pm.reorder_by_degree(hg)
        assert sorted(nid.tolist()) == list(range(hg.n))
        d_old, d_new = hg.degrees(), rg.degrees()
        assert (np.diff(d_new) <= 0).all()  # highest degree first
        assert (d_new[nid] == d_old).all() and (rg.labels[nid] == hg.labels).all()
        for v in range(0, hg.n, 37):  # lists are the same neighbourhoods, renamed and sorted
            got = rg.colidx[rg.rowptr[nid[v]]:rg.rowptr[nid[v] + 1]].tolist()
            assert got == sorted(nid[hg.colidx[hg.rowptr[v]:hg.rowptr[v + 1]]].tolist())
        cases = [(P.to_g(*P.cycle(4)), False), (P.to_g(*P.clique(4)), False), (P.to_g(*P.house()), False),
                 (P.to_g(*P.cycle(5), [0, 1, 0, 1, 2]), True), (P.to_g(*P.star(4), [1, 0, 1, 2]), True)]
        for text, labeled in cases:
            counts = []
            for g in (hg, rg):
                og = orc.Graph(g.rowptr, g.colidx, g.labels if labeled else None)
                p = orc.plan(text, labeled)
                counts.append(orc.count(og, p, orc.roots(og, p), threads=4)[0])
            assert counts[0] == counts[1], (name, text)


def test_halve_keeps_each_edge_once_towards_the_heavier_end():
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", "rmat512"), labeled=False)
    rp, ci, md = pm.halve(hg)
    deg = hg.degrees()
    assert len(ci) * 2 == hg.n_adj
    pairs = set()
    for u in range(hg.n):
        for w in ci[rp[u]:rp[u + 1]].tolist():
            assert deg[w] > deg[u] or (deg[w] == deg[u] and w > u)
            pairs.add((min(u, w), max(u, w)))
    assert len(pairs) == len(ci)
    assert md == int(np.diff(rp).max())


def test_reorder_and_halve_reject_bad_csr():
    bad = pm.HostGraph(np.array([0, 1, 2], dtype=np.uint64), np.array([1, 5], dtype=np.int32))
    for fn in (pm.reorder_by_degree, pm.halve):
        try:
            fn(bad)
            raise AssertionError("expected an error")
        except pm.PmError as e:
            assert e.status == pm.PM_ERR_FORMAT


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "ref_relabel")), reason="reference tools not built")
@pytest.mark.parametrize("name", ["cl400", "rmat512", "dense60"])
def test_cli_order_and_halve_match_the_reference_tools(tmp_path, name):
    """`convert --order=degree` and `convert --halve` write the same vertex and
    edge files as the reference's relabel and halve, built from its sources."""
    cli = os.path.join(os.path.dirname(pm.CLI_PATH), "convert")
    ours, theirs = str(tmp_path / "ours"), str(tmp_path / "theirs")
    _copy_graph(name, ours, labeled=False)
    _copy_graph(name, theirs, labeled=False)
    for flag, tool, suffix in (("--order=degree", "ref_relabel", ".ord"), ("--halve", "ref_halve", ".half")):
        r = subprocess.run([cli, flag, ours], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        r = subprocess.run([os.path.join(REF, tool), theirs], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        for ext in (".vertex.bin", ".edge.bin"):
            a = open(ours + suffix + ext, "rb").read()
            b = open(theirs + suffix + ext, "rb").read()
            assert a == b, (name, flag, ext)
        ma = open(ours + suffix + ".meta.txt").read().split()
        mb = open(theirs + suffix + ".meta.txt").read().split()
        assert [int(x) for x in ma] == [int(x) for x in mb], (name, flag)


def test_cli_transform_errors(tmp_path):
    cli = os.path.join(os.path.dirname(pm.CLI_PATH), "convert")
    r = subprocess.run([cli, "--halve", str(tmp_path / "missing")], capture_output=True, text=True)
    assert r.returncode == 1 and "read" in r.stderr
    r = subprocess.run([cli, "--order=degree"], capture_output=True, text=True)
    assert r.returncode == 2
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 2 and "--order=degree" in r.stderr and "--halve" in r.stderr


def test_cli_order_keeps_labels(tmp_path):
    """`convert --order=degree` on a labeled graph writes the labels in the
    new vertex order."""
    cli = os.path.join(os.path.dirname(pm.CLI_PATH), "convert")
    pre = str(tmp_path / "g")
    hg = _copy_graph("rmat512", pre, labeled=True)
    r = subprocess.run([cli, "--order=degree", pre], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    og = pm.HostGraph.read(pre + ".ord", labeled=True)
    rg, nid = pm.reorder_by_degree(hg)
    assert (og.rowptr == rg.rowptr).all() and (og.colidx == rg.colidx).all() and (og.labels == rg.labels).all()
