"""SNAP text -> CSR files, the reference's converter pipeline
(graph_converter/convert.sh: snapToBin, makeLists, compactify, labelize)."""
import ctypes
import os
import subprocess

import numpy as np

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
