"""Multi-process sharding logic on CPU (gloo, world size 2 and 3): every root
chunk is owned by exactly one rank, and the per-rank oracle counts over the
owned chunks all-reduce to the single-process count."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pumatch_b200 import dist as pmdist


def test_shard_ranges_partition():
    for n in (0, 1, 17, 1000):
        for chunk in (1, 7, 64):
            for world in (1, 2, 3, 8):
                owned = []
                for r in range(world):
                    owned += [i for b, e in pmdist.shard_ranges(n, chunk, r, world) for i in range(b, e)]
                assert sorted(owned) == list(range(n))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import pm_oracle as orc
    import pumatch_b200 as pm
    from pumatch_b200 import patterns as P
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        hg = pm.HostGraph.read(os.path.join(root, "tests", "golden", "graphs", "cl3000"), labeled=True)
        res = []
        for text, labeled in ((P.to_g(*P.cycle(5)), False), (P.to_g(*P.house(), [0, 1, 0, 1, 1]), True)):
            g = orc.Graph(hg.rowptr, hg.colidx, hg.labels if labeled else None)
            p = orc.plan(text, labeled)
            roots = orc.roots(g, p)
            mine = 0
            for b, e in pmdist.shard_ranges(len(roots), 16, rank, world):
                c, _ = orc.count(g, p, roots, b, e)
                mine += c
            mult = 1 if labeled else p.multiplicity
            total = pmdist.reduce_counts([mine * mult])[0]
            full, _ = orc.count(g, p, roots)
            res.append((total, full * mult))
        t = pmdist.max_over_ranks([float(rank)])[0]
        q.put((rank, res, t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_sharded_counts_sum_to_total(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, res, t in out:
        assert t == world - 1
        for total, full in res:
            assert total == full
