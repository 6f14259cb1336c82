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


def test_cost_split_covers_the_prefix_in_order():
    rng = np.random.default_rng(5)
    for n in (0, 1, 5, 100, 1000):
        cost = rng.pareto(1.2, n) if n else []
        for world in (1, 2, 3, 8):
            for frac in (0.0, 0.5, 0.8, 1.0):
                ranges, tail = pmdist.cost_split(cost, world, frac)
                assert len(ranges) == world and 0 <= tail <= n
                assert ranges[0][0] == 0 and ranges[-1][1] == tail
                for (b0, e0), (b1, e1) in zip(ranges, ranges[1:]):
                    assert b0 <= e0 == b1 <= e1
    # balanced: with equal costs the static pieces differ by at most one root
    ranges, tail = pmdist.cost_split([1.0] * 1000, 4, 0.8)
    sizes = [e - b for b, e in ranges]
    assert tail == 800 and max(sizes) - min(sizes) <= 1


def _dyn_worker(rank, world, port, q):
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
        text = P.to_g(*P.house(), [0, 1, 0, 1, 1])
        g = orc.Graph(hg.rowptr, hg.colidx, hg.labels)
        p = orc.plan(text, True)
        roots = orc.roots(g, p)
        # "predicted" cost: a degree product, heavy first, the way the learned
        # order feeds the split
        cost = np.array([float((hg.rowptr[r + 1] - hg.rowptr[r]) * (hg.rowptr[c + 1] - hg.rowptr[c]))
                         for r, c in roots])
        order = np.argsort(-cost, kind="stable")
        ordered = np.ascontiguousarray(np.asarray(roots)[order])
        seen = []

        def run_range(b, e):
            seen.append((b, e))
            c, _ = orc.count(g, p, ordered, b, e)
            return [c]

        store = dist.distributed_c10d._get_default_store()
        mine = pmdist.run_sharded(run_range, 1, len(roots), rank, world, store, "claims-house",
                                  pred_cost=cost[order], static_frac=0.7, tail_chunk=37)
        total = pmdist.reduce_counts(mine)[0]
        full, _ = orc.count(g, p, roots)
        q.put((rank, total, full, seen, len(roots)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_dynamic_tail_counts_sum_to_total(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dyn_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    covered = []
    for rank, total, full, seen, n in out:
        assert total == full
        covered += [i for b, e in seen for i in range(b, e)]
    assert sorted(covered) == list(range(out[0][4]))  # every root position exactly once
