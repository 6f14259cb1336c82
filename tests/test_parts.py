"""Partitioned residency, host side (no GPU): slice bounds, the label-grouped
layout the slices hold for labeled graphs, the owner root ranges, and the
file-descriptor exchange between the ranks of a one-process-per-GPU job
(gloo ranks on CPU, memfd descriptors standing in for exported slices)."""
import datetime
import os
import socket
import uuid

import numpy as np
import pytest
import torch.multiprocessing as mp

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import parts
from pumatch_b200 import patterns as P

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("nbytes", [0, 1, 4095, 2 << 20, (2 << 20) + 4, 17 << 20, 100 << 20])
@pytest.mark.parametrize("n_parts", [1, 2, 3, 8])
@pytest.mark.parametrize("page", [4096, 64 << 10, 4 << 20])
def test_slice_bounds_cover_and_align(nbytes, n_parts, page):
    gran = 2 << 20
    begins, total = parts.slice_bounds(nbytes, n_parts, gran, page)
    align = max(gran, page)
    assert begins[0] == 0 and 1 <= len(begins) <= n_parts
    assert total >= max(nbytes, 1) and total % align == 0 and total - nbytes < align + 1
    ends = begins[1:] + [total]
    for b, e in zip(begins, ends):
        assert b % align == 0 and e > b
    sizes = [e - b for b, e in zip(begins, ends)]
    assert all(s == sizes[0] for s in sizes[:-1]) and sizes[-1] <= sizes[0]


def test_slice_bounds_rejects_bad_sizes():
    with pytest.raises(ValueError):
        parts.slice_bounds(10, 0, 2 << 20, 4096)
    with pytest.raises(ValueError):
        parts.slice_bounds(10, 2, 3 << 20, 4096)


@pytest.mark.parametrize("name", ["cl400", "rmat512", "dense60"])
def test_label_grouped_layout(name):
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", name), labeled=True)
    got = parts.label_grouped(hg)
    for v in range(hg.n):
        b, e = int(hg.rowptr[v]), int(hg.rowptr[v + 1])
        lst = hg.colidx[b:e]
        want = lst[np.argsort(hg.labels[lst], kind="stable")]
        assert np.array_equal(got[b:e], want), v


def test_label_grouped_rejects_bad_input():
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", "cl400"), labeled=True)
    bad = pm.HostGraph(hg.rowptr, hg.colidx, np.full(hg.n, 40, dtype=np.uint32))
    with pytest.raises(pm.PmError):
        parts.label_grouped(bad)
    with pytest.raises(ValueError):
        parts.label_grouped(pm.HostGraph(hg.rowptr, hg.colidx))


def test_owner_root_ranges_follow_the_slices():
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", "cl3000"), labeled=False)
    p = orc.plan(P.to_g(*P.cycle(4)), False)
    roots = orc.roots(orc.Graph(hg.rowptr, hg.colidx, None), p)
    nbytes = 4 * hg.n_adj
    for k in (1, 2, 3, 5):
        unit = 4096
        begins, total = parts.slice_bounds(nbytes, k, unit, unit)
        rng = parts.owner_root_ranges(hg.rowptr, roots, begins, total)
        assert len(rng) == len(begins) and rng[0][0] == 0 and rng[-1][1] == len(roots)
        ends = begins[1:] + [total]
        for (b, e), lo, hi in zip(rng, begins, ends):
            assert b <= e
            for i in range(b, e):
                s = 4 * int(hg.rowptr[roots[i, 0]])
                assert lo <= s < hi
        assert all(rng[i][1] == rng[i + 1][0] for i in range(len(rng) - 1))


def _fd_worker(rank, world, port, job, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from pumatch_b200 import parts as pp
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = {}
        for a in range(2):  # two arrays, as a labeled graph has
            if rank == world - 1 and world > 2:
                break  # a rank without a slice (an array too small for every rank) sends none
            fd = os.memfd_create(f"slice{a}-{rank}")
            os.write(fd, f"array {a} slice {rank}".encode())
            mine[a * world + rank] = fd
        dist.barrier()
        theirs = pp.exchange_fds(job, rank, world, mine, timeout_s=30)
        seen = {}
        for key, fd in theirs.items():
            seen[key] = os.pread(fd, 64, 0).decode()
            os.close(fd)
        for fd in mine.values():
            os.close(fd)
        dist.barrier()
        q.put((rank, seen))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_exchange_slice_descriptors(world):
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    job = uuid.uuid4().hex[:12]
    port = _free_port()
    procs = [ctx.Process(target=_fd_worker, args=(r, world, port, job, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get() for _ in range(world))
    for r in range(world):
        owners = [s for s in range(world) if not (s == world - 1 and world > 2)]
        want = {a * world + s: f"array {a} slice {s}" for a in range(2) for s in owners if s != r}
        assert got[r] == want


def test_single_rank_exchange_is_empty():
    assert parts.exchange_fds("solo", 0, 1, {0: 5}) == {}


class _FakeRange:
    """Stands in for a device range on CPU: a slice allocated here is a memfd,
    exported as a duplicate descriptor; an imported slice keeps the peer's
    descriptor.  Reading a slice reads what its owner wrote."""
    log = None

    def __init__(self, device, begins, total):
        self.begins, self.total = list(begins), total
        self.fds = {}
        self.mapped = False

    def bounds(self, p):
        return self.begins[p], self.begins[p + 1] if p + 1 < len(self.begins) else self.total

    def alloc(self, p, owner_device):
        b, e = self.bounds(p)
        fd = os.memfd_create(f"slice{p}")
        os.ftruncate(fd, e - b)
        self.fds[p] = fd

    def export(self, p):
        return os.dup(self.fds[p])

    def import_(self, p, fd):
        self.fds[p] = os.dup(fd)

    def map(self):
        assert sorted(self.fds) == list(range(len(self.begins))), "a slice has no memory"
        self.mapped = True

    @property
    def ptr(self):
        return id(self)

    def fill_slice(self, p, array):
        assert self.mapped
        b, e = self.bounds(p)
        raw = array.view(np.uint8)
        os.pwrite(self.fds[p], raw[b:min(e, raw.nbytes)].tobytes(), 0)

    def read_all(self, nbytes):
        out = bytearray()
        for p in range(len(self.begins)):
            b, e = self.bounds(p)
            out += os.pread(self.fds[p], e - b, 0)
        return bytes(out[:nbytes])

    def close(self):
        for fd in self.fds.values():
            os.close(fd)
        self.fds = {}


def _place_worker(rank, world, port, job, labeled, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import pumatch_b200 as pmm
    from pumatch_b200 import parts as pp
    import test_parts as t
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        hg = pmm.HostGraph.read(os.path.join(root, "tests", "golden", "graphs", "cl3000"), labeled=True)
        seen = {}

        def fake_place(hg_, src, srt, **kw):
            ranges = kw["keep_alive"]
            seen["views"] = [r.read_all(4 * hg_.n_adj) for r in ranges]
            seen["ptrs"] = (src == ranges[0].ptr, srt == (ranges[1].ptr if kw["labeled"] else None))
            return "graph"

        pp.Range = t._FakeRange
        pp.granularity = lambda device=0: 4096
        pmm.GraphPreprocessor.from_paged_source = staticmethod(fake_place)
        g = pp.place_distributed(hg, rank, world, job=job, device=0, barrier=dist.barrier, labeled=labeled,
                                 page_bytes=4096)
        want = [pp.label_grouped(hg).tobytes(), hg.colidx.tobytes()] if labeled else [hg.colidx.tobytes()]
        q.put((rank, g == "graph" and seen["views"] == want and all(seen["ptrs"])))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("labeled", [True, False], ids=["labeled", "unlabeled"])
def test_gloo_distributed_placement_sees_every_slice_filled(labeled):
    """place_distributed's order on three gloo ranks, with a memfd standing in
    for each rank's slice: every rank allocates its own slice, imports the
    others', and builds the graph only after every slice was written, seeing
    each array whole."""
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    job = uuid.uuid4().hex[:12]
    procs = [ctx.Process(target=_place_worker, args=(r, world, port, job, labeled, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get() for _ in range(world))
    assert all(got[r] for r in range(world)), got
