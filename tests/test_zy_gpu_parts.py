"""Partitioned residency on the GPU: a paged graph whose pages come from an
adjacency array cut into slices of device memory mapped into one range
(pm_parts_*), here with every slice on the one GPU a run has, standing in
for the slices of several GPUs.  Counts and set operations must equal the
oracle's (on a small graph, the HBM placement's), misses must be served from
the range (warp copies and the host service thread's device-to-device
copies), slices passed through file descriptors must work like local ones,
and two processes that each own one slice and import the other's must
together count what the oracle counts.
The file is collected after every other GPU test but the allocation-free
entry's."""
import datetime
import os
import socket
import uuid

import pytest
import torch.multiprocessing as mp

import pm_oracle as orc
import pumatch_b200 as pm
from pumatch_b200 import parts
from pumatch_b200 import patterns as P

pytestmark = pytest.mark.gpu

_cache = {}


def workload():
    # 3.2M adjacency entries (12.8 MB): three slices at the 2 MB granularity
    if "w" not in _cache:
        hg = pm.gen_chung_lu(400_000, 1_600_000, gamma=2.1, i0=3.0, max_w=2500.0, seed=43)
        lab = pm.gen_labels(hg.n, 4, seed=44)
        _cache["w"] = pm.HostGraph(hg.rowptr, hg.colidx, lab)
    return _cache["w"]


TEXTS = {
    "C4_lab": (P.to_g(*P.cycle(4), [0, 1, 2, 1]), True),
    "house_lab": (P.to_g(*P.house(), [1, 2, 0, 3, 2]), True),
    "K4": (P.to_g(*P.clique(4)), False),
    "C4": (P.to_g(*P.cycle(4)), False),
}


def root_range(n_roots):
    """20,000 root positions from the middle of the list (the first roots are
    the hubs', far heavier): a bounded amount of work per run."""
    b = n_roots // 2
    return b, min(n_roots, b + 20000)


def oracle_counts(hg, labeled):
    """The oracle's count and set operations of each pattern over its root
    range (a few seconds each on the CPU)."""
    key = ("oracle", labeled)
    if key not in _cache:
        g = orc.Graph(hg.rowptr, hg.colidx, hg.labels if labeled else None)
        res = {}
        for name, (text, lab) in TEXTS.items():
            if lab != labeled:
                continue
            p = orc.plan(text, labeled)
            roots = orc.roots(g, p)
            b, e = root_range(len(roots))
            c, st = orc.count(g, p, roots, b, e)
            res[name] = ((b, e), c if labeled else c * p.multiplicity, st["set_ops"])
        _cache[key] = res
    return _cache[key]


GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("export_import", [False, True], ids=["local", "fd"])
def test_one_slice_source_counts_equal_hbm(ctx, export_import):
    """A golden graph in one slice (48 KB of adjacency, 12 pages of 4 KB
    through a pool of 4 frames): labeled and unlabeled counts and set
    operations equal the HBM placement's, with warp copies and with the host
    service thread's device-to-device copies."""
    hg = pm.HostGraph.read(os.path.join(GOLD, "graphs", "cl3000"), labeled=True)
    for text, labeled in ((P.to_g(*P.cycle(5), [0, 0, 1, 1, 0]), True), (P.to_g(*P.clique(4)), False)):
        p = pm.PatternPreprocessor(text=text, labeled=labeled)
        g = pm.GraphPreprocessor.from_host(hg, labeled=labeled)
        want, st = ctx.match(g, [p], timeout_ms=20000)
        g.close()
        g = parts.place_local(hg, 1, labeled=labeled, frame_pool_bytes=4 * 4096, page_bytes=4096,
                              export_import=export_import)
        try:
            for hc in (0, 1):
                got, s2 = ctx.match(g, [p], cold_cache=True, timeout_ms=20000, host_page_copy=hc)
                assert got == want and s2["set_ops"] == st["set_ops"], (labeled, hc)
                assert s2["page_misses"] > 0
        finally:
            g.close()


@pytest.mark.parametrize("labeled", [True, False], ids=["labeled", "unlabeled"])
@pytest.mark.parametrize("mode", ["local", "fd", "host-copies"])
def test_three_slices_count_like_the_oracle(ctx, labeled, mode):
    hg = workload()
    pb = 16 << 10
    g = parts.place_local(hg, 3, labeled=labeled, frame_pool_bytes=64 * pb, page_bytes=pb,
                          static_pool_bytes=16 * pb, export_import=(mode == "fd"))
    assert len(parts.slice_bounds(4 * hg.n_adj, 3, parts.granularity(0), pb)[0]) == 3
    try:
        info = g.info()
        assert info["residency"] == pm.PM_RESIDENT_PAGED and info["n_frames"] == 64
        assert info["n_static_frames"] == 16
        want = oracle_counts(hg, labeled)
        for name, (text, lab) in TEXTS.items():
            if lab != labeled:
                continue
            (b, e), count, ops = want[name]
            p = pm.PatternPreprocessor(text=text, labeled=labeled)
            for cold in (True, False):
                got, st = ctx.match(g, [p], root_begin=b, root_end=e, cold_cache=cold, timeout_ms=120000,
                                    host_page_copy=int(mode == "host-copies"))
                assert (got[0], st["set_ops"]) == (count, ops), (name, mode, cold)
                if cold:
                    assert st["page_misses"] > 0
                    assert st["pages_loaded"] + st["device_page_loads"] > 0, (name, mode)
    finally:
        g.close()


def test_cli_parts_count_equals_hbm(tmp_path):
    """The drop-in CLI with --parts prints the count the HBM placement
    prints (the last stdout line, "<ms> <count>")."""
    import subprocess
    gold = os.path.join(GOLD, "graphs", "cl3000")
    pat = tmp_path / "c5.g"
    pat.write_text(P.to_g(*P.cycle(5), [0, 0, 1, 1, 0]))
    counts = []
    for extra in ([], ["--parts=2", "--parts-device=0", "--page-kb=4", "--frame-mb=1"]):
        r = subprocess.run([pm.CLI_PATH, gold, str(pat), *extra], capture_output=True, text=True, cwd=tmp_path,
                           timeout=300)
        assert r.returncode == 0, r.stderr
        counts.append(int(r.stdout.strip().splitlines()[-1].split()[1]))
    assert counts[0] == counts[1] > 0


def test_source_arguments_are_checked():
    hg = workload()
    with pytest.raises(pm.PmError):  # labeled without the id-sorted array
        pm.GraphPreprocessor.from_paged_source(hg, 1 << 40, None, labeled=True)
    with pytest.raises(pm.PmError):  # misaligned source
        pm.GraphPreprocessor.from_paged_source(hg, (1 << 40) + 4, None, labeled=False)
    gran = parts.granularity(0)
    with pytest.raises(pm.PmError):  # a slice boundary off the granularity
        parts.Range(0, [0, gran // 2], 2 * gran)
    r = parts.Range(0, [0, gran], 2 * gran)
    try:
        r.alloc(0, 0)
        with pytest.raises(pm.PmError):  # slice 1 has no memory
            r.map()
    finally:
        r.close()


def _rank_worker(rank, world, port, job, labeled, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    import pumatch_b200 as pmm
    from pumatch_b200 import parts as pp
    import test_zy_gpu_parts as t
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        hg = t.workload()
        pb = 16 << 10
        g = pp.place_distributed(hg, rank, world, job=job, device=0, barrier=dist.barrier, labeled=labeled,
                                 frame_pool_bytes=64 * pb, page_bytes=pb)
        ctx = pmm.Context(0)
        out = {}
        for name, (text, lab) in t.TEXTS.items():
            if lab != labeled:
                continue
            p = pmm.PatternPreprocessor(text=text, labeled=labeled)
            roots = ctx.roots(g, p)
            begins, total = pp.slice_bounds(4 * hg.n_adj, world, pp.granularity(0), pb)
            rng = pp.owner_root_ranges(hg.rowptr, roots, begins, total)
            b, e = rng[rank] if rank < len(rng) else (0, 0)
            # this rank's roots within the pattern's root range
            r0, r1 = t.root_range(len(roots))
            b, e = max(b, r0), min(e, r1)
            if b >= e:
                out[name] = (0, 0)
                continue
            c, st = ctx.match(g, [p], root_begin=b, root_end=e, cold_cache=True, timeout_ms=120000)
            out[name] = (c[0], st["set_ops"])
        dist.barrier()  # no rank unmaps its slice while another may still read it
        g.close()
        ctx.close()
        dist.barrier()
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("labeled", [True, False], ids=["labeled", "unlabeled"])
def test_two_processes_each_owning_a_slice_count_the_whole(ctx, labeled):
    hg = workload()
    want = {name: (c, ops) for name, (_, c, ops) in oracle_counts(hg, labeled).items()}
    world = 2
    mpc = mp.get_context("spawn")
    q = mpc.SimpleQueue()
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    job = uuid.uuid4().hex[:12]
    procs = [mpc.Process(target=_rank_worker, args=(r, world, port, job, labeled, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        if p.exitcode is None:
            p.kill()
        assert p.exitcode == 0
    got = dict(q.get() for _ in range(world))
    for name in want:
        c = sum(got[r][name][0] for r in range(world))
        ops = sum(got[r][name][1] for r in range(world))
        assert (c, ops) == want[name], name
