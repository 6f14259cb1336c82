"""Resumable runs (host logic, CPU): an interrupted run continues from its
saved cursor and ends with the full count; a state file of another job is
refused."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pm_oracle as orc  # noqa: E402
import pumatch_b200 as pm  # noqa: E402
from pumatch_b200 import patterns as P  # noqa: E402
from pumatch_b200 import resume  # noqa: E402


class Crash(Exception):
    pass


def _job():
    hg = pm.HostGraph.read(os.path.join(ROOT, "tests", "golden", "graphs", "cl3000"), labeled=True)
    texts = [P.to_g(*P.cycle(4)), P.to_g(*P.house())]
    g = orc.Graph(hg.rowptr, hg.colidx, None)
    plans = [orc.plan(t, False) for t in texts]
    roots = [orc.roots(g, p) for p in plans]
    n = max(len(r) for r in roots)

    def run_range(b, e):
        out = []
        for p, r in zip(plans, roots):
            bb, ee = min(b, len(r)), min(e, len(r))
            out.append(orc.count(g, p, r, bb, ee)[0] * p.multiplicity if ee > bb else 0)
        return out

    full = [orc.count(g, p, r)[0] * p.multiplicity for p, r in zip(plans, roots)]
    return run_range, n, full


def test_resume_after_interruptions(tmp_path):
    run_range, n, full = _job()
    path = str(tmp_path / "state.json")
    calls = {"k": 0}

    def flaky(b, e):
        calls["k"] += 1
        if calls["k"] in (3, 7):  # die in the middle of the run, twice
            raise Crash()
        return run_range(b, e)

    for _ in range(3):
        try:
            got = resume.run_resumable(flaky, n, 2, path, key="job-a", chunk_roots=500)
            break
        except Crash:
            saved = json.load(open(path))
            assert 0 <= saved["next"] <= n and saved["next"] % 500 == 0
    assert got == full
    assert json.load(open(path))["next"] == n
    # a finished state returns its totals without running anything
    assert resume.run_resumable(lambda b, e: 1 / 0, n, 2, path, key="job-a", chunk_roots=500) == full


def test_resume_refuses_another_jobs_state(tmp_path):
    run_range, n, _ = _job()
    path = str(tmp_path / "state.json")
    resume.run_resumable(run_range, n, 2, path, key="job-a", chunk_roots=2000)
    for kw in (dict(key="job-b", n_roots=n, n_patterns=2), dict(key="job-a", n_roots=n + 1, n_patterns=2),
               dict(key="job-a", n_roots=n, n_patterns=3)):
        with pytest.raises(ValueError):
            resume.run_resumable(run_range, kw["n_roots"], kw["n_patterns"], path, key=kw["key"])


def test_job_key_changes_with_what_changes_counts():
    a = resume.job_key({"n_vertices": 5}, [{"nslots": 3}], {"truncate": 0})
    assert a == resume.job_key({"n_vertices": 5}, [{"nslots": 3}], {"truncate": 0})
    assert a != resume.job_key({"n_vertices": 6}, [{"nslots": 3}], {"truncate": 0})
    assert a != resume.job_key({"n_vertices": 5}, [{"nslots": 3}], {"truncate": 16})
    # same shape, other edges (root lists differ) or another root order: another job
    assert a != resume.job_key({"n_vertices": 5}, [{"nslots": 3}], {"truncate": 0}, ["roots-x"])
    assert (resume.job_key({"n_vertices": 5}, [{"nslots": 3}], {"truncate": 0}, ["roots-x"])
            != resume.job_key({"n_vertices": 5}, [{"nslots": 3}], {"truncate": 0}, ["roots-x", "order:1"]))


def test_same_shape_other_edges_gives_another_key():
    """Two graphs of one shape (vertices, adjacency entries, max degree) but
    different edges: their root lists differ, so their jobs do."""
    import hashlib

    import numpy as np
    rp = np.array([0, 2, 4, 6, 8], dtype=np.uint64)
    a = np.array([1, 2, 0, 3, 0, 3, 1, 2], dtype=np.int32)  # 4-cycle 0-1-3-2-0
    b = np.array([1, 3, 0, 2, 1, 3, 0, 2], dtype=np.int32)  # 4-cycle 0-1-2-3-0
    p = orc.plan(P.to_g(*P.path(3)), False)
    keys = []
    for ci in (a, b):
        g = orc.Graph(rp, ci, None)
        digest = hashlib.sha256(np.ascontiguousarray(orc.roots(g, p), dtype=np.int32).tobytes()).hexdigest()
        keys.append(resume.job_key({"n_vertices": 4, "n_adj": 8, "max_degree": 2}, [{"p": 1}], {"truncate": 0},
                                   [digest]))
    assert keys[0] != keys[1]


@pytest.mark.gpu
def test_gpu_match_resumable_equals_one_launch(tmp_path):
    ctx = pm.Context(0)
    try:
        hg = pm.HostGraph.read(os.path.join(ROOT, "tests", "golden", "graphs", "cl3000"), labeled=False)
        g = pm.GraphPreprocessor.from_host(hg)
        plans = [pm.PatternPreprocessor(text=P.to_g(*P.clique(5)), labeled=False),
                 pm.PatternPreprocessor(text=P.to_g(*P.house()), labeled=False)]
        want, _ = ctx.match(g, plans)
        path = str(tmp_path / "state.json")
        assert resume.match_resumable(ctx, g, plans, path, chunk_roots=997) == want
        assert resume.match_resumable(ctx, g, plans, path, chunk_roots=997) == want  # finished state
        # a root order is part of the job: its state file is another job's
        import numpy as np
        n = ctx.count_roots(g, plans[0])
        order = np.random.default_rng(3).permutation(n).astype(np.int32)
        want1, _ = ctx.match(g, plans[:1])
        with pytest.raises(ValueError):
            resume.match_resumable(ctx, g, plans[:1], path, chunk_roots=997, root_order=order)
        p2 = str(tmp_path / "state2.json")
        assert resume.match_resumable(ctx, g, plans[:1], p2, chunk_roots=997, root_order=order) == want1
        g.close()
    finally:
        ctx.close()
