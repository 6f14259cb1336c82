"""The C-ABI boundary: the library loads, exports every entry point that
include/pumatch.h declares, the ctypes mirror matches the C struct layouts,
and the product refuses to run without a GPU (no CPU fallback)."""
import os
import re
import subprocess

import pytest
import torch

import pumatch_b200 as pm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def declared():
    names = set()
    for h in HEADERS:
        src = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"^[A-Za-z_][\w \*]*?\b(pm_\w+)\s*\(", src, flags=re.M))
    return names


def test_header_declares_entry_points():
    names = declared()
    for n in ("pm_graph_open", "pm_plan_compile", "pm_match", "pm_ctx_create", "pm_strerror"):
        assert n in names


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", pm.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r" T (pm_\w+)", out.stdout))
    missing = declared() - exported
    assert not missing, missing
    L = pm.lib()
    for n in declared():
        assert hasattr(L, n)
    # the Python mirror binds every declared entry point
    assert declared() <= set(pm.SIGNATURES)


def test_struct_layouts_match_c():
    """Compiles a probe against the header and compares sizeof/offsetof."""
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "pumatch.h"
int main(void){
 printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(pm_graph_opts), sizeof(pm_graph_info), sizeof(pm_plan_desc),
        sizeof(pm_run_opts), sizeof(pm_stats), offsetof(pm_run_opts, root_begin), offsetof(pm_run_opts, root_counts),
        offsetof(pm_stats, kernel_ms));
 return 0; }'''
    import ctypes as C
    import tempfile
    d = tempfile.mkdtemp()
    open(os.path.join(d, "p.c"), "w").write(src)
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", os.path.join(d, "p"), os.path.join(d, "p.c")],
                   check=True)
    vals = [int(x) for x in subprocess.run([os.path.join(d, "p")], capture_output=True, text=True).stdout.split()]
    assert vals == [C.sizeof(pm.GraphOpts), C.sizeof(pm.GraphInfo), C.sizeof(pm.PlanDesc), C.sizeof(pm.RunOpts),
                    C.sizeof(pm.Stats), pm.RunOpts.root_begin.offset, pm.RunOpts.root_counts.offset,
                    pm.Stats.kernel_ms.offset]


def test_strerror():
    assert pm.lib().pm_strerror(pm.PM_ERR_NO_DEVICE) == b"no CUDA device"
    assert pm.lib().pm_strerror(pm.PM_OK) == b"ok"


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback():
    with pytest.raises(pm.PmError) as e:
        pm.Context(0)
    assert e.value.status == pm.PM_ERR_NO_DEVICE
    hg = pm.gen_chung_lu(100, 300, seed=1)
    with pytest.raises(pm.PmError) as e:
        pm.GraphPreprocessor.from_host(hg)
    assert e.value.status == pm.PM_ERR_NO_DEVICE
    # partitioned residency: no device range without a device
    from pumatch_b200 import parts
    with pytest.raises(pm.PmError) as e:
        parts.granularity(0)
    assert e.value.status == pm.PM_ERR_NO_DEVICE
    with pytest.raises(pm.PmError) as e:
        pm.GraphPreprocessor.from_paged_source(hg, 1 << 20)  # refused before the pointer is used
    assert e.value.status == pm.PM_ERR_NO_DEVICE
    # the drop-in CLI fails loudly too
    gold = os.path.join(ROOT, "tests", "golden", "graphs", "cl400")
    pat = os.path.join(ROOT, "tests", "golden", "_c4.g")
    from pumatch_b200 import patterns as P
    open(pat, "w").write(P.to_g(*P.cycle(4)))
    try:
        r = subprocess.run([pm.CLI_PATH, gold, pat], capture_output=True, text=True)
        assert r.returncode != 0 and "no CUDA device" in r.stderr
    finally:
        os.remove(pat)


def test_static_entry_argument_checks():
    """pm_match_static refuses, before touching a device, what it cannot run:
    vertex ids beyond int32 and the per-root options it does not support."""
    import ctypes as C
    from pumatch_b200 import patterns as P
    plan = pm.PatternPreprocessor(text=P.to_g(*P.cycle(4)), labeled=False)
    fake = C.c_void_p(16)  # never dereferenced: the checks come first
    cnt = C.c_uint64()
    rc = pm.lib().pm_match_static(fake, fake, None, 1 << 31, 10, 4, plan._h, None, None, C.byref(cnt), None)
    assert rc == pm.PM_ERR_INVALID and b"int32" in pm.lib().pm_last_error()
    o = pm.Context._opts(root_counts_ptr=16)
    rc = pm.lib().pm_match_static(fake, fake, None, 100, 10, 4, plan._h, C.byref(o), None, C.byref(cnt), None)
    assert rc == pm.PM_ERR_INVALID


def test_cli_usage():
    r = subprocess.run([pm.CLI_PATH], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    assert "--tuned" in r.stderr


def test_cli_tuned_file_errors(tmp_path):
    gold = os.path.join(ROOT, "tests", "golden", "graphs", "cl400")
    r = subprocess.run([pm.CLI_PATH, gold, "x.g", "--tuned=" + str(tmp_path / "none.json")],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open" in r.stderr
    bad = tmp_path / "bad.json"
    bad.write_text('{"results": []}')
    r = subprocess.run([pm.CLI_PATH, gold, "x.g", "--tuned=" + str(bad)], capture_output=True, text=True)
    assert r.returncode == 1 and "best" in r.stderr
    r = subprocess.run([pm.CLI_PATH, gold, "x.g", "--bogus"], capture_output=True, text=True)
    assert r.returncode == 2


def test_cli_parts_options():
    """--parts (partitioned residency) is validated before anything runs, and
    without a GPU the CLI fails loudly: no slice is ever placed in host
    memory instead."""
    gold = os.path.join(ROOT, "tests", "golden", "graphs", "cl400")
    r = subprocess.run([pm.CLI_PATH], capture_output=True, text=True)
    assert "--parts=K" in r.stderr
    for bad in (["--parts-device=0"], ["--parts=-1"], ["--parts=5000"]):
        r = subprocess.run([pm.CLI_PATH, gold, "x.g", *bad], capture_output=True, text=True)
        assert r.returncode == 2 and "--parts" in r.stderr, bad
    if not torch.cuda.is_available():
        from pumatch_b200 import patterns as P
        pat = os.path.join(ROOT, "tests", "golden", "_c4_parts.g")
        open(pat, "w").write(P.to_g(*P.cycle(4)))
        try:
            r = subprocess.run([pm.CLI_PATH, gold, pat, "--parts=2"], capture_output=True, text=True)
            assert r.returncode == 1 and "no CUDA device" in r.stderr
        finally:
            os.remove(pat)


def test_run_option_keywords():
    """Every run option the bench, the tests and the learned/autotune helpers
    pass maps onto a pm_run_opts field; a misspelt one is an error, not a
    silently ignored attribute."""
    o = pm.Context._opts(truncate=4, warps_per_block=8, blocks_per_sm=2, chunk=7, split_level1=16, shard_rank=1,
                         shard_count=2, root_begin=3, root_end=9, timeout_ms=1000, cold_cache=True,
                         high_occupancy=2, leaf_per_lane=1, lane_subtree_max=-1, use_graph=True, root_counts_ptr=0,
                         root_cost_ptr=0, root_order_ptr=0, root_reads_ptr=0)
    assert (o.truncate, o.chunk, o.root_begin, o.root_end, o.leaf_per_lane, o.high_occupancy) == (4, 7, 3, 9, 1, 2)
    assert o.cold_cache == 1 and o.use_graph == 1 and o.root_order is None
    d = pm.Context._opts()
    assert d.root_begin == -1 and d.root_end == -1 and d.leaf_per_lane == 0 and d.lane_subtree_max == 0
    assert o.lane_subtree_max == -1
    with pytest.raises(TypeError):
        pm.Context._opts(leaf_mode=1)


def test_new_fields_match_c():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "pumatch.h"
int main(void){
 printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", offsetof(pm_graph_opts, static_pool_bytes),
        offsetof(pm_graph_info, n_static_frames),
        offsetof(pm_run_opts, leaf_per_lane), offsetof(pm_run_opts, lane_subtree_max), offsetof(pm_stats, warp_ns),
        offsetof(pm_stats, idle_ns), offsetof(pm_run_opts, own_arena_words), offsetof(pm_run_opts, max_borrowed),
        offsetof(pm_stats, borrowed_arenas), offsetof(pm_stats, arena_pool), sizeof(pm_run_opts), sizeof(pm_stats));
 printf("%zu %zu %zu\n", offsetof(pm_stats, leaf_cycles), offsetof(pm_stats, level_cycles), offsetof(pm_stats, prefix_cycles));
 printf("%zu %zu %zu %zu %zu %zu\n", offsetof(pm_run_opts, prefetch_ahead), offsetof(pm_run_opts, prefetch_off),
        offsetof(pm_run_opts, prefetch_pages), offsetof(pm_run_opts, prefetch_chunks), offsetof(pm_stats, prefetch_requests),
        offsetof(pm_run_opts, root_split));
 printf("%zu %zu %zu %zu\n", offsetof(pm_stats, page_requests), offsetof(pm_stats, page_dropped),
        offsetof(pm_stats, device_page_loads), offsetof(pm_run_opts, host_page_copy));
 return 0; }'''
    import ctypes as C
    import tempfile
    d = tempfile.mkdtemp()
    open(os.path.join(d, "p.c"), "w").write(src)
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", os.path.join(d, "p"), os.path.join(d, "p.c")],
                   check=True)
    vals = [int(x) for x in subprocess.run([os.path.join(d, "p")], capture_output=True, text=True).stdout.split()]
    assert vals == [pm.GraphOpts.static_pool_bytes.offset, pm.GraphInfo.n_static_frames.offset,
                    pm.RunOpts.leaf_per_lane.offset, pm.RunOpts.lane_subtree_max.offset, pm.Stats.warp_ns.offset,
                    pm.Stats.idle_ns.offset, pm.RunOpts.own_arena_words.offset, pm.RunOpts.max_borrowed.offset,
                    pm.Stats.borrowed_arenas.offset, pm.Stats.arena_pool.offset, C.sizeof(pm.RunOpts),
                    C.sizeof(pm.Stats), pm.Stats.leaf_cycles.offset, pm.Stats.level_cycles.offset,
                    pm.Stats.prefix_cycles.offset, pm.RunOpts.prefetch_ahead.offset, pm.RunOpts.prefetch_off.offset,
                    pm.RunOpts.prefetch_pages.offset, pm.RunOpts.prefetch_chunks.offset,
                    pm.Stats.prefetch_requests.offset, pm.RunOpts.root_split.offset,
                    pm.Stats.page_requests.offset, pm.Stats.page_dropped.offset,
                    pm.Stats.device_page_loads.offset, pm.RunOpts.host_page_copy.offset]


def test_c_program_links_and_runs_host_entry_points(tmp_path):
    """A plain C caller that only includes pumatch.h: compile a pattern,
    describe it, build and renumber a graph, and get PM_ERR_NO_DEVICE (not a
    CPU fallback) from the device entry points."""
    src = r'''
#include <stdio.h>
#include <stdlib.h>
#include "pumatch.h"
int main(void){
  pm_plan* p = NULL;
  const char* k4 = "v 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 0 2 1\ne 0 3 1\ne 1 2 1\ne 1 3 1\ne 2 3 1\n";
  if (pm_plan_compile_text(k4, 0, &p) != PM_OK) { printf("compile %s\n", pm_last_error()); return 1; }
  pm_plan_desc d;
  if (pm_plan_describe(p, &d) != PM_OK) return 2;
  uint64_t* rp = NULL; int32_t* ci = NULL; int64_t nadj = 0; int32_t md = 0;
  if (pm_gen_chung_lu(500, 2000, 2.1, 5.0, 100.0, 3, &rp, &ci, &nadj, &md) != PM_OK) return 3;
  uint64_t* rp2 = malloc(sizeof(uint64_t) * 501); int32_t* ci2 = malloc(sizeof(int32_t) * nadj);
  if (pm_reorder_by_degree(500, nadj, rp, ci, NULL, rp2, ci2, NULL, NULL) != PM_OK) return 4;
  pm_ctx* c = NULL;
  pm_status s = pm_ctx_create(0, &c);
  printf("%d %d %d %lld %d\n", d.nnodes, d.multiplicity, (int)(rp2[1] - rp2[0]) == md, (long long)nadj,
         s == PM_ERR_NO_DEVICE);
  pm_host_free(rp); pm_host_free(ci); free(rp2); free(ci2); pm_plan_free(p);
  return 0; }'''
    lib_dir = os.path.dirname(pm.LIB_PATH)
    exe = str(tmp_path / "c_caller")
    open(str(tmp_path / "c.c"), "w").write(src)
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe, str(tmp_path / "c.c"), "-L", lib_dir,
                    "-lpumatch_b200", "-Wl,-rpath," + lib_dir], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    nn, mult, maxfirst, nadj, nodev = r.stdout.split()
    assert (nn, mult, maxfirst, nodev) == ("4", "24", "1", "1") and int(nadj) == 4000


def test_stats_json_sidecar():
    import ctypes as C
    import json as js
    st = pm.Stats()
    st.kernel_ms, st.n_roots, st.set_ops, st.alg_bytes = 2000.0, 7, 11, 4_000_000_000
    st.page_hits, st.warp_ns, st.idle_ns, st.grid_blocks = 5, 1000, 250, 444
    st.borrowed_arenas, st.arena_pool = 3, 9
    counts = (C.c_uint64 * 2)(10, 2**63)
    need = C.c_size_t()
    assert pm.lib().pm_stats_json(C.byref(st), counts, 2, None, 0, C.byref(need)) == pm.PM_ERR_INVALID
    buf = C.create_string_buffer(need.value)
    assert pm.lib().pm_stats_json(C.byref(st), counts, 2, buf, need.value, None) == pm.PM_OK
    d = js.loads(buf.value.decode())
    assert d["counts"] == [10, 2**63] and d["set_ops"] == 11 and d["n_roots"] == 7
    assert abs(d["alg_gbs"] - 2.0) < 1e-9 and abs(d["warp_idle_share"] - 0.25) < 1e-9
    assert abs(d["matches_per_s"] - (10 + 2**63) / 2.0) / d["matches_per_s"] < 1e-6
    assert d["grid_blocks"] == 444 and d["device_status"] == 0
    assert d["borrowed_arenas"] == 3 and d["arena_pool"] == 9
