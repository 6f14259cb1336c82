"""pumatch_b200 -- B200-native subgraph matcher.

Host-side mirror of the reference's driver interface (PUMatch ``test.cu`` and
its header-only preprocessors) over the C-ABI of ``libpumatch_b200.so``:

    GraphPreprocessor(prefix)          -> reference src/graph.h:34-41
    PatternPreprocessor(path)          -> reference src/pattern.h:48-58
    count_roots(graph, pattern)        -> reference src/job_queue.h:39-64
    match(graph, patterns, ...)        -> reference test.cu:171-198

Every call goes through the compiled library; there is no Python or CPU
fallback.  If the library is missing, importing the matcher API raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Iterable, Optional, Sequence

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libpumatch_b200.so")
CLI_PATH = os.path.join(_PKG, "bin", "test")

PM_OK, PM_ERR_IO, PM_ERR_FORMAT, PM_ERR_OOM, PM_ERR_CUDA = 0, 1, 2, 3, 4
PM_ERR_TIMEOUT, PM_ERR_INVALID, PM_ERR_INTERNAL, PM_ERR_NO_DEVICE = 5, 6, 7, 8
PM_RESIDENT_HBM, PM_RESIDENT_PAGED = 0, 1
MAX_PAT, MAX_SLOTS = 7, 15


class PmError(RuntimeError):
    """A non-OK pm_status, with the library's message for this thread."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message


class GraphOpts(C.Structure):
    _fields_ = [("labeled", C.c_int), ("device", C.c_int), ("residency", C.c_int),
                ("page_bytes", C.c_uint32), ("frame_pool_bytes", C.c_uint64), ("static_pool_bytes", C.c_uint64)]


class GraphInfo(C.Structure):
    _fields_ = [("n_vertices", C.c_int64), ("n_adj", C.c_int64), ("max_degree", C.c_int32),
                ("labeled", C.c_int32), ("n_labels", C.c_int32), ("residency", C.c_int32),
                ("device_bytes", C.c_uint64), ("n_pages", C.c_uint64), ("n_frames", C.c_uint64),
                ("n_static_frames", C.c_uint64)]


class PlanDesc(C.Structure):
    _fields_ = [("nnodes", C.c_int32), ("nslots", C.c_int32), ("multiplicity", C.c_int32),
                ("labeled", C.c_int32), ("level_begin", C.c_int32 * (MAX_PAT + 1)),
                ("degree", C.c_int32 * MAX_PAT), ("vertex_label", C.c_int32 * MAX_PAT),
                ("slot_labels", C.c_uint32 * MAX_SLOTS), ("partial", C.c_uint32 * MAX_SLOTS),
                ("set_ops", C.c_uint8 * MAX_SLOTS), ("pad_", C.c_uint8)]


class RunOpts(C.Structure):
    _fields_ = [("truncate", C.c_int32), ("warps_per_block", C.c_int32), ("blocks_per_sm", C.c_int32),
                ("chunk", C.c_int32), ("split_level1", C.c_int32), ("shard_rank", C.c_int32),
                ("shard_count", C.c_int32), ("use_graph", C.c_int32), ("timeout_ms", C.c_int32),
                ("root_begin", C.c_int64), ("root_end", C.c_int64), ("cold_cache", C.c_int32),
                ("high_occupancy", C.c_int32), ("leaf_per_lane", C.c_int32), ("lane_subtree_max", C.c_int32),
                ("root_counts", C.c_void_p), ("root_cost", C.c_void_p), ("root_order", C.c_void_p),
                ("root_reads", C.c_void_p), ("own_arena_words", C.c_int64), ("max_borrowed", C.c_int32),
                ("prefetch_ahead", C.c_int32), ("prefetch_off", C.c_void_p), ("prefetch_pages", C.c_void_p),
                ("prefetch_chunks", C.c_int64), ("root_split", C.c_void_p),
                ("host_page_copy", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("n_roots", C.c_uint64), ("set_ops", C.c_uint64), ("alg_bytes", C.c_uint64),
                ("splits", C.c_uint64), ("page_hits", C.c_uint64), ("page_misses", C.c_uint64),
                ("h2d_page_bytes", C.c_uint64), ("zero_copy_bytes", C.c_uint64),
                ("pages_loaded", C.c_uint64), ("evictions", C.c_uint64), ("kernel_ms", C.c_float),
                ("roots_ms", C.c_float), ("grid_blocks", C.c_int32), ("block_threads", C.c_int32),
                ("arena_bytes", C.c_uint64), ("device_status", C.c_uint32), ("pad_", C.c_uint32),
                ("warp_ns", C.c_uint64), ("idle_ns", C.c_uint64), ("borrowed_arenas", C.c_uint64),
                ("arena_pool", C.c_uint64), ("leaf_cycles", C.c_uint64), ("level_cycles", C.c_uint64),
                ("prefix_cycles", C.c_uint64), ("prefetch_requests", C.c_uint64),
                ("page_requests", C.c_uint64), ("page_dropped", C.c_uint64),
                ("device_page_loads", C.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.endswith("_")}


_lib = None

# name -> (restype, argtypes) of every C-ABI entry point in include/pumatch.h
_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
SIGNATURES = {
    "pm_graph_opts_default": (None, [C.POINTER(GraphOpts)]),
    "pm_graph_open": (C.c_int, [C.c_char_p, C.POINTER(GraphOpts), _PP]),
    "pm_graph_from_host": (C.c_int, [C.c_int64, C.c_int64, _P, _P, _P, C.POINTER(GraphOpts), _PP]),
    "pm_graph_from_device": (C.c_int, [C.c_int64, C.c_int64, C.c_int32, _P, _P, _P, C.c_int, _PP]),
    "pm_graph_get_info": (C.c_int, [_P, C.POINTER(GraphInfo)]),
    "pm_graph_set_resident_pages": (C.c_int, [_P, _P, C.c_int64]),
    "pm_graph_close": (None, [_P]),
    "pm_graph_read": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                C.POINTER(C.c_int32), _PP, _PP, _PP]),
    "pm_graph_write": (C.c_int, [C.c_char_p, C.c_int64, C.c_int64, _P, _P, _P]),
    "pm_host_free": (None, [_P]),
    "pm_convert_snap": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.POINTER(C.c_int64),
                                  C.POINTER(C.c_int64)]),
    "pm_reorder_by_degree": (C.c_int, [C.c_int64, C.c_int64, _P, _P, _P, _P, _P, _P, _P]),
    "pm_stats_json": (C.c_int, [_P, _P, C.c_int, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "pm_halve": (C.c_int, [C.c_int64, C.c_int64, _P, _P, _P, _P, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "pm_gen_chung_lu": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                  _PP, _PP, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "pm_gen_rmat": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                              _PP, _PP, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "pm_gen_rmat_device": (C.c_int, [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                     C.c_int, _PP, _PP, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "pm_gen_labels": (C.c_int, [C.c_int64, C.c_int, C.c_uint64, _PP]),
    "pm_plan_compile": (C.c_int, [C.c_char_p, C.c_int, _PP]),
    "pm_plan_compile_text": (C.c_int, [C.c_char_p, C.c_int, _PP]),
    "pm_plan_describe": (C.c_int, [_P, C.POINTER(PlanDesc)]),
    "pm_plan_free": (None, [_P]),
    "pm_count_roots": (C.c_int, [_P, _P, _P, C.POINTER(C.c_int64)]),
    "pm_debug_roots": (C.c_int, [_P, _P, _P, _P, C.c_int64, C.POINTER(C.c_int64)]),
    "pm_ctx_create": (C.c_int, [C.c_int, _PP]),
    "pm_ctx_destroy": (None, [_P]),
    "pm_ctx_stream": (C.c_void_p, [_P]),
    "pm_run_opts_default": (None, [C.POINTER(RunOpts)]),
    "pm_match": (C.c_int, [_P, _P, _PP, C.c_int, C.POINTER(RunOpts), C.POINTER(C.c_uint64),
                           C.POINTER(Stats)]),
    "pm_query_prepare": (C.c_int, [_P, _P, _PP, C.c_int, C.POINTER(RunOpts), _PP]),
    "pm_query_run": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(Stats)]),
    "pm_query_free": (None, [_P]),
    "pm_root_features": (C.c_int, [_P, _P, _P, _P, C.c_int64, C.POINTER(C.c_int64)]),
    "pm_mlp_create": (C.c_int, [C.c_int, C.c_uint64, _PP]),
    "pm_mlp_free": (None, [_P]),
    "pm_mlp_forward": (C.c_int, [_P, _P, C.c_int64, _P]),
    "pm_mlp_gradient": (C.c_int, [_P, _P, _P, C.c_int64, _P, C.POINTER(C.c_float)]),
    "pm_mlp_train_step": (C.c_int, [_P, _P, _P, C.c_int64, C.c_float, C.POINTER(C.c_float)]),
    "pm_mlp_get_weights": (C.c_int, [_P, _P]),
    "pm_mlp_set_weights": (C.c_int, [_P, _P]),
    "pm_match_static": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int64, C.c_int32, _P, C.POINTER(RunOpts), _P,
                                  C.POINTER(C.c_uint64), C.POINTER(Stats)]),
    "pm_parts_granularity": (C.c_int, [C.c_int, C.POINTER(C.c_uint64)]),
    "pm_parts_create": (C.c_int, [C.c_int, C.c_int, _P, C.c_uint64, _PP]),
    "pm_parts_alloc": (C.c_int, [_P, C.c_int, C.c_int]),
    "pm_parts_export": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "pm_parts_import": (C.c_int, [_P, C.c_int, C.c_int]),
    "pm_parts_map": (C.c_int, [_P]),
    "pm_parts_ptr": (C.c_void_p, [_P]),
    "pm_parts_write": (C.c_int, [_P, C.c_uint64, _P, C.c_uint64]),
    "pm_parts_free": (None, [_P]),
    "pm_graph_from_paged_source": (C.c_int, [C.c_int64, C.c_int64, _P, _P, _P, _P, C.POINTER(GraphOpts), _PP]),
    "pm_label_group_host": (C.c_int, [C.c_int64, C.c_int64, _P, _P, _P, _P]),
    "pm_strerror": (C.c_char_p, [C.c_int]),
    "pm_last_error": (C.c_char_p, []),
}


def lib() -> C.CDLL:
    """Loads libpumatch_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m pumatch_b200.build` "
                              "(there is no fallback implementation)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status != PM_OK:
        raise PmError(status, lib().pm_last_error().decode(errors="replace"))


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _take(ptr: C.c_void_p, n: int, dtype) -> np.ndarray:
    """Copies n elements of a malloc'd array into numpy and frees it."""
    if n == 0:
        lib().pm_host_free(ptr)
        return np.zeros(0, dtype=dtype)
    buf = (C.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr.value)
    out = np.frombuffer(buf, dtype=dtype).copy()
    lib().pm_host_free(ptr)
    return out


# ---------------------------------------------------------------- host CSR

class HostGraph:
    """CSR arrays in host memory in the reference's on-disk layout."""

    def __init__(self, rowptr: np.ndarray, colidx: np.ndarray, labels: Optional[np.ndarray] = None):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
        self.colidx = np.ascontiguousarray(colidx, dtype=np.int32)
        self.labels = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint32)

    @property
    def n(self) -> int:
        return len(self.rowptr) - 1

    @property
    def n_adj(self) -> int:
        return len(self.colidx)

    @property
    def max_degree(self) -> int:
        return int(np.diff(self.rowptr).max()) if self.n else 0

    def degrees(self) -> np.ndarray:
        return np.diff(self.rowptr).astype(np.int64)

    def write(self, prefix: str) -> None:
        """Writes <prefix>.meta.txt/.vertex.bin/.edge.bin[/.label.bin]."""
        _check(lib().pm_graph_write(prefix.encode(), self.n, self.n_adj, _ptr(self.rowptr),
                                    _ptr(self.colidx), _ptr(self.labels)))

    @staticmethod
    def read(prefix: str, labeled: bool) -> "HostGraph":
        n, nadj, md = C.c_int64(), C.c_int64(), C.c_int32()
        rp, ci, lb = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _check(lib().pm_graph_read(prefix.encode(), int(labeled), C.byref(n), C.byref(nadj), C.byref(md),
                                   C.byref(rp), C.byref(ci), C.byref(lb)))
        rowptr = _take(rp, n.value + 1, np.uint64)
        colidx = _take(ci, nadj.value, np.int32)
        labels = _take(lb, n.value, np.uint32) if labeled else None
        return HostGraph(rowptr, colidx, labels)


def convert_snap(snap_path: str, out_prefix: Optional[str] = None, n_labels: int = 10,
                 keep_self_loops: bool = False):
    """SNAP text -> the reference's CSR files (default prefix: the text path,
    as graph_converter/convert.sh names them).  Returns (n_vertices, n_adj)."""
    n, nadj = C.c_int64(), C.c_int64()
    _check(lib().pm_convert_snap(snap_path.encode(), (out_prefix or snap_path).encode(), n_labels,
                                 int(keep_self_loops), C.byref(n), C.byref(nadj)))
    return n.value, nadj.value


def reorder_by_degree(hg: HostGraph):
    """The same graph with vertices renumbered by (degree, id), highest first
    (graph_converter/relabel.cpp); labels move with their vertices.  Returns
    (HostGraph, new_id) where new_id[old] is the vertex's new id."""
    rp = np.zeros(hg.n + 1, dtype=np.uint64)
    ci = np.zeros(max(hg.n_adj, 1), dtype=np.int32)
    lb = np.zeros(max(hg.n, 1), dtype=np.uint32) if hg.labels is not None else None
    nid = np.zeros(max(hg.n, 1), dtype=np.int32)
    _check(lib().pm_reorder_by_degree(hg.n, hg.n_adj, _ptr(hg.rowptr), _ptr(hg.colidx),
                                      _ptr(hg.labels) if hg.labels is not None else None, _ptr(rp), _ptr(ci),
                                      _ptr(lb) if lb is not None else None, _ptr(nid)))
    return HostGraph(rp, ci[:hg.n_adj], None if lb is None else lb[:hg.n]), nid[:hg.n]


def halve(hg: HostGraph):
    """Each undirected edge once, towards its heavier end
    (graph_converter/halve.cpp).  Returns (rowptr, colidx, max_degree)."""
    rp = np.zeros(hg.n + 1, dtype=np.uint64)
    ci = np.zeros(max(hg.n_adj, 1), dtype=np.int32)
    nadj, md = C.c_int64(), C.c_int32()
    _check(lib().pm_halve(hg.n, hg.n_adj, _ptr(hg.rowptr), _ptr(hg.colidx), _ptr(rp), _ptr(ci), C.byref(nadj),
                          C.byref(md)))
    return rp, ci[:nadj.value].copy(), md.value


def gen_chung_lu(n: int, n_edges: int, gamma: float = 2.1, i0: float = 10.0, max_w: float = 5000.0,
                 seed: int = 1) -> HostGraph:
    """Seeded Chung-Lu power-law graph (sorted, deduplicated, no self-loops)."""
    rp, ci, nadj, md = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int32()
    _check(lib().pm_gen_chung_lu(n, n_edges, gamma, i0, max_w, seed, C.byref(rp), C.byref(ci),
                                 C.byref(nadj), C.byref(md)))
    return HostGraph(_take(rp, n + 1, np.uint64), _take(ci, nadj.value, np.int32))


def gen_rmat(n: int, n_edges: int, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 2, device: Optional[int] = None) -> HostGraph:
    """Seeded R-MAT graph (ids >= n rejected; sorted, deduplicated, no self-loops).
    device: compute it on that GPU (same arrays), for graphs too large to sort
    on the host quickly."""
    rp, ci, nadj, md = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int32()
    if device is not None:
        _check(lib().pm_gen_rmat_device(n, n_edges, a, b, c, seed, device, C.byref(rp), C.byref(ci),
                                        C.byref(nadj), C.byref(md)))
    else:
        _check(lib().pm_gen_rmat(n, n_edges, a, b, c, seed, C.byref(rp), C.byref(ci), C.byref(nadj),
                                 C.byref(md)))
    return HostGraph(_take(rp, n + 1, np.uint64), _take(ci, nadj.value, np.int32))


def gen_labels(n: int, n_labels: int, seed: int) -> np.ndarray:
    lb = C.c_void_p()
    _check(lib().pm_gen_labels(n, n_labels, seed, C.byref(lb)))
    return _take(lb, n, np.uint32)


# ---------------------------------------------------------------- patterns

class PatternPreprocessor:
    """A compiled pattern plan (reference src/pattern.h:48-58)."""

    def __init__(self, path: Optional[str] = None, *, text: Optional[str] = None, labeled: bool = True):
        h = C.c_void_p()
        if text is not None:
            _check(lib().pm_plan_compile_text(text.encode(), int(labeled), C.byref(h)))
        elif path is not None:
            _check(lib().pm_plan_compile(path.encode(), int(labeled), C.byref(h)))
        else:
            raise ValueError("give a .g path or text=")
        self._h = h
        self.path = path
        self.labeled = labeled

    def describe(self) -> dict:
        d = PlanDesc()
        _check(lib().pm_plan_describe(self._h, C.byref(d)))
        n, ns = d.nnodes, d.nslots
        return {
            "labeled": d.labeled, "nnodes": n, "multiplicity": d.multiplicity, "nslots": ns,
            "level_begin": list(d.level_begin)[:n], "degree": list(d.degree)[:n],
            "vertex_label": list(d.vertex_label)[:n], "partial": list(d.partial)[:ns],
            "slot_labels": [0] + list(d.slot_labels)[1:ns], "set_ops": [0] + list(d.set_ops)[1:ns],
        }

    @property
    def PatternMultiplicity(self) -> int:  # noqa: N802 -- reference spelling
        return self.describe()["multiplicity"]

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().pm_plan_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- device graph

class GraphPreprocessor:
    """A CSR graph placed on the device (reference src/graph.h:34-41, 169-208).

    ``GraphPreprocessor(prefix)`` reads the reference's file layout;
    ``GraphPreprocessor.from_host(HostGraph)`` places in-memory arrays.
    """

    def __init__(self, prefix: Optional[str] = None, *, labeled: bool = True, device: int = 0,
                 paged: bool = False, frame_pool_bytes: int = 4 << 30, page_bytes: int = 64 << 10,
                 static_pool_bytes: int = 0,
                 _handle=None):
        self._h = None
        if _handle is not None:
            self._h = _handle
            return
        o = self._opts(labeled, device, paged, frame_pool_bytes, page_bytes, static_pool_bytes)
        h = C.c_void_p()
        _check(lib().pm_graph_open(prefix.encode(), C.byref(o), C.byref(h)))
        self._h = h

    @staticmethod
    def _opts(labeled, device, paged, frame_pool_bytes, page_bytes, static_pool_bytes=0) -> GraphOpts:
        o = GraphOpts()
        lib().pm_graph_opts_default(C.byref(o))
        o.labeled = int(labeled)
        o.device = device
        o.residency = PM_RESIDENT_PAGED if paged else PM_RESIDENT_HBM
        o.frame_pool_bytes = frame_pool_bytes
        o.page_bytes = page_bytes
        o.static_pool_bytes = static_pool_bytes
        return o

    @classmethod
    def from_host(cls, hg: HostGraph, *, labeled: bool = False, device: int = 0, paged: bool = False,
                  frame_pool_bytes: int = 4 << 30, page_bytes: int = 64 << 10,
                  static_pool_bytes: int = 0) -> "GraphPreprocessor":
        o = cls._opts(labeled, device, paged, frame_pool_bytes, page_bytes, static_pool_bytes)
        h = C.c_void_p()
        _check(lib().pm_graph_from_host(hg.n, hg.n_adj, _ptr(hg.rowptr), _ptr(hg.colidx),
                                        _ptr(hg.labels) if labeled else None, C.byref(o), C.byref(h)))
        return cls(_handle=h)

    @classmethod
    def from_device(cls, n: int, n_adj: int, max_degree: int, rowptr_ptr: int, colidx_ptr: int,
                    labels_ptr: Optional[int], device: int = 0) -> "GraphPreprocessor":
        h = C.c_void_p()
        _check(lib().pm_graph_from_device(n, n_adj, max_degree, C.c_void_p(rowptr_ptr), C.c_void_p(colidx_ptr),
                                          C.c_void_p(labels_ptr) if labels_ptr else None, device, C.byref(h)))
        return cls(_handle=h)

    @classmethod
    def from_paged_source(cls, hg: HostGraph, src_ptr: int, sorted_ptr: Optional[int] = None, *,
                          labeled: bool = False, device: int = 0, frame_pool_bytes: int = 4 << 30,
                          page_bytes: int = 64 << 10, static_pool_bytes: int = 0,
                          keep_alive=None) -> "GraphPreprocessor":
        """A paged graph whose pages come from a device-visible array (a
        partitioned range, pumatch_b200.parts) instead of pinned host memory.
        src_ptr: the paged layout (label-grouped when labeled); sorted_ptr:
        the id-sorted array (labeled graphs).  keep_alive: objects that must
        outlive the graph (the ranges the pointers come from)."""
        o = cls._opts(labeled, device, True, frame_pool_bytes, page_bytes, static_pool_bytes)
        h = C.c_void_p()
        _check(lib().pm_graph_from_paged_source(hg.n, hg.n_adj, _ptr(hg.rowptr),
                                                _ptr(hg.labels) if labeled else None, C.c_void_p(src_ptr),
                                                C.c_void_p(sorted_ptr) if sorted_ptr else None, C.byref(o),
                                                C.byref(h)))
        g = cls(_handle=h)
        g._keep = keep_alive
        return g

    def info(self) -> dict:
        gi = GraphInfo()
        _check(lib().pm_graph_get_info(self._h, C.byref(gi)))
        return {k: getattr(gi, k) for k, _ in gi._fields_}

    def set_resident_pages(self, pages) -> None:
        """Paged graphs: pages the frame pool starts each warm run with."""
        arr = np.ascontiguousarray(pages, dtype=np.int64)
        _check(lib().pm_graph_set_resident_pages(self._h, arr.ctypes.data_as(C.c_void_p), len(arr)))

    def close(self) -> None:
        if self._h:
            lib().pm_graph_close(self._h)
            self._h = None
        self._keep = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """Device, streams and reusable scratch (one per host thread)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().pm_ctx_create(device, C.byref(h)))
        self._h = h
        self.device = device

    def close(self) -> None:
        if self._h:
            lib().pm_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_ptr(self) -> int:
        """cudaStream_t of this context's launches (for torch.cuda.ExternalStream)."""
        return lib().pm_ctx_stream(self._h) or 0

    def count_roots(self, g: GraphPreprocessor, p: PatternPreprocessor) -> int:
        n = C.c_int64()
        _check(lib().pm_count_roots(self._h, g._h, p._h, C.byref(n)))
        return n.value

    def roots(self, g: GraphPreprocessor, p: PatternPreprocessor) -> np.ndarray:
        """The root list (reference Job[] order) as an (n, 2) int32 array."""
        n = self.count_roots(g, p)
        out = np.zeros((max(n, 1), 2), dtype=np.int32)
        got = C.c_int64()
        _check(lib().pm_debug_roots(self._h, g._h, p._h, _ptr(out), n, C.byref(got)))
        return out[:n]

    @staticmethod
    def _opts(**kw) -> RunOpts:
        """pm_run_opts from keyword arguments named after its fields (device
        pointers as <field>_ptr); an unknown name is a TypeError."""
        o = RunOpts()
        lib().pm_run_opts_default(C.byref(o))
        fields = {name for name, _ in RunOpts._fields_ if not name.endswith("_")}
        for k, v in kw.items():
            name = k[:-4] if k.endswith("_ptr") else k
            if name not in fields:
                raise TypeError(f"unknown run option {k!r}")
            if k.endswith("_ptr"):
                setattr(o, name, v or None)
            else:
                setattr(o, name, int(v))
        return o

    def prepare(self, g: GraphPreprocessor, patterns: Sequence[PatternPreprocessor], **kw) -> "Query":
        """A prepared batched launch replayed from a CUDA graph (pm_query_*)."""
        return Query(self, g, patterns, self._opts(**kw))

    def match(self, g: GraphPreprocessor, patterns: Sequence[PatternPreprocessor], **kw):
        """Runs all patterns in one launch; returns (counts list, stats dict).
        Keyword arguments are pm_run_opts fields (truncate, warps_per_block,
        chunk, split_level1, shard_rank/shard_count, root_begin/root_end,
        timeout_ms, cold_cache, high_occupancy, leaf_per_lane, lane_subtree_max, use_graph,
        own_arena_words, max_borrowed, prefetch_ahead, prefetch_chunks) and
        device pointers root_counts_ptr, root_cost_ptr, root_order_ptr,
        root_reads_ptr, prefetch_off_ptr, prefetch_pages_ptr, root_split_ptr."""
        o = self._opts(**kw)
        k = len(patterns)
        arr = (C.c_void_p * k)(*[p._h.value for p in patterns])
        counts = (C.c_uint64 * k)()
        st = Stats()
        _check(lib().pm_match(self._h, g._h, C.cast(arr, _PP), k, C.byref(o), counts, C.byref(st)))
        return [int(x) for x in counts], st.as_dict()


class Query:
    """pm_query_prepare / pm_query_run / pm_query_free."""

    def __init__(self, ctx: Context, g: GraphPreprocessor, patterns: Sequence[PatternPreprocessor], o: RunOpts):
        self._keep = (ctx, g, list(patterns))
        k = len(patterns)
        arr = (C.c_void_p * k)(*[p._h.value for p in patterns])
        h = C.c_void_p()
        _check(lib().pm_query_prepare(ctx._h, g._h, C.cast(arr, _PP), k, C.byref(o), C.byref(h)))
        self._h = h
        self.k = k

    def run(self):
        counts = (C.c_uint64 * self.k)()
        st = Stats()
        _check(lib().pm_query_run(self._h, counts, C.byref(st)))
        return [int(x) for x in counts], st.as_dict()

    def close(self) -> None:
        if self._h:
            lib().pm_query_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def match(g: GraphPreprocessor, patterns, ctx: Optional[Context] = None, **kw):
    """Counts every pattern in one persistent launch (reference test.cu:171-198)."""
    own = ctx is None
    ctx = ctx or Context(0)
    try:
        pats = patterns if isinstance(patterns, (list, tuple)) else [patterns]
        return ctx.match(g, pats, **kw)
    finally:
        if own:
            ctx.close()


__all__ = [
    "PmError", "HostGraph", "GraphPreprocessor", "PatternPreprocessor", "Context", "Query", "match",
    "gen_chung_lu", "gen_rmat", "gen_labels", "convert_snap", "lib", "LIB_PATH", "CLI_PATH", "SIGNATURES",
]
