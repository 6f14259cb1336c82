"""ctypes wrapper of liboracle.so -- TEST INFRASTRUCTURE ONLY.

The CPU oracle (pm_oracle.c) is the checker for the CUDA path.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg load it; the product
package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
MAX_PAT, MAX_SLOTS = 7, 15


class OrcPlan(C.Structure):
    _fields_ = [("nnodes", C.c_int), ("nslots", C.c_int), ("multiplicity", C.c_int), ("labeled", C.c_int),
                ("level_begin", C.c_int * (MAX_PAT + 1)), ("degree", C.c_int * MAX_PAT),
                ("vertex_label", C.c_int * MAX_PAT), ("slot_labels", C.c_uint32 * MAX_SLOTS),
                ("partial", C.c_uint32 * MAX_SLOTS), ("set_ops", C.c_uint8 * MAX_SLOTS)]

    def as_dict(self) -> dict:
        n, ns = self.nnodes, self.nslots
        return {
            "labeled": self.labeled, "nnodes": n, "multiplicity": self.multiplicity, "nslots": ns,
            "level_begin": list(self.level_begin)[:n], "degree": list(self.degree)[:n],
            "vertex_label": list(self.vertex_label)[:n], "partial": list(self.partial)[:ns],
            "slot_labels": [0] + list(self.slot_labels)[1:ns], "set_ops": [0] + list(self.set_ops)[1:ns],
        }


class OrcGraph(C.Structure):
    _fields_ = [("n", C.c_int64), ("n_adj", C.c_int64), ("rowptr", C.c_void_p), ("colidx", C.c_void_p),
                ("labels", C.c_void_p)]


class OrcStats(C.Structure):
    _fields_ = [("set_ops", C.c_uint64), ("alg_bytes", C.c_uint64), ("roots", C.c_uint64)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
                os.path.join(HERE, "pm_oracle.c")):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_plan_compile_text.argtypes = [C.c_char_p, C.c_int, C.POINTER(OrcPlan)]
        L.orc_plan_compile_text.restype = C.c_int
        L.orc_roots.argtypes = [C.POINTER(OrcGraph), C.POINTER(OrcPlan), C.c_void_p, C.c_int64]
        L.orc_roots.restype = C.c_int64
        L.orc_count.argtypes = [C.POINTER(OrcGraph), C.POINTER(OrcPlan), C.c_void_p, C.c_int64, C.c_int64,
                                C.c_int, C.c_void_p, C.POINTER(OrcStats)]
        L.orc_count.restype = C.c_uint64
        L.orc_count_mt.argtypes = [C.POINTER(OrcGraph), C.POINTER(OrcPlan), C.c_void_p, C.c_int64, C.c_int64,
                                   C.c_int, C.c_int, C.POINTER(OrcStats)]
        L.orc_count_mt.restype = C.c_uint64
        L.orc_estimate.argtypes = [C.POINTER(OrcGraph), C.POINTER(OrcPlan), C.c_void_p, C.c_int64, C.c_int,
                                   C.c_uint64, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double)]
        L.orc_estimate.restype = None
        L.orc_count_split.argtypes = [C.POINTER(OrcGraph), C.POINTER(OrcPlan), C.c_void_p, C.c_int64, C.c_int,
                                      C.c_int, C.c_double, C.c_uint64, C.c_void_p, C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int64), C.POINTER(OrcStats)]
        L.orc_count_split.restype = C.c_uint64
        for name in ("orc_gen_chung_lu", "orc_gen_rmat"):
            f = getattr(L, name)
            f.argtypes = [C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                          C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]
            f.restype = C.c_int
        L.orc_gen_labels.argtypes = [C.c_int64, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]
        L.orc_gen_labels.restype = C.c_int
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_free.restype = None
        _lib = L
    return _lib


def plan(text: str, labeled: bool) -> OrcPlan:
    p = OrcPlan()
    rc = lib().orc_plan_compile_text(text.encode(), int(labeled), C.byref(p))
    if rc != 0:
        raise ValueError(f"oracle plan compile failed ({rc})")
    return p


class Graph:
    """Keeps numpy arrays alive behind an OrcGraph view."""

    def __init__(self, rowptr: np.ndarray, colidx: np.ndarray, labels: Optional[np.ndarray]):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
        self.colidx = np.ascontiguousarray(colidx, dtype=np.int32)
        self.labels = None if labels is None else np.ascontiguousarray(labels, dtype=np.uint32)
        self.g = OrcGraph(len(self.rowptr) - 1, len(self.colidx), self.rowptr.ctypes.data,
                          self.colidx.ctypes.data, None if self.labels is None else self.labels.ctypes.data)


def roots(g: Graph, p: OrcPlan) -> np.ndarray:
    n = lib().orc_roots(C.byref(g.g), C.byref(p), None, 0)
    out = np.zeros((max(n, 1), 2), dtype=np.int32)
    lib().orc_roots(C.byref(g.g), C.byref(p), out.ctypes.data, n)
    return out[:n]


def count(g: Graph, p: OrcPlan, rts: np.ndarray, begin: int = 0, end: Optional[int] = None,
          truncate: int = 0, per_root: bool = False, threads: int = 1):
    """Raw DFS count over roots [begin, end) (not multiplied by |Aut|).
    Returns (count, stats dict[, per-root counts])."""
    rts = np.ascontiguousarray(rts, dtype=np.int32)
    end = len(rts) if end is None else end
    st = OrcStats()
    if threads > 1 and not per_root:
        c = lib().orc_count_mt(C.byref(g.g), C.byref(p), rts.ctypes.data, begin, end, truncate, threads,
                               C.byref(st))
        return int(c), {"set_ops": st.set_ops, "alg_bytes": st.alg_bytes, "roots": st.roots}
    pr = np.zeros(max(end - begin, 1), dtype=np.uint64) if per_root else None
    c = lib().orc_count(C.byref(g.g), C.byref(p), rts.ctypes.data, begin, end, truncate,
                        None if pr is None else pr.ctypes.data, C.byref(st))
    res = (int(c), {"set_ops": st.set_ops, "alg_bytes": st.alg_bytes, "roots": st.roots})
    return res + ((pr[: end - begin],) if per_root else ())


def total(g: Graph, text: str, labeled: bool, truncate: int = 0, threads: int = 1) -> int:
    """Final count as the reference prints it (x |Aut| when unlabeled, test.cu:198)."""
    p = plan(text, labeled)
    r = roots(g, p)
    c, _ = count(g, p, r, truncate=truncate, threads=threads)
    return c if labeled else c * p.multiplicity


def count_split(g: Graph, p: OrcPlan, rts: np.ndarray, threads: int = 1, time_limit_s: float = 0.0,
                shuffle_seed: int = 0, truncate: int = 0):
    """Raw per-root counts of the roots in `rts`, each root's DFS divided over
    `threads` at the candidates of level 1 (pieces in a seeded shuffled order
    when shuffle_seed != 0).  With time_limit_s > 0 the run stops at the limit,
    also inside a piece: the counts are then the matches found by then.
    Returns (total, per_root, pieces_finished, pieces_total, stats)."""
    rts = np.ascontiguousarray(rts, dtype=np.int32)
    pr = np.zeros(max(len(rts), 1), dtype=np.uint64)
    done, tot = C.c_int64(), C.c_int64()
    st = OrcStats()
    c = lib().orc_count_split(C.byref(g.g), C.byref(p), rts.ctypes.data, len(rts), truncate, threads,
                              float(time_limit_s), shuffle_seed, pr.ctypes.data, C.byref(done), C.byref(tot),
                              C.byref(st))
    return int(c), pr[:len(rts)], done.value, tot.value, {"set_ops": st.set_ops, "alg_bytes": st.alg_bytes,
                                                          "roots": st.roots}


def _take(ptr: C.c_void_p, n: int, dtype) -> np.ndarray:
    if n == 0:
        lib().orc_free(ptr)
        return np.zeros(0, dtype=dtype)
    buf = (C.c_char * (n * np.dtype(dtype).itemsize)).from_address(ptr.value)
    out = np.frombuffer(buf, dtype=dtype).copy()
    lib().orc_free(ptr)
    return out


def gen_chung_lu(n: int, m: int, gamma: float, i0: float, max_w: float, seed: int):
    """(rowptr, colidx) of the seeded Chung-Lu graph (the product generator's definition)."""
    rp, ci, nadj = C.c_void_p(), C.c_void_p(), C.c_int64()
    if lib().orc_gen_chung_lu(n, m, gamma, i0, max_w, seed, C.byref(rp), C.byref(ci), C.byref(nadj)) != 0:
        raise ValueError("orc_gen_chung_lu failed")
    return _take(rp, n + 1, np.uint64), _take(ci, nadj.value, np.int32)


def gen_rmat(n: int, m: int, a: float, b: float, c: float, seed: int):
    """(rowptr, colidx) of the seeded R-MAT graph (the product generator's definition)."""
    rp, ci, nadj = C.c_void_p(), C.c_void_p(), C.c_int64()
    if lib().orc_gen_rmat(n, m, a, b, c, seed, C.byref(rp), C.byref(ci), C.byref(nadj)) != 0:
        raise ValueError("orc_gen_rmat failed")
    return _take(rp, n + 1, np.uint64), _take(ci, nadj.value, np.int32)


def gen_labels(n: int, n_labels: int, seed: int) -> np.ndarray:
    lb = C.c_void_p()
    if lib().orc_gen_labels(n, n_labels, seed, C.byref(lb)) != 0:
        raise ValueError("orc_gen_labels failed")
    return _take(lb, n, np.uint32)


def estimate(g: Graph, p: OrcPlan, rts: np.ndarray, probes: int = 2000, seed: int = 7):
    so, by, ct = C.c_double(), C.c_double(), C.c_double()
    rts = np.ascontiguousarray(rts, dtype=np.int32)
    lib().orc_estimate(C.byref(g.g), C.byref(p), rts.ctypes.data, len(rts), probes, seed, C.byref(so),
                       C.byref(by), C.byref(ct))
    return so.value, by.value, ct.value
