"""Partitioned residency: the adjacency array held once across the GPUs of a node.

The reference pages the edges beyond its device partition from host memory
(test.cu:22-43, src/buffer.cu:986-1060), and its multi-node mode copies the
whole graph to every rank (test_mpi.cu:317-349).  Here the array is cut into
slices of whole pages; slice p lives in the HBM of GPU p only, and every GPU
maps all slices into one device address range (libpumatch_b200's pm_parts_*
calls over the CUDA virtual memory API).  A paged graph placed with
GraphPreprocessor.from_paged_source takes its pages from that range, so a page
that misses in a GPU's frame pool is copied from its owner's HBM over NVLink,
not from host memory.  Labeled graphs need two such ranges: the label-grouped
layout the frames cache, and the id-sorted array the kernel reads whole lists
from.

place_local() builds the ranges in one process (its slices on one or more
devices: a single GPU with several slices stands in for several GPUs).
place_distributed() is the one-process-per-GPU form: each rank allocates and
fills its own slice, the ranks pass their slices to each other as POSIX file
descriptors over Unix sockets (exchange_fds), and each maps all of them.
owner_root_ranges() gives each rank the root edges whose first vertex's list
lies in its own slice (roots are in first-vertex order, so these are
contiguous ranges of root positions).
"""
from __future__ import annotations

import ctypes as C
import os
import socket
import struct
import threading
import time
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import GraphPreprocessor, HostGraph, _check, lib


def granularity(device: int = 0) -> int:
    """Allocation granularity of a slice on device (bytes)."""
    g = C.c_uint64()
    _check(lib().pm_parts_granularity(device, C.byref(g)))
    return int(g.value)


def slice_bounds(nbytes: int, n_parts: int, gran: int, page_bytes: int) -> Tuple[List[int], int]:
    """Byte offsets where the slices of an nbytes array start, and the range's
    padded size.  Boundaries fall on multiples of both the allocation
    granularity and the page size (powers of two: the larger of the two), so
    a page never straddles two slices; slices are equal but for the last.  An
    array too small for n_parts slices gets fewer."""
    if n_parts < 1 or nbytes < 0:
        raise ValueError("need n_parts >= 1 and nbytes >= 0")
    for x in (gran, page_bytes):
        if x <= 0 or x & (x - 1):
            raise ValueError("granularity and page size must be powers of two")
    align = max(gran, page_bytes)
    units = max(1, -(-nbytes // align))
    per = -(-units // n_parts)
    begins = [p * per * align for p in range(n_parts) if p * per < units]
    return begins, units * align


class Range:
    """A pm_parts range as one device sees it (slices at the given byte
    offsets, total bytes a multiple of the granularity)."""

    def __init__(self, device: int, begins: Sequence[int], total: int):
        arr = np.ascontiguousarray(begins, dtype=np.uint64)
        h = C.c_void_p()
        _check(lib().pm_parts_create(device, len(arr), arr.ctypes.data_as(C.c_void_p), int(total), C.byref(h)))
        self._h = h
        self.device = device
        self.begins = [int(b) for b in begins]
        self.total = int(total)

    def bounds(self, p: int) -> Tuple[int, int]:
        return self.begins[p], self.begins[p + 1] if p + 1 < len(self.begins) else self.total

    def alloc(self, p: int, owner_device: int) -> None:
        _check(lib().pm_parts_alloc(self._h, p, owner_device))

    def export(self, p: int) -> int:
        fd = C.c_int(-1)
        _check(lib().pm_parts_export(self._h, p, C.byref(fd)))
        return fd.value

    def import_(self, p: int, fd: int) -> None:
        _check(lib().pm_parts_import(self._h, p, fd))

    def map(self) -> None:
        _check(lib().pm_parts_map(self._h))

    @property
    def ptr(self) -> int:
        v = lib().pm_parts_ptr(self._h)
        if not v:
            raise RuntimeError("the range is not mapped")
        return int(v)

    def write(self, offset: int, data: np.ndarray) -> None:
        data = np.ascontiguousarray(data)
        _check(lib().pm_parts_write(self._h, int(offset), data.ctypes.data_as(C.c_void_p), data.nbytes))

    def fill_slice(self, p: int, array: np.ndarray) -> None:
        """Writes slice p's part of array (bytes beyond the array stay unwritten)."""
        b, e = self.bounds(p)
        raw = array.view(np.uint8)
        if b < raw.nbytes:
            self.write(b, raw[b:min(e, raw.nbytes)])

    def close(self) -> None:
        if self._h:
            lib().pm_parts_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def label_grouped(hg: HostGraph) -> np.ndarray:
    """The label-grouped layout a labeled paged graph caches (every list
    stably sorted by label), computed on the host."""
    if hg.labels is None:
        raise ValueError("an unlabeled graph has no label-grouped layout")
    out = np.empty(hg.n_adj, dtype=np.int32)
    lab = np.ascontiguousarray(hg.labels, dtype=np.uint32)
    _check(lib().pm_label_group_host(hg.n, hg.n_adj, hg.rowptr.ctypes.data_as(C.c_void_p),
                                     hg.colidx.ctypes.data_as(C.c_void_p), lab.ctypes.data_as(C.c_void_p),
                                     out.ctypes.data_as(C.c_void_p)))
    return out


def _arrays(hg: HostGraph, labeled: bool) -> List[np.ndarray]:
    """The arrays to partition: [paged layout] or [grouped layout, id-sorted]."""
    return [label_grouped(hg), hg.colidx] if labeled else [hg.colidx]


def place_local(hg: HostGraph, n_parts: int, *, device: int = 0, owners: Optional[Sequence[int]] = None,
                labeled: bool = False, frame_pool_bytes: int = 4 << 30, page_bytes: int = 64 << 10,
                static_pool_bytes: int = 0, export_import: bool = False) -> GraphPreprocessor:
    """A paged graph on `device` whose pages come from n_parts slices, slice p
    allocated on owners[p] (default: all on `device`).  export_import passes
    every slice through a file descriptor into a second range, the path
    another process takes, and places the graph on that one."""
    gran = granularity(device)
    begins, total = slice_bounds(4 * hg.n_adj, n_parts, gran, page_bytes)
    owners = list(owners) if owners is not None else [device] * len(begins)
    ranges = []
    try:
        for arr in _arrays(hg, labeled):
            r = Range(device, begins, total)
            ranges.append(r)
            for p in range(len(begins)):
                r.alloc(p, owners[p % len(owners)])
            if export_import:
                r2 = Range(device, begins, total)
                ranges.append(r2)
                for p in range(len(begins)):
                    fd = r.export(p)
                    try:
                        r2.import_(p, fd)
                    finally:
                        os.close(fd)
                r.map()
                for p in range(len(begins)):
                    r.fill_slice(p, arr)
                r2.map()
            else:
                r.map()
                for p in range(len(begins)):
                    r.fill_slice(p, arr)
        used = ranges[1::2] if export_import else ranges
        src, srt = used[0].ptr, (used[1].ptr if labeled else None)
        return GraphPreprocessor.from_paged_source(hg, src, srt, labeled=labeled, device=device,
                                                   frame_pool_bytes=frame_pool_bytes, page_bytes=page_bytes,
                                                   static_pool_bytes=static_pool_bytes, keep_alive=ranges)
    except BaseException:
        for r in ranges:
            r.close()
        raise


# --- one process per GPU -----------------------------------------------------

def _sock_name(job: str, rank: int) -> bytes:
    # Linux abstract namespace: no file to clean up, gone with the process
    return f"\0pumatch-parts-{job}-{rank}".encode()


def exchange_fds(job: str, rank: int, world: int, mine: Dict[int, int], timeout_s: float = 60.0) -> Dict[int, int]:
    """Sends this rank's file descriptors (key -> fd) to every other rank and
    returns theirs (key -> a new fd in this process), over Unix sockets in
    the abstract namespace named by job.  Keys must be distinct across ranks.
    The caller closes the descriptors it receives (and its own) when done."""
    if world == 1:
        return {}
    srv = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
    srv.bind(_sock_name(job, rank))
    srv.listen(world)
    srv.settimeout(timeout_s)
    got: Dict[int, int] = {}
    err: List[BaseException] = []

    def serve():
        try:
            for _ in range(world - 1):
                conn, _ = srv.accept()
                with conn:
                    conn.settimeout(timeout_s)
                    hdr = b""
                    fds: List[int] = []
                    while len(hdr) < 4:
                        msg, more, _, _ = socket.recv_fds(conn, 4 - len(hdr), 16)
                        if not msg:
                            raise ConnectionError("peer closed before its header")
                        hdr += msg
                        fds += more
                    (n,) = struct.unpack("<i", hdr)
                    body = b""
                    while len(body) < 8 * n:
                        msg, more, _, _ = socket.recv_fds(conn, 8 * n - len(body), 16)
                        if not msg:
                            raise ConnectionError("peer closed before its keys")
                        body += msg
                        fds += more
                    keys = struct.unpack(f"<{n}q", body)
                    if len(fds) != n:
                        raise ConnectionError(f"expected {n} descriptors, got {len(fds)}")
                    got.update(zip(keys, fds))
        except BaseException as e:  # noqa: BLE001 -- re-raised by the caller
            err.append(e)

    th = threading.Thread(target=serve, daemon=True)
    th.start()
    keys = list(mine)
    payload = struct.pack("<i", len(keys)) + struct.pack(f"<{len(keys)}q", *keys)
    deadline = time.monotonic() + timeout_s
    try:
        for q in range(world):
            if q == rank:
                continue
            while True:
                s = socket.socket(socket.AF_UNIX, socket.SOCK_STREAM)
                try:
                    s.connect(_sock_name(job, q))
                    break
                except (ConnectionRefusedError, FileNotFoundError):
                    s.close()
                    if time.monotonic() > deadline:
                        raise TimeoutError(f"rank {q} never listened")
                    time.sleep(0.01)
            with s:
                # header and keys in one message, with every descriptor attached
                if keys:
                    socket.send_fds(s, [payload], [mine[k] for k in keys])
                else:
                    s.sendall(payload)
        th.join(max(0.0, deadline - time.monotonic()) + 1.0)
        if th.is_alive():
            raise TimeoutError("peers did not send their descriptors in time")
        if err:
            raise err[0]
    finally:
        srv.close()
    return got


def place_distributed(hg: HostGraph, rank: int, world: int, *, job: str, device: int,
                      barrier: Callable[[], None], labeled: bool = False, frame_pool_bytes: int = 4 << 30,
                      page_bytes: int = 64 << 10, static_pool_bytes: int = 0) -> GraphPreprocessor:
    """The one-process-per-GPU placement: rank r holds slice r of each array
    in the HBM of `device`, imports the other ranks' slices and maps all of
    them.  barrier() must block until every rank has reached it (a
    torch.distributed barrier); it separates filling the slices from reading
    them.  Every rank computes the same slice bounds from the array size, the
    granularity and the page size."""
    gran = granularity(device)
    begins, total = slice_bounds(4 * hg.n_adj, world, gran, page_bytes)
    arrays = _arrays(hg, labeled)
    ranges = [Range(device, begins, total) for _ in arrays]
    try:
        mine = {}
        if rank < len(begins):
            for a, r in enumerate(ranges):
                r.alloc(rank, device)
                mine[a * world + rank] = r.export(rank)
        try:
            theirs = exchange_fds(job, rank, world, mine)
        finally:
            for fd in mine.values():
                os.close(fd)
        try:
            for key, fd in theirs.items():
                a, p = divmod(key, world)
                ranges[a].import_(p, fd)
        finally:
            for fd in theirs.values():
                os.close(fd)
        for r in ranges:
            r.map()
        if rank < len(begins):
            for arr, r in zip(arrays, ranges):
                r.fill_slice(rank, arr)
        barrier()  # every slice written before any rank reads the range
        return GraphPreprocessor.from_paged_source(hg, ranges[0].ptr, ranges[1].ptr if labeled else None,
                                                   labeled=labeled, device=device,
                                                   frame_pool_bytes=frame_pool_bytes, page_bytes=page_bytes,
                                                   static_pool_bytes=static_pool_bytes, keep_alive=ranges)
    except BaseException:
        for r in ranges:
            r.close()
        raise


def owner_root_ranges(rowptr: np.ndarray, roots: np.ndarray, begins: Sequence[int], total: int) -> List[Tuple[int, int]]:
    """Per slice, the root positions [b, e) whose first vertex's list starts
    in that slice (roots: int32 pairs in the reference's order, first vertex
    ascending).  Running its own range, a rank reads its roots' first lists
    from its own HBM."""
    starts = 4 * np.asarray(rowptr, dtype=np.uint64)[np.asarray(roots)[:, 0]]
    edges = np.asarray(list(begins)[1:] + [total], dtype=np.uint64)
    cut = np.searchsorted(starts, edges, side="left")
    out, b = [], 0
    for c in cut:
        out.append((b, int(c)))
        b = int(c)
    out[-1] = (out[-1][0], len(starts))
    return out
