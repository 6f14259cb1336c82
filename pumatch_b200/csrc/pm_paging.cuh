// pm_paging.cuh -- device side of the adjacency page cache (paged residency).
//
// Replaces the reference's GPU-side LRU package buffer and its fault
// handshake (src/buffer.cu:197-261 get_neighbors_from_buffer, :581-628
// lruAccess_bucket, :800-871 update_buffer, :1859-1936 add_vertex_block) and
// the missing-branch tree (src/missing_tree.cu) with a design in which no
// device thread ever waits for the host:
//   * the adjacency array stays in pinned, mapped host memory; a page is a
//     fixed power-of-two range of it; a device frame pool caches pages;
//   * page_frame[page] is the device-resident page table (frame index, or
//     ABSENT / LOADING / EVICTING);
//   * a warp that finds a list resident pins its frame (one acquire add on
//     the frame's (page, pins) word, no fence), re-checks the mapping and
//     reads the frame; a list spanning several pages is gathered into the
//     warp's arena when all its pages are resident;
//   * otherwise the warp reads the list straight from host memory over the
//     link (so every branch finishes where it started -- nothing is parked or
//     lost, counts stay exact) and, for an absent page, claims a victim frame
//     with a bounded CLOCK sweep (skipping pinned and referenced frames) and
//     posts (page, frame) to a ring in mapped host memory;
//   * a warp that misses on a list within one page copies that page into
//     the claimed frame itself (16-byte loads from the mapped array) and
//     publishes the entry after a fence, and so does a warp for up to two
//     pages its lanes missed on in a last-level batch; other loads (lists
//     over several pages, prefetch lists, and every load when the run asks
//     for host copies) are posted to a host service thread, which copies
//     posted pages into their frames with
//     cudaMemcpyAsync on a side stream and publishes each page by copying its
//     page-table entry after the data (same stream, so the entry lands
//     after the page).
#pragma once

#include "pm_device.cuh"

namespace pm {

enum : int32_t { PAGE_EVICTING = -3 };

struct PageCounters {
  unsigned long long hits, misses, zc_bytes, requests, evictions, dropped, dev_loads, dev_bytes;
};

__device__ __forceinline__ int32_t ld_vol(const int32_t* p) { return *(const volatile int32_t*)p; }

// Reserves one ring slot if the host has room; returns the slot or ~0ull.
__device__ __forceinline__ unsigned long long ring_reserve(const DPaging& pg) {
  for (int t = 0; t < 8; t++) {
    const unsigned long long head = *(volatile unsigned long long*)pg.ring_head;
    const unsigned long long done = *(volatile unsigned long long*)pg.host_tail;
    if (head - done >= (unsigned long long)pg.ring_mask) return ~0ull;  // full
    if (atomicCAS(pg.ring_head, head, head + 1) == head) return head;
  }
  return ~0ull;
}

__device__ __forceinline__ void ring_post(const DPaging& pg, unsigned long long slot, int32_t page, int32_t frame) {
  pg.ring[slot & pg.ring_mask] = make_int2(page, frame);
  __threadfence_system();
  *(volatile unsigned long long*)&pg.ring_seq[slot & pg.ring_mask] = slot + 1;
}

// Frame state words: (page << 32) | pins.
__device__ __forceinline__ int32_t fs_page(unsigned long long s) { return (int32_t)(s >> 32); }
__device__ __forceinline__ uint32_t fs_pins(unsigned long long s) { return (uint32_t)s; }

__device__ __forceinline__ unsigned long long ld_vol64(const unsigned long long* p) {
  return *(const volatile unsigned long long*)p;
}

// Atomic add on a frame state with acquire (pin) or release (unpin)
// semantics at GPU scope.
__device__ __forceinline__ unsigned long long fs_add_acquire(unsigned long long* p, unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.add.acquire.gpu.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ void fs_add_release(unsigned long long* p, unsigned long long v) {
  asm volatile("red.add.release.gpu.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// CAS with release semantics: what this thread wrote before (the new page's
// LOADING entry) is visible to a reader that sees the new tag.
__device__ __forceinline__ unsigned long long fs_cas_release(unsigned long long* p, unsigned long long cmp,
                                                             unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.cas.release.gpu.b64 %0, [%1], %2, %3;" : "=l"(old) : "l"(p), "l"(cmp), "l"(v) : "memory");
  return old;
}

// One thread.  Claims a frame for page p if p is absent: the entry goes
// ABSENT -> LOADING, and a never-used frame or a CLOCK victim is tagged p.
// Returns the frame, or -1 when p is not absent or no frame is free (then
// the entry is ABSENT again).  The caller fills the frame and publishes it.
//
// Eviction of page q from frame h: the entry page_frame[q] goes h ->
// EVICTING, then the frame's state goes (q, 0 pins) -> (p, 0 pins) by CAS,
// so a reader that pinned h first makes the CAS fail (the entry is put back);
// a reader that pins afterwards sees tag p and backs off.  The frame is then
// LOADING for p (page_frame[p] = LOADING) until it is published.
static __device__ int32_t claim_frame(const DPaging& pg, int32_t p, PageCounters& pc) {
  if (atomicCAS(&pg.page_frame[p], PAGE_ABSENT, PAGE_LOADING) != PAGE_ABSENT) return -1;  // someone else has it
  const unsigned long long tag_p = (unsigned long long)(uint32_t)p << 32;
  int32_t f = -1;
  const unsigned long long k = atomicAdd(pg.next_free, 1ull);
  const int64_t n_dyn = pg.n_frames - pg.n_static;  // evictable frames
  if (k < (unsigned long long)pg.n_frames) {
    // a never-used frame: no page entry names it, so no reader can pin it
    f = (int32_t)k;
    atomicExch(&pg.frame_state[f], tag_p);
  } else if (n_dyn > 0) {
    const int sweep = (int)min((int64_t)4096, 2 * n_dyn + 8);  // bounded CLOCK sweep
    for (int t = 0; t < sweep && f < 0; t++) {
      const int32_t h = pg.n_static + (int32_t)(atomicAdd(pg.clock_hand, 1ull) % (unsigned long long)n_dyn);
      if (pg.frame_ref[h]) { pg.frame_ref[h] = 0; continue; }
      const unsigned long long st = ld_vol64(&pg.frame_state[h]);
      if (fs_pins(st) != 0) continue;
      const int32_t q = fs_page(st);
      if (q < 0) continue;
      if (atomicCAS(&pg.page_frame[q], h, PAGE_EVICTING) != h) continue;  // loading, or moved
      if (fs_cas_release(&pg.frame_state[h], st, tag_p) != st) {  // a reader pinned it meanwhile
        atomicExch(&pg.page_frame[q], h);
        continue;
      }
      atomicExch(&pg.page_frame[q], PAGE_ABSENT);
      f = h;
      pc.evictions++;
    }
  }
  if (f < 0) {  // every frame busy: stay on the host-read path
    atomicExch(&pg.page_frame[p], PAGE_ABSENT);
    pc.dropped++;
  }
  return f;
}

// One thread (lane 0 of a warp, or a lane for its own list).  Starts
// loading page p if it is absent: reserve a ring slot, claim a frame, post
// (page, frame) for the host service thread.  Never waits for the host.
static __device__ void request_page(const DPaging& pg, int32_t p, PageCounters& pc) {
  if (pg.n_static >= pg.n_frames) return;  // no evictable frame to load into
  if (ld_vol(&pg.page_frame[p]) != PAGE_ABSENT) return;
  const unsigned long long slot = ring_reserve(pg);
  if (slot == ~0ull) { pc.dropped++; return; }
  const int32_t f = claim_frame(pg, p, pc);
  if (f < 0) {
    ring_post(pg, slot, -1, -1);
    return;
  }
  ring_post(pg, slot, p, f);
  pc.requests++;
}

// Whole warp, p uniform.  Loads absent page p into a frame itself: claim a
// frame, copy the page from the mapped host array (16-byte loads, eight in
// flight per lane: 4 KB per round trip for the warp), then publish the
// entry after a fence.  Returns the frame, or -1 (p not absent, or no frame).
// The copy is bounded work; nothing waits on the host or on other warps.
static __device__ __noinline__ int32_t warp_load_page(const DPaging& pg, int32_t p, PageCounters& pc) {
  const int lane = threadIdx.x & 31;
  int32_t f = -1;
  if (lane == 0 && pg.n_static < pg.n_frames && ld_vol(&pg.page_frame[p]) == PAGE_ABSENT) f = claim_frame(pg, p, pc);
  f = __shfl_sync(0xffffffffu, f, 0);
  if (f < 0) return -1;
  const int sh = pg.page_shift;
  const int64_t first = (int64_t)p << sh;
  const int n = (int)min((int64_t)1 << sh, pg.n_ints - first);
  const int32_t* hsrc = pg.host_colidx + first;  // 16-byte aligned: pages start at multiples of 1,024 ints
  int32_t* fdst = pg.frames + ((uint64_t)f << sh);
  const int4* src = reinterpret_cast<const int4*>(hsrc);
  int4* dst = reinterpret_cast<int4*>(fdst);
  const int nv = n >> 2;
  for (int base = 0; base < nv; base += 256) {
    int4 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = base + q * 32 + lane;
      v[q] = i < nv ? src[i] : make_int4(0, 0, 0, 0);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = base + q * 32 + lane;
      if (i < nv) __stcg(dst + i, v[q]);
    }
  }
  for (int i = 4 * nv + lane; i < n; i += 32) __stcg(fdst + i, hsrc[i]);
  __threadfence();  // each lane's stores before the publish below
  __syncwarp();
  if (lane == 0) {
    pg.frame_ref[f] = 1;  // not the first victim of the next sweep
    atomicExch(&pg.page_frame[p], f);
    pc.dev_loads++;
    pc.dev_bytes += 4ull * (unsigned long long)n;
  }
  __syncwarp();
  return f;
}

// Pins the frame holding page p if it is resident; returns the frame or -1.
// A static frame is returned as is: its entry never changes during a run.
// The pin is one acquire add on the frame's state word; the tag it returns
// says whether the frame still holds p.  The entry is read once more after
// the pin: the frame may have been given back to p for a new load in between
// (then the entry reads LOADING until the host publishes it again).
__device__ __forceinline__ int32_t try_pin(const DPaging& pg, int32_t p) {
  const int32_t f = ld_vol(&pg.page_frame[p]);
  if (f < 0) return -1;
  if (f < pg.n_static) return f;
  const unsigned long long st = fs_add_acquire(&pg.frame_state[f], 1ull);
  if (fs_page(st) != p || ld_vol(&pg.page_frame[p]) != f) {
    fs_add_release(&pg.frame_state[f], ~0ull);  // -1
    return -1;
  }
  if (!pg.frame_ref[f]) pg.frame_ref[f] = 1;
  return f;
}

__device__ __forceinline__ void unpin_frame(const DPaging& pg, int32_t f) {
  if (f >= pg.n_static) fs_add_release(&pg.frame_state[f], ~0ull);
}

// Frame of page p0 when pages p0..p1 all sit in consecutive static frames (a
// list over them can be read in place), else -1.
__device__ __forceinline__ int32_t static_run(const DPaging& pg, int32_t p0, int32_t p1) {
  const int32_t f0 = ld_vol(&pg.page_frame[p0]);
  if (f0 < 0 || f0 + (p1 - p0) >= pg.n_static) return -1;
  for (int32_t k = p0 + 1; k <= p1; k++)
    if (ld_vol(&pg.page_frame[k]) != f0 + (k - p0)) return -1;
  return f0;
}

struct ListRef {
  const int32_t* p;
  int len;
  int32_t pinned;  // frame to unpin after use, or -1
  bool cg;         // an evictable frame: read through L2 only (refilled during the launch)
};

// Copies a list out of mapped host memory into gather (whole warp), eight
// reads in flight per lane (one round trip per 256 entries), so that the set
// operation runs on device memory.
__device__ __forceinline__ ListRef host_list_copy(const int32_t* src, int len, int32_t* gather) {
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < len; base += 256) {
    int v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = base + q * 32 + lane;
      v[q] = i < len ? src[i] : 0;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = base + q * 32 + lane;
      if (i < len) gather[i] = v[q];
    }
  }
  __syncwarp();
  return ListRef{gather, len, -1};
}

// Most pages one list may span and still be gathered from frames; longer
// lists are read from host memory.
#define PM_MAX_LIST_PAGES 64

// Resolves the adjacency list [b, b+len) of colidx for the whole warp.
// gather: arena space for a copied list (>= len words); pins: per-warp
// shared scratch of PM_MAX_LIST_PAGES frame indices.  Frames are remembered
// from the pin, never re-read from the table (an evictor can hold an entry at
// PAGE_EVICTING for a moment even while the frame is pinned).
static __device__ __noinline__ ListRef paged_list(const DPaging& pg, uint64_t b, int len, int32_t* gather, int32_t* pins,
                                     PageCounters& pc) {
  const int lane = threadIdx.x & 31;
  if (len == 0) return ListRef{pg.host_colidx + b, 0, -1};
  const int sh = pg.page_shift;
  const int32_t p0 = (int32_t)(b >> sh);
  const int32_t p1 = (int32_t)((b + (uint64_t)len - 1) >> sh);
  const bool can_load = pg.dev_copy && pg.n_static < pg.n_frames;
  int mode = 1;  // 0 frame, 1 host read, 2 gathered, 3 several pages to pin
  int32_t f0 = -1;
  int32_t load = -1;  // a one-page list on an absent page: the warp loads the page
  if (lane == 0) {
    if (p0 == p1) {
      f0 = try_pin(pg, p0);
      if (f0 >= 0) mode = 0;
      else if (can_load && ld_vol(&pg.page_frame[p0]) == PAGE_ABSENT) load = p0;
      else request_page(pg, p0, pc);
    } else if ((f0 = static_run(pg, p0, p1)) >= 0) {
      mode = 0;  // contiguous in the static frames: read in place, no pins
    } else if (p1 - p0 < PM_MAX_LIST_PAGES) {
      mode = 3;
    }
  }
  mode = __shfl_sync(0xffffffffu, mode, 0);
  f0 = __shfl_sync(0xffffffffu, f0, 0);
  load = __shfl_sync(0xffffffffu, load, 0);
  bool hit = mode == 0;
  if (load >= 0 && warp_load_page(pg, load, pc) >= 0) {
    if (lane == 0) f0 = try_pin(pg, load);  // fails only if evicted at once
    f0 = __shfl_sync(0xffffffffu, f0, 0);
    if (f0 >= 0) mode = 0;
  }
  if (mode == 3) {
    // several pages: the lanes pin them (page p0 + lane, p0 + lane + 32);
    // when some are absent the warp loads them one by one and pins again
    // (only when a quarter of the evictable frames holds them all; else a
    // list's own loads would evict each other)
    const bool load_all = can_load && 4ll * (p1 - p0 + 1) <= pg.n_frames - pg.n_static;
    bool all = false;
    for (int attempt = 0; attempt < 2 && !all; attempt++) {
      if (attempt == 1) {
        if (!load_all) {
          if (lane == 0)
            for (int32_t j = p0, posted = 0; j <= p1 && posted < 4; j++)
              if (ld_vol(&pg.page_frame[j]) == PAGE_ABSENT) { request_page(pg, j, pc); posted++; }
          break;
        }
        for (int32_t k = p0; k <= p1; k++) warp_load_page(pg, k, pc);
      }
      bool ok = true;
      for (int32_t k = p0 + lane; k <= p1; k += 32) {
        const int32_t f = try_pin(pg, k);
        pins[k - p0] = f;
        ok = ok && f >= 0;
      }
      all = __all_sync(0xffffffffu, ok);
      if (!all)
        for (int32_t k = p0 + lane; k <= p1; k += 32)
          if (pins[k - p0] >= 0) unpin_frame(pg, pins[k - p0]);
      if (attempt == 0) hit = all;
    }
    __syncwarp();
    mode = all ? 2 : 1;
  }
  if (lane == 0) {
    if (hit) pc.hits++;
    else pc.misses++;
  }
  if (mode == 0) {
    const uint64_t off = b & ((1ull << sh) - 1);
    return ListRef{pg.frames + ((uint64_t)f0 << sh) + off, len, f0, f0 >= pg.n_static};
  }
  if (mode == 1) {
    if (lane == 0) pc.zc_bytes += 4ull * (unsigned long long)len;
    return host_list_copy(pg.host_colidx + b, len, gather);
  }
  // gather the pinned pages into the arena, then unpin them
  const uint64_t e = b + (uint64_t)len;
  for (int32_t k = p0; k <= p1; k++) {
    const int32_t f = pins[k - p0];
    const uint64_t s0 = max(b, (uint64_t)k << sh), s1 = min(e, ((uint64_t)k + 1) << sh);
    const int32_t* src = pg.frames + ((uint64_t)f << sh) + (s0 - ((uint64_t)k << sh));
    int32_t* dst = gather + (s0 - b);
    for (uint64_t i = lane; i < s1 - s0; i += 32) dst[i] = __ldcg(src + i);
  }
  __syncwarp();
  for (int32_t k = p0 + lane; k <= p1; k += 32) unpin_frame(pg, pins[k - p0]);
  __syncwarp();
  return ListRef{gather, len, -1};
}

__device__ __forceinline__ void unpin(const DPaging& pg, const ListRef& r) {
  if (r.pinned >= 0 && (threadIdx.x & 31) == 0) unpin_frame(pg, r.pinned);
}

}  // namespace pm
