// pm_device.cu -- device half of libpumatch_b200.so: graph placement, the GPU
// root filter, and the persistent DFS subgraph-enumeration kernel.
//
// Kernel design (sm_100a, 148 SMs):
//   * one persistent grid, sized to the SM count times the resident blocks
//     per SM; every warp runs its own depth-first search;
//   * work = root edges (v0, v1) of one or more plans, handed out in chunks
//     by 64-bit atomic cursors (one per plan, warps start on different plans
//     so a batch of patterns interleaves);
//   * a warp that still holds a candidate range (at any DFS level) when the
//     queue has run dry donates the upper half of its shallowest splittable
//     range, with the path prefix, to a global donation ring that idle warps
//     drain (replaces the reference's disabled stealing,
//     src/gpu_match.cu:21-148, 818-853);
//   * each level's candidate sets ("slots") are computed by a warp-cooperative
//     sorted-set operation -- 32 candidates per step, per-lane membership
//     search, __ballot_sync/__popc compaction -- and stored in a per-warp
//     arena in HBM sized to the plan's worst case, so nothing is truncated
//     (the reference caps every set at GRAPH_DEGREE=4096; that cap is kept
//     only as an explicit emulation switch);
//   * the last level is counted, never materialised: work-balanced across
//     the warp (leaf_flat), one candidate per lane (leaf_batch), or, for
//     clique-like plans, the last two levels one candidate per lane
//     (lane_subtree).
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "pm_common.h"
#include "pm_device.cuh"
#include "pm_paging.cuh"

namespace pm {
const Plan* plan_of(const pm_plan* h);
}
using namespace pm;

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(PM_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                  __LINE__);                                                             \
  } while (0)

static constexpr unsigned FULL = 0xffffffffu;

// =====================================================================
// Handles
// =====================================================================

// =====================================================================
// Device helpers
// =====================================================================

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Publication of a donated item: the donor's release store of the slot's
// sequence number orders its item writes before it; the taker's acquire load
// orders its item reads after it.
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

struct MatchArgs {
  const uint64_t* rowptr;
  const int32_t* colidx;        // HBM residency
  const uint8_t* labels;
  const int32_t* colidx_lab;    // label-grouped lists (labeled, HBM) or null
  const int32_t* lab_off;       // label group offsets (labeled, HBM or paged) or null
  const int32_t* host_sorted;   // labeled paged: the id-sorted lists in mapped host memory
  int32_t leaf_flat;            // last level: 0 one candidate per lane, 1 flat in lane-contiguous parts,
                                // 2 flat strided (leaf_flat)
  int32_t lane_subtree_max;     // lane_subtree when the parent set is at most this long; 0 = never
  int32_t nl1;
  int32_t pad1;
  int32_t n;
  int32_t nplans;
  int32_t T;
  int32_t chunk;
  int32_t shard_rank;
  int32_t shard_count;
  int32_t split_min;            // donate last-but-one-level ranges at least this long
  int32_t maxdeg;
  unsigned long long* cursors;  // [nplans]
  unsigned long long* counts;   // [nplans]
  unsigned long long* stats;    // [16]
  unsigned int* status;
  int32_t* arena;               // the warps' own arenas
  int64_t arena_words;          // per warp, including the gather space
  int64_t slot_words;           // per warp, slots only (gather space follows)
  int64_t gather_words;         // per warp: space for lists copied out of frames or host memory (paged)
  // Borrowed arenas: a warp whose candidate sets or copied lists outgrow its
  // own arena borrows one of n_big arenas sized for the plans' worst case,
  // for the rest of the root (or donated piece) it is on.
  int32_t* big_arena;
  int64_t big_slot_words;       // per borrowed arena: slots
  int64_t big_gather_words;     // per borrowed arena: gather space after the slots
  unsigned int* big_owner;      // [n_big]: 0 free, 1 held
  int32_t n_big;
  int32_t pad2;
  unsigned long long* root_counts;
  float* root_cost;
  float* root_reads;
  const int32_t* root_order;
  const int32_t* root_split;      // optional per-root donation threshold of the last-but-one level (plan 0)
  // donation ring: items (plan, root, level, begin, end, path[2..level])
  int4* don_items;                // 3 int4 per slot
  unsigned long long* don_head;   // next slot to fill
  unsigned long long* don_ready;  // per slot: sequence number + 1 when filled
  unsigned int don_mask;
  unsigned int* active;           // warps holding work (phase 1 or a donation)
  unsigned int total_warps;
  unsigned long long* don_tail;   // next slot to take
  unsigned long long* heartbeat;  // bumped by busy warps
  unsigned long long timeout_ns;  // hard limit on the launch; idle warps also give
                                  // up after this long without a heartbeat
  DPaging pg;
  // prefetch (paged, plan 0): pages to request for each root chunk, posted
  // when the chunk pf_ahead chunks earlier is claimed (CSR over chunks)
  const int32_t* pf_off;
  const int32_t* pf_pages;
  int32_t pf_ahead;
  int32_t pf_chunks;
  // the launch's plans, in the kernel's own parameter block: every launch
  // carries its own copy, so launches that overlap on a device (other
  // contexts, prepared queries, the allocation-free entry) never see each
  // other's plans
  DPlan plans[PM_MAX_BATCH];
};

enum { ST_SETOPS = 0, ST_BYTES = 1, ST_ROOTS = 2, ST_SPLITS = 3, ST_HITS = 4, ST_MISSES = 5,
       ST_ZC_BYTES = 6, ST_REQUESTS = 7, ST_EVICTIONS = 8, ST_DROPPED = 9, ST_WARP_NS = 10, ST_IDLE_NS = 11,
       ST_BORROWS = 12, ST_LEAF_CYC = 13, ST_LEVEL_CYC = 14, ST_PREFIX_CYC = 15, ST_PREFETCH = 16,
       ST_DEV_LOADS = 17, ST_DEV_BYTES = 18 };
// control block words: cursors[32] counts[32] stats[kStatWords] status/active ...
constexpr int kStatWords = 24;

#define PM_SB_MAX 512      // ints of a leaf batch's common operand kept in shared memory
#define PM_LANE_MAX 96     // longest first operand one lane handles alone in a leaf batch
#define PM_LEAF_BATCH 512  // candidates per leaf batch
#define PM_WIN 256         // window of a merged second operand held in shared memory

struct alignas(16) WarpState {
  int32_t path[8];
  int32_t iter[8];
  int32_t iend[8];   // exclusive end of the iteration range per level
  int32_t top[9];    // arena offset where level L's slots start
  int32_t off[16];
  int32_t size[16];
  unsigned long long next_beat;  // setops value at which to bump the heartbeat
  unsigned long long next_split; // setops value at which to look for idle warps
  unsigned long long t_start;    // %globaltimer at kernel entry (ns)
  int32_t* arena;                // slots of the current path: the warp's own arena or a borrowed one
  int32_t* gather;               // gather space for lists copied out of frames or host memory (paged)
  int64_t cap;                   // slot words at `arena`
  int32_t ghalf;                 // words in each of the two gather halves (first and second operand)
  int32_t big;                   // borrowed arena, or -1
  int32_t split;                 // donation threshold of the last-but-one level for the current root
  int32_t pins[PM_MAX_LIST_PAGES];  // paged mode: frames pinned for a gather
  alignas(16) int32_t sb[PM_SB_MAX + 4];  // the common operand (bitmap, hash table or sorted copy); +4 for a
                                         // bulk copy that starts up to 3 words before it
  unsigned long long mbar;               // completion barrier of the warp's bulk copies
  uint32_t mphase;                       // its current phase
  int32_t wb[PM_WIN];               // intersections by merge: the current window of the second operand
  unsigned long long lrb[32];       // leaf batches: start of each candidate's first operand in colidx
  int32_t lexcl[33];                // leaf batches: offset of each candidate's operand in the flat layout
};

// Per-warp work counters (registers; flushed once at kernel exit).
struct Work {
  unsigned long long setops, bytes, reads, borrows, prefetched;
  unsigned long long leaf_cyc, level_cyc, prefix_cyc;  // SM cycles by phase (lane 0's clock)
  unsigned int err;
  PageCounters pc;
};

// CG: the list may sit in an evictable frame; cg: it does (runtime).
template <bool CG>
__device__ __forceinline__ int32_t ld(const int32_t* p, bool cg = true) {
  if (CG && cg) return __ldcg(p);  // evictable frames are refilled during the launch: skip L1
  return *p;
}

// First index of sorted A[0,len) whose element is >= ub: a 32-ary search,
// one strided probe per lane per round (log32(len) rounds).
template <bool CG>
__device__ __forceinline__ int warp_lower_bound(const int32_t* A, int len, int ub, bool cg = true) {
  const int lane = lane_id();
  int lo = 0, hi = len;
  while (hi - lo > 32) {
    const int step = (hi - lo + 31) >> 5;
    const long long idx = lo + (long long)lane * step;
    const bool lt = idx < hi && ld<CG>(A + idx, cg) < ub;
    const int k = __popc(__ballot_sync(FULL, lt));
    if (k == 0) return lo;
    const int nhi = min(hi, lo + k * step);
    lo = lo + (k - 1) * step + 1;
    hi = nhi;
  }
  const int idx = lo + lane;
  const bool lt = idx < hi && ld<CG>(A + idx, cg) < ub;
  return lo + __popc(__ballot_sync(FULL, lt));
}

// Membership of x in sorted B[0, len) by binary search (per lane).
template <bool CG>
__device__ __forceinline__ bool bsearch_in(const int32_t* B, int len, int x, bool cg = true) {
  int lo = 0, hi = len;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ld<CG>(B + mid, cg) < x) lo = mid + 1; else hi = mid;
  }
  return lo < len && ld<CG>(B + lo, cg) == x;
}

// Adjacency list of v in id order: a slice of colidx in HBM, or resolved
// through the page cache (frame, gathered copy, or host read).  A labeled
// paged graph caches its label-grouped copy, so its whole sorted lists are
// read from host memory.
template <bool PAGED>
__device__ __forceinline__ ListRef adj(const MatchArgs& a, WarpState& S, int v, int32_t* gather, Work& w) {
  const uint64_t b = a.rowptr[v];
  const int len = (int)(a.rowptr[v + 1] - b);
  w.reads++;
  if (!PAGED) return ListRef{a.colidx + b, len, -1};
  if (a.host_sorted) return host_list_copy(a.host_sorted + b, len, gather);
  return paged_list(a.pg, b, len, gather, S.pins, w.pc);
}

// Start (relative to v's list) and length of the label-l part of v's list;
// empty for a label no vertex of the graph carries.
__device__ __forceinline__ int2 label_range(const MatchArgs& a, int v, int l) {
  if (l >= a.nl1 - 1) return make_int2(0, 0);
  const int32_t* o = a.lab_off + (int64_t)v * a.nl1;
  const int s0 = o[l];
  return make_int2(s0, o[l + 1] - s0);
}

// The label-l part of v's list, in id order: from the grouped copy in HBM,
// or through the page cache over the grouped copy.
template <bool PAGED>
__device__ __forceinline__ ListRef adj_label(const MatchArgs& a, WarpState& S, int v, int l, int32_t* gather,
                                             Work& w) {
  const uint64_t b = a.rowptr[v];
  const int2 r = label_range(a, v, l);
  w.reads++;
  if (!PAGED) return ListRef{a.colidx_lab + b + r.x, r.y, -1};
  return paged_list(a.pg, b + (uint64_t)r.x, r.y, gather, S.pins, w.pc);
}

// Operands shorter than this are staged by the lanes' own loads: a bulk
// copy's round trip through the mbarrier costs more than a few loads.
#define PM_BULK_MIN 256

// Stages n <= PM_SB_MAX words of the warp's arena into S.sb with one bulk
// asynchronous copy (cp.async.bulk, completion counted in bytes on the warp's
// mbarrier) and returns where src[0] landed: the copy starts at src rounded
// down to 16 bytes and covers whole 16-byte units, which stay inside the
// arena's allocation (every arena allocation has at least 256 bytes of slack
// after its last word).  The wait is bounded: a copy not complete after
// ~2^20 polls returns src itself (the caller reads B from global memory and
// reports DEV_TIMEOUT).
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __noinline__ const int32_t* stage_bulk(WarpState& S, const int32_t* src, int n) {
  const int lane = lane_id();
  if (n < PM_BULK_MIN) {
    __syncwarp();
    for (int i = lane; i < n; i += 32) S.sb[i] = src[i];
    __syncwarp();
    return S.sb;
  }
  const uintptr_t sa = reinterpret_cast<uintptr_t>(src);
  const uintptr_t a0 = sa & ~(uintptr_t)15;
  const int head = (int)((sa - a0) >> 2);
  const uint32_t bytes = (uint32_t)(((head + n) * 4 + 15) & ~15);
  const uint32_t mbar = smem_addr(&S.mbar);
  const uint32_t phase = S.mphase;
  // the lanes' earlier generic writes of the slot (global) and accesses of
  // S.sb (shared) come before the asynchronous proxy's read and write
  asm volatile("fence.proxy.async;" ::: "memory");
  __syncwarp();
  if (lane == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(S.sb)),
                 "l"(a0), "r"(bytes), "r"(mbar)
                 : "memory");
  }
  uint32_t done = 0;
  for (int spin = 0; spin < (1 << 20) && !done; spin++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
  }
  done = __all_sync(FULL, done);
  __syncwarp();
  if (!done) return src;
  if (lane == 0) S.mphase = phase ^ 1u;
  __syncwarp();
  return S.sb + head;
}

// Borrows a worst-case arena for the rest of the current root: copies the
// live slots [0, live) over (same offsets) and switches the warp to it.  The
// warp's own arena is left as it was, so operands already resolved into it
// stay valid.  Waits, up to the launch deadline, while every borrowed arena
// is held; a holder never waits for another one, so holders always finish.
// False (DEV_ARENA_OVERFLOW without a pool, DEV_TIMEOUT at the deadline) when
// none could be had.  Kept out of line: it is rare, and it must not pull the
// caller's counters out of registers.
__device__ __noinline__ unsigned borrow_arena(const MatchArgs& a, WarpState& S, int64_t live) {
  const int lane = lane_id();
  if (S.big >= 0 || a.n_big == 0) return DEV_ARENA_OVERFLOW;
  int got = -1;
  if (lane == 0) {
    const unsigned start = (unsigned)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) % (unsigned)a.n_big;
    while (got < 0) {
      for (int k = 0; k < a.n_big && got < 0; k++) {
        const int i = (int)((start + (unsigned)k) % (unsigned)a.n_big);
        if (*(volatile unsigned int*)&a.big_owner[i] == 0u && atomicCAS(&a.big_owner[i], 0u, 1u) == 0u) got = i;
      }
      if (got < 0) {
        if (global_ns() - S.t_start > a.timeout_ns) break;
        __nanosleep(2000);
      }
    }
  }
  got = __shfl_sync(FULL, got, 0);
  if (got < 0) return DEV_TIMEOUT;
  int32_t* dst = a.big_arena + (int64_t)got * (a.big_slot_words + a.big_gather_words);
  const int32_t* src = S.arena;
  for (int64_t i = lane; i < live; i += 32) dst[i] = src[i];
  __syncwarp();
  if (lane == 0) {
    S.arena = dst;
    S.cap = a.big_slot_words;
    S.gather = dst + a.big_slot_words;
    S.ghalf = (int32_t)(a.big_gather_words / 2);
    S.big = got;
  }
  __syncwarp();
  return 0;
}

__device__ __forceinline__ bool borrow(const MatchArgs& a, WarpState& S, int64_t live, Work& w) {
  const unsigned f = borrow_arena(a, S, live);
  w.err |= f;
  w.borrows += f ? 0 : 1;
  return f == 0;
}

// Gives a borrowed arena back (after the warp's writes to it) and returns
// the warp to its own arena.
__device__ __forceinline__ void return_arena(const MatchArgs& a, WarpState& S, int32_t* own) {
  if (S.big < 0) return;
  __syncwarp();
  __threadfence();
  __syncwarp();
  if (lane_id() == 0) {
    atomicExch(&a.big_owner[S.big], 0u);
    S.arena = own;
    S.cap = a.slot_words;
    S.gather = own + a.slot_words;
    S.ghalf = (int32_t)(a.gather_words / 2);
    S.big = -1;
  }
  __syncwarp();
}

// Room for `need` slot words from `top` on, borrowing an arena if the warp's
// own is too small; false (w.err set) when no arena can hold them.
__device__ __forceinline__ bool slot_room(const MatchArgs& a, WarpState& S, int64_t top, int64_t need, Work& w) {
  if (top + need <= S.cap) return true;
  if (!borrow(a, S, top, w)) return false;
  if (top + need <= S.cap) return true;
  w.err |= DEV_ARENA_OVERFLOW;
  return false;
}

// Room for copying a list of `len` words into either gather half (slots
// [0, live) are kept), borrowing an arena if needed.
__device__ __forceinline__ bool gather_room(const MatchArgs& a, WarpState& S, int64_t live, int64_t len, Work& w) {
  if (len <= S.ghalf) return true;
  if (!borrow(a, S, live, w)) return false;
  if (len <= S.ghalf) return true;
  w.err |= DEV_ARENA_OVERFLOW;
  return false;
}

// ---------------------------------------------------------------------
// One slot of level L for the warp's current path.  Restates compute_set
// (src/gpu_match.cu:238-319) with the operand choice of extend
// (src/gpu_match.cu:409-812): returns the slot size (at the last level the
// count), writes the slot to arena[top...] unless `last`.
// ---------------------------------------------------------------------
template <bool LABELED, bool PAGED>
__device__ int run_slot(const MatchArgs& a, const DPlan& P, WarpState& S, int L, int s, int top, bool last,
                        Work& w) {
  const int lane = lane_id();
  const int kind = P.kind[s];
  const int vL = S.path[L];
  ListRef RA, RB{nullptr, 0, -1};
  // one-label masks read only that label's part of an adjacency list: same
  // survivors in the same order, no label gathers (accounting still charges
  // the whole list, as the reference scans it)
  const uint32_t mask0 = P.slot_labels[s];
  const bool by_label = LABELED && a.lab_off && __popc(mask0) == 1 && (kind != SLOT_COPY || L == 1);
  if (PAGED) {
    // the adjacency operands may be copied into the gather halves: make room
    auto list_len = [&](int v) -> int64_t {
      return by_label ? label_range(a, v, __ffs(mask0) - 1).y : (int64_t)(a.rowptr[v + 1] - a.rowptr[v]);
    };
    int64_t need = 0;
    if (kind != SLOT_COPY) need = list_len(vL);
    else if (L == 1) need = list_len(S.path[0]);
    if (kind == SLOT_INTERSECT && L == 1) need = max(need, list_len(S.path[0]));
    if (!gather_room(a, S, top, need, w)) return 0;
  }
  int32_t* arena = S.arena;
  int32_t* gatherA = S.gather;
  int32_t* gatherB = S.gather + S.ghalf;
  int full_len = -1;  // length of the whole list when by_label
  int full_lenB = -1; // the same for a level-1 second operand read by label (paged)
  if (by_label) {
    const int v = (kind != SLOT_COPY) ? vL : S.path[0];
    full_len = (int)(a.rowptr[v + 1] - a.rowptr[v]);
    RA = adj_label<PAGED>(a, S, v, __ffs(mask0) - 1, gatherA, w);
  } else if (kind != SLOT_COPY) {
    RA = adj<PAGED>(a, S, vL, gatherA, w);
  } else if (L > 1) {
    RA = ListRef{arena + S.off[P.parent[s]], S.size[P.parent[s]], -1};
  } else {
    RA = adj<PAGED>(a, S, S.path[0], gatherA, w);
  }
  if (kind == SLOT_INTERSECT) {
    if (L > 1) {
      RB = ListRef{arena + S.off[P.parent[s]], S.size[P.parent[s]], -1};
    } else if (PAGED && by_label) {
      // only the label-l part of N(v0) can meet the label-l part of N(vL)
      const int v0 = S.path[0];
      full_lenB = (int)(a.rowptr[v0 + 1] - a.rowptr[v0]);
      RB = adj_label<PAGED>(a, S, v0, __ffs(mask0) - 1, gatherB, w);
    } else {
      RB = adj<PAGED>(a, S, S.path[0], gatherB, w);
    }
  }
  const int32_t* A = RA.p;
  const int32_t* B = RB.p;
  int lenA = RA.len;
  const int lenB = RB.len;
  const bool cgA = RA.cg;
  bool cgB = RB.cg;
  // a parent slot small enough goes to shared memory for the per-lane searches
  bool b_shared = false;
  if (kind == SLOT_INTERSECT && L > 1 && lenB <= PM_SB_MAX) {
    if (lenB > 0) {
      const int32_t* Bs = stage_bulk(S, B, lenB);
      b_shared = Bs != B;
      if (!b_shared) w.err |= DEV_TIMEOUT;
      B = Bs;
      cgB = cgB && !b_shared;
    }
  }

  // symmetry-breaking upper bound (unlabeled only, src/gpu_match.cu:426-458)
  if (!LABELED && P.partial[s]) {
    const bool is_main = (s == P.level_begin[L]);
    long long ub = is_main ? INT_MAX : -1;
    for (int j = 0; j <= L; j++) {
      if (!(P.partial[s] & (1u << j))) continue;
      const long long v = S.path[j];
      if (is_main) { if (v <= ub) ub = v; }
      else if (ub < v) ub = v;
    }
    if (ub == -1) ub = INT_MAX;
    if (ub != INT_MAX) lenA = warp_lower_bound<PAGED>(A, lenA, (int)ub, cgA);
  }

  const int T = a.T;
  int scan = lenA;
  const bool fresh_unl = (!LABELED && kind == SLOT_FRESH);
  if (fresh_unl && T && scan > T) scan = T;  // first pass keeps A's prefix
  int cnt = 0;
  // the slot holds at most the first T survivors
  if (!last && !slot_room(a, S, top, (T && scan > T) ? T : scan, w)) scan = 0;
  int32_t* out = S.arena + top;
  const uint32_t mask = P.slot_labels[s];
  // an intersection whose second operand is not in shared memory and at
  // most 4x the scanned part of the first: merge, B streamed through shared
  // memory in coalesced windows; else a search per element of A (which reads
  // less of a much longer B)
  const bool merge = kind == SLOT_INTERSECT && !b_shared && lenB > PM_WIN && (long long)lenB <= 4ll * scan;
  int bpos = 0;  // merge: B[0, bpos) is below every element still to come
  for (int base = 0; base < scan; base += 32) {
    const int i = base + lane;
    const bool valid = i < scan;
    const int x = valid ? ld<PAGED>(A + i, cgA) : 0;
    bool keep = valid;
    if (merge) {
      const int xlo = __shfl_sync(FULL, x, 0);
      const int xhi = __shfl_sync(FULL, x, min(31, scan - 1 - base));
      bpos += warp_lower_bound<PAGED>(B + bpos, lenB - bpos, xlo, cgB);
      bool open = valid;  // this lane's membership still undecided
      keep = false;
      while (__any_sync(FULL, open)) {
        const int wn = min(PM_WIN, lenB - bpos);
        if (wn <= 0) break;  // B exhausted: the rest of the tile is not in B
        __syncwarp();
        for (int k = lane; k < wn; k += 32) S.wb[k] = ld<PAGED>(B + bpos + k, cgB);
        __syncwarp();
        const int wlast = S.wb[wn - 1];
        if (open && x <= wlast) {
          keep = bsearch_in<false>(S.wb, wn, x);
          open = false;
        }
        if (xhi <= wlast) break;
        bpos += wn;
      }
      // bpos stays at the last window: it may hold elements of the next tile
    } else if (kind == SLOT_INTERSECT && keep) {
      keep = bsearch_in<PAGED>(B, lenB, x, cgB);
    }
    if (LABELED) {
      if (keep && !by_label) keep = (mask >> a.labels[x]) & 1u;
    } else if (kind == SLOT_COPY) {
      keep = keep && x != vL;
    } else if (kind == SLOT_FRESH) {
      for (int j = 0; j <= L; j++) keep = keep && x != S.path[j];
    }
    const unsigned bal = __ballot_sync(FULL, keep);
    if (!last && keep) {
      const int pos = cnt + __popc(bal & lanemask_lt());
      if (!T || pos < T) out[pos] = x;
    }
    cnt += __popc(bal);
    if (T && cnt >= T && !fresh_unl) break;  // result is the first T survivors
  }
  if (PAGED) {
    __syncwarp();
    unpin(a.pg, RA);
    unpin(a.pg, RB);
  }
  if (T && cnt > T) cnt = T;
  const int alenA = by_label ? full_len : lenA;
  const int alenB = full_lenB >= 0 ? full_lenB : lenB;
  w.setops++;
  w.bytes += 4ull * (unsigned long long)(alenA + alenB + cnt) + (LABELED ? (unsigned long long)alenA : 0ull);
  return cnt;
}

// Bound of slot s at level L from the partial order: the smallest (main
// slot) or largest (helper slot) constrained path vertex; INT_MAX if none.
template <bool LABELED>
__device__ __forceinline__ int slot_bound(const DPlan& P, const WarpState& S, int L, int s) {
  if (LABELED || !P.partial[s]) return INT_MAX;
  const bool is_main = (s == P.level_begin[L]);
  long long ub = is_main ? INT_MAX : -1;
  for (int j = 0; j <= L; j++) {
    if (!(P.partial[s] & (1u << j))) continue;
    const long long v = S.path[j];
    if (is_main) { if (v <= ub) ub = v; }
    else if (ub < v) ub = v;
  }
  return ub == -1 ? INT_MAX : (int)ub;
}

// A slot equal to, or a prefix of, a slot already computed at this level:
// no scan, only the reference's accounting for the set operation it stands
// for (its first operand's length below its bound, its result length).
template <bool LABELED, bool PAGED>
__device__ void alias_slot(const MatchArgs& a, const DPlan& P, WarpState& S, int L, int s, int live, Work& w) {
  const int t = P.alias[s];
  const int ub = slot_bound<LABELED>(P, S, L, s);
  if (PAGED && ub != INT_MAX) {
    const int v = P.kind[s] != SLOT_COPY ? S.path[L] : S.path[0];
    if ((P.kind[s] != SLOT_COPY || L == 1) && !gather_room(a, S, live, (int64_t)(a.rowptr[v + 1] - a.rowptr[v]), w))
      return;
  }
  const int32_t* arena = S.arena;
  int size = S.size[t];
  if (P.alias_prefix[s] && ub != INT_MAX) size = warp_lower_bound<false>(arena + S.off[t], size, ub);
  // first operand length as the reference would scan it
  const int kind = P.kind[s];
  int lenA, lenB = 0;
  if (kind != SLOT_COPY) {
    const int v = S.path[L];
    lenA = (int)(a.rowptr[v + 1] - a.rowptr[v]);
    if (ub != INT_MAX) {
      if (PAGED) {
        ListRef r = adj<PAGED>(a, S, v, S.gather, w);
        lenA = warp_lower_bound<PAGED>(r.p, r.len, ub, r.cg);
        __syncwarp();
        unpin(a.pg, r);
      } else {
        lenA = warp_lower_bound<false>(a.colidx + a.rowptr[v], lenA, ub);
      }
    }
  } else if (L > 1) {
    lenA = S.size[P.parent[s]];
    if (ub != INT_MAX) lenA = warp_lower_bound<false>(arena + S.off[P.parent[s]], lenA, ub);
  } else {
    const int v = S.path[0];
    lenA = (int)(a.rowptr[v + 1] - a.rowptr[v]);
    if (ub != INT_MAX) {
      if (PAGED) {
        ListRef r = adj<PAGED>(a, S, v, S.gather, w);
        lenA = warp_lower_bound<PAGED>(r.p, r.len, ub, r.cg);
        __syncwarp();
        unpin(a.pg, r);
      } else {
        lenA = warp_lower_bound<false>(a.colidx + a.rowptr[v], lenA, ub);
      }
    }
  }
  if (kind == SLOT_INTERSECT) {
    if (L > 1) lenB = S.size[P.parent[s]];
    else lenB = (int)(a.rowptr[S.path[0] + 1] - a.rowptr[S.path[0]]);
  }
  w.setops++;
  w.bytes += 4ull * (unsigned long long)(lenA + lenB + size) + (LABELED ? (unsigned long long)lenA : 0ull);
  if (lane_id() == 0) { S.off[s] = S.off[t]; S.size[s] = size; }
}

// Computes every slot of level L; returns the arena top after them.
template <bool LABELED, bool PAGED>
__device__ __forceinline__ int run_level(const MatchArgs& a, const DPlan& P, WarpState& S, int L, Work& w) {
  int top = S.top[L];
  for (int s = P.level_begin[L]; s < P.level_begin[L + 1]; s++) {
    if (P.alias[s] >= 0) continue;
    const int sz = run_slot<LABELED, PAGED>(a, P, S, L, s, top, false, w);
    if (lane_id() == 0) { S.off[s] = top; S.size[s] = sz; }
    top += sz;
  }
  __syncwarp();
  for (int s = P.level_begin[L]; s < P.level_begin[L + 1]; s++) {
    if (P.alias[s] < 0) continue;
    alias_slot<LABELED, PAGED>(a, P, S, L, s, top, w);
  }
  if (lane_id() == 0) S.top[L + 1] = top;
  __syncwarp();
  return top;
}

// First index of sorted A[0,len) whose element is >= x (one lane).  A list
// wholly below x (the common case for a symmetry-breaking bound) costs one
// load instead of a dependent chain.
template <bool CG = false>
__device__ __forceinline__ int lane_lower_bound(const int32_t* A, int len, int x, bool cg = true) {
  if (len == 0 || ld<CG>(A + len - 1, cg) < x) return len;
  int lo = 0, hi = len - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ld<CG>(A + mid, cg) < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// One lane intersects the part of sorted A[0,deg) below ub with sorted B
// (usually in shared memory), galloping through B; four loads of A in
// flight.  Sets *lenA to the number of elements of A below ub (the
// reference's scan length) and returns the count of members (label-checked
// when LABELED), or -1 when more than `cap` elements would be scanned (the
// caller hands the candidate to the whole warp).
template <bool LABELED, bool CG>
__device__ __forceinline__ int lane_intersect(const int32_t* A, int deg, int ub, const int32_t* B, int lenB,
                                              const uint8_t* labels, uint32_t mask, int* lenA, bool cg,
                                              int cap = PM_LANE_MAX) {
  int k = 0, p = 0, x = 0;
  while (true) {
    if (x >= cap) return -1;
    int v[4];
#pragma unroll
    for (int q = 0; q < 4; q++) v[q] = (x + q < deg) ? ld<CG>(A + x + q, cg) : INT_MAX;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int val = v[q];
      if (x + q >= deg || val >= ub) { *lenA = x + q; return k; }
      int lo = p, step = 1;
      while (lo + step < lenB && B[lo + step] < val) { lo += step; step <<= 1; }
      int hi = min(lo + step + 1, lenB);
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (B[mid] < val) lo = mid + 1; else hi = mid;
      }
      p = lo;
      if (p < lenB && B[p] == val && (!LABELED || ((mask >> labels[val]) & 1u))) k++;
      if (p >= lenB) {  // the rest of A is above all of B: only its length matters
        const int r0 = x + q + 1;
        *lenA = r0 + lane_lower_bound<CG>(A + r0, deg - r0, ub, cg);
        return k;
      }
    }
    x += 4;
  }
}

// Membership of x (>= 0) in an open-addressing table of 2^bits slots, empty
// slots -1, at most half full (so every probe run ends at an empty slot).
__device__ __forceinline__ bool in_table(const int32_t* t, int bits, int x) {
  unsigned h = ((unsigned)x * 0x9E3779B1u) >> (32 - bits);
  const unsigned m = (1u << bits) - 1;
  while (true) {
    const int y = t[h];
    if (y == x) return true;
    if (y < 0) return false;
    h = (h + 1) & m;
  }
}

// Membership structures for a leaf batch's common operand B (sorted), built
// in the warp's shared staging buffer (PM_SB_MAX words):
enum : int {
  MEMB_BITMAP = 0,  // max B < 32 * PM_SB_MAX: one bit per id in [0, max B]
  MEMB_FILTER = 1,  // |B| <= PM_SB_MAX / 4: a one-hash filter of 16 * PM_SB_MAX bits, then a hash table
  MEMB_HASH = 2,    // |B| <= PM_SB_MAX / 2: an open-addressing table at most half full
  MEMB_SORTED = 3   // else: the sorted copy, binary search
};

struct LeafSet {
  const int32_t* t;
  int bits;       // hash table: log2(slots)
  int lo, hi;     // min and max of B: outside [lo, hi] nothing is a member
};

__device__ __forceinline__ unsigned leaf_hash(int x, int bits) { return ((unsigned)x * 0x9E3779B1u) >> (32 - bits); }

template <int MODE>
__device__ __forceinline__ bool leaf_member(const LeafSet& m, int lenB, int x) {
  if (x < m.lo || x > m.hi) return false;
  if (MODE == MEMB_BITMAP) return (((const unsigned int*)m.t)[x >> 5] >> (x & 31)) & 1u;
  if (MODE == MEMB_FILTER) {
    const unsigned f = ((unsigned)x * 0x2545F491u) >> 19;  // 13 bits: PM_SB_MAX / 2 words of filter
    if (!((((const unsigned int*)m.t)[f >> 5] >> (f & 31)) & 1u)) return false;
    return in_table(m.t + PM_SB_MAX / 2, m.bits, x);
  }
  if (MODE == MEMB_HASH) return in_table(m.t, m.bits, x);
  return bsearch_in<false>(m.t, lenB, x);
}

// Builds the structure for B (whole warp) and returns its mode.
__device__ int leaf_build(WarpState& S, const int32_t* B, int lenB, LeafSet& m) {
  const int lane = lane_id();
  m.t = S.sb;
  m.lo = lenB ? B[0] : 1;
  m.hi = lenB ? B[lenB - 1] : 0;
  m.bits = 5;
  int mode;
  if (m.hi < 32 * PM_SB_MAX) {
    mode = MEMB_BITMAP;
    const int words = lenB ? (m.hi >> 5) + 1 : 0;
    for (int i = lane; i < words; i += 32) S.sb[i] = 0;
    __syncwarp();
    for (int i = lane; i < lenB; i += 32) atomicOr((unsigned int*)&S.sb[B[i] >> 5], 1u << (B[i] & 31));
  } else if (lenB <= PM_SB_MAX / 2) {
    mode = lenB <= PM_SB_MAX / 4 ? MEMB_FILTER : MEMB_HASH;
    int32_t* tab = S.sb + (mode == MEMB_FILTER ? PM_SB_MAX / 2 : 0);
    const int cap = mode == MEMB_FILTER ? PM_SB_MAX / 2 : PM_SB_MAX;
    while ((1 << m.bits) < 2 * lenB) m.bits++;
    if (mode == MEMB_FILTER) {
      while ((2 << m.bits) <= cap && (1 << m.bits) < 4 * lenB) m.bits++;  // at most a quarter full
      for (int i = lane; i < PM_SB_MAX / 2; i += 32) S.sb[i] = 0;
    }
    const int size = 1 << m.bits;  // <= cap
    for (int i = lane; i < size; i += 32) tab[i] = -1;
    __syncwarp();
    for (int i = lane; i < lenB; i += 32) {
      const int x = B[i];
      if (mode == MEMB_FILTER) {
        const unsigned f = ((unsigned)x * 0x2545F491u) >> 19;
        atomicOr((unsigned int*)&S.sb[f >> 5], 1u << (f & 31));
      }
      unsigned h = leaf_hash(x, m.bits);
      while (atomicCAS(&tab[h], -1, x) != -1) h = (h + 1) & (unsigned)(size - 1);
    }
  } else {
    mode = MEMB_SORTED;
    for (int i = lane; i < lenB; i += 32) S.sb[i] = B[i];
  }
  __syncwarp();
  return mode;
}

// One lane's contiguous part [t, tend) of a leaf batch's flat layout
// (candidate j's first operand occupies [lexcl[j], lexcl[j+1]) and starts at
// colidx[lrb[j]]): members of B, label-checked when LABELED.
template <bool LABELED, int MODE>
__device__ __forceinline__ unsigned leaf_walk(const MatchArgs& a, const WarpState& S, const LeafSet& m, int lenB,
                                              uint32_t mask, int t, int tend) {
  unsigned k = 0;
  auto test = [&](int x) {
    bool hit = leaf_member<MODE>(m, lenB, x);
    if (LABELED && hit) hit = (mask >> a.labels[x]) & 1u;
    k += hit ? 1u : 0u;
  };
  int j = 0;  // the last candidate whose offset is <= t
#pragma unroll
  for (int step = 16; step; step >>= 1)
    if (S.lexcl[j + step] <= t) j += step;
  while (t < tend) {
    const int jbeg = S.lexcl[j];
    const int stop = min(tend, S.lexcl[j + 1]);
    const int32_t* src = a.colidx + S.lrb[j] + (unsigned long long)(t - jbeg);
    const int n = stop - t;
    // scalar up to a 16-byte boundary, then 128-bit loads, four in flight (two, one at the tail)
    int q = min(n, (int)((4 - ((reinterpret_cast<uintptr_t>(src) >> 2) & 3)) & 3));
    for (int u = 0; u < q; u++) test(__ldg(src + u));
    const int4* v = reinterpret_cast<const int4*>(src + q);
    const int nv = (n - q) >> 2;
    int i = 0;
    for (; i + 4 <= nv; i += 4) {
      const int4 a0 = __ldg(v + i), a1 = __ldg(v + i + 1), a2 = __ldg(v + i + 2), a3 = __ldg(v + i + 3);
      test(a0.x); test(a0.y); test(a0.z); test(a0.w);
      test(a1.x); test(a1.y); test(a1.z); test(a1.w);
      test(a2.x); test(a2.y); test(a2.z); test(a2.w);
      test(a3.x); test(a3.y); test(a3.z); test(a3.w);
    }
    for (; i + 2 <= nv; i += 2) {
      const int4 a0 = __ldg(v + i), a1 = __ldg(v + i + 1);
      test(a0.x); test(a0.y); test(a0.z); test(a0.w);
      test(a1.x); test(a1.y); test(a1.z); test(a1.w);
    }
    if (i < nv) {
      const int4 a0 = __ldg(v + i);
      test(a0.x); test(a0.y); test(a0.z); test(a0.w);
    }
    for (q += 4 * nv; q < n; q++) test(__ldg(src + q));
    t = stop;
    j++;
  }
  return k;
}

// The last-level intersections of candidates [b, e) with the common operand B
// (|B| <= PM_SB_MAX), work-balanced across the warp: the first operands of 32
// candidates (each cut at its symmetry-breaking bound) are laid end to end
// and split into 32 contiguous parts, one per lane.  A lane finds the
// candidate owning its part's start once and walks on through the following
// lists, four 128-bit loads in flight, testing each element against B's structure in
// shared memory (leaf_build).  Counts only; no truncation.  Same set
// operations, counts and accounting as lane_intersect per candidate.
// Batches averaging under 16 elements per lane, and a.leaf_flat == 2, use
// the strided layout instead (element t0 + lane, owner found per element by
// shuffles): it has no per-lane setup per candidate.
template <bool LABELED>
__device__ unsigned long long leaf_flat(const MatchArgs& a, WarpState& S, const int32_t* cand, int b, int e,
                                        const int32_t* B, int lenB, uint32_t mask, int common_ub, bool self_ub,
                                        Work& w) {
  const int lane = lane_id();
  LeafSet m;
  const int mode = leaf_build(S, B, lenB, m);
  unsigned long long cnt = 0, bytes = 0, ops = 0;  // per lane
  for (int base = b; base < e; base += 32) {
    const int i = base + lane;
    const bool mine = i < e;
    int lenA = 0;
    unsigned long long rb = 0;
    if (mine) {
      const int c = cand[i];
      rb = a.rowptr[c];
      const int deg = (int)(a.rowptr[c + 1] - rb);
      const int ub = self_ub ? min(common_ub, c) : common_ub;
      lenA = (ub == INT_MAX) ? deg : lane_lower_bound(a.colidx + rb, deg, ub);
      bytes += 4ull * (unsigned long long)(lenA + lenB) + (LABELED ? (unsigned long long)lenA : 0ull);
      ops++;
    }
    int incl = lenA;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    // short lists (under 16 elements per lane): the strided layout has no
    // per-candidate setup per lane
    if (a.leaf_flat == 2 || total < 16 * 32) {
      const int excl = incl - lenA;
      for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        int j = 0, ej = 0;  // the last lane whose offset is <= t owns element t
#pragma unroll
        for (int step = 16; step; step >>= 1) {
          const int e2 = __shfl_sync(FULL, excl, j + step);
          if (e2 <= t) { j += step; ej = e2; }
        }
        const unsigned long long rbj = __shfl_sync(FULL, rb, j);
        if (t < total) {
          const int x = a.colidx[rbj + (unsigned long long)(t - ej)];
          bool hit = mode == MEMB_BITMAP   ? leaf_member<MEMB_BITMAP>(m, lenB, x)
                     : mode == MEMB_FILTER ? leaf_member<MEMB_FILTER>(m, lenB, x)
                     : mode == MEMB_HASH   ? leaf_member<MEMB_HASH>(m, lenB, x)
                                           : leaf_member<MEMB_SORTED>(m, lenB, x);
          if (LABELED && hit) hit = (mask >> a.labels[x]) & 1u;
          cnt += hit ? 1u : 0u;
        }
      }
      continue;
    }
    S.lrb[lane] = rb;
    S.lexcl[lane] = incl - lenA;
    if (lane == 31) S.lexcl[32] = total;
    __syncwarp();
    const int chunk = (total + 31) >> 5;
    const int t = min(total, lane * chunk);
    const int tend = min(total, t + chunk);
    unsigned k;
    if (mode == MEMB_BITMAP) k = leaf_walk<LABELED, MEMB_BITMAP>(a, S, m, lenB, mask, t, tend);
    else if (mode == MEMB_FILTER) k = leaf_walk<LABELED, MEMB_FILTER>(a, S, m, lenB, mask, t, tend);
    else if (mode == MEMB_HASH) k = leaf_walk<LABELED, MEMB_HASH>(a, S, m, lenB, mask, t, tend);
    else k = leaf_walk<LABELED, MEMB_SORTED>(a, S, m, lenB, mask, t, tend);
    cnt += k;
    __syncwarp();
  }
  bytes += 4ull * cnt;  // the results
  for (int o = 16; o; o >>= 1) {
    cnt += __shfl_xor_sync(FULL, cnt, o);
    bytes += __shfl_xor_sync(FULL, bytes, o);
    ops += __shfl_xor_sync(FULL, ops, o);
  }
  w.setops += ops;
  w.bytes += bytes;
  return cnt;
}

// The last level for the candidates [b, e) of level L's main slot (each is
// v_{n-2} in turn): one lane per candidate, counting only.  Same set
// operations and counts as run_slot(last) per candidate, organised so that
// short operands cost one lane each:
//   * unlabeled fresh sets and copies are counted with binary searches (the
//     prefix below the bound, minus path vertices found in it);
//   * intersections merge the candidate's list with the common second operand
//     (staged in shared memory when it fits), galloping through it;
//   * a labeled copy is the same for every candidate: counted once;
//   * candidates whose first operand is longer than PM_LANE_MAX go back to the
//     warp-cooperative run_slot.
template <bool LABELED, bool PAGED>
__device__ unsigned long long leaf_batch(const MatchArgs& a, const DPlan& P, WarpState& S, int L, int b, int e,
                                         Work& w) {
  const int32_t* arena = S.arena;
  const int lane = lane_id();
  const int s = P.last_slot;
  const int kind = P.kind[s];
  const int Lf = L + 1;
  const int32_t* cand = arena + S.off[P.level_begin[L]];
  const int par = P.parent[s];
  const int32_t* B = arena + S.off[par];  // intersect: second operand; copy: first operand
  const int lenB = S.size[par];
  const uint32_t mask = P.slot_labels[s];
  const int T = a.T;
  unsigned long long cnt_warp = 0;  // uniform across lanes
  if (LABELED && kind == SLOT_COPY) {
    int k = 0;
    for (int i = lane; i < lenB; i += 32) k += (mask >> a.labels[B[i]]) & 1u;
    for (int o = 16; o; o >>= 1) k += __shfl_xor_sync(FULL, k, o);
    if (T && k > T) k = T;
    const unsigned long long m = (unsigned long long)(e - b);
    w.setops += m;
    w.bytes += m * (4ull * (unsigned long long)(lenB + k) + (unsigned long long)lenB);
    return m * (unsigned long long)k;
  }
  // symmetry-breaking bound: bits 0..L are common, bit L+1 is the candidate
  int common_ub = INT_MAX;
  bool self_ub = false;
  if (!LABELED && P.partial[s]) {
    for (int j = 0; j <= L; j++)
      if (P.partial[s] & (1u << j)) common_ub = min(common_ub, S.path[j]);
    self_ub = (P.partial[s] >> Lf) & 1u;
  }
  if (!PAGED && kind == SLOT_INTERSECT && T == 0 && lenB <= PM_SB_MAX && a.leaf_flat &&
      !(LABELED && a.lab_off && __popc(mask) == 1))
    return leaf_flat<LABELED>(a, S, cand, b, e, B, lenB, mask, common_ub, self_ub, w);
  const int32_t* Bs = B;
  if (kind == SLOT_INTERSECT && lenB <= PM_SB_MAX && lenB > 0) {
    Bs = stage_bulk(S, B, lenB);
    if (Bs == B) w.err |= DEV_TIMEOUT;
  }
  unsigned long long cnt = 0, bytes = 0, ops = 0;  // per lane
  PageCounters lpc = {};                           // per lane (paged residency)
  for (int base = b; base < e; base += 32) {
    const int i = base + lane;
    const bool mine = i < e;
    const int c = mine ? cand[i] : 0;
    bool deferred = false;
    int32_t want = -1;  // an absent page this lane read around, for the warp to load
    if (mine) {
      const int ub = self_ub ? min(common_ub, c) : common_ub;
      if (kind == SLOT_COPY) {  // unlabeled: A = parent slot minus the candidate
        const int lenA = (ub == INT_MAX) ? lenB : lane_lower_bound(B, lenB, ub);
        const int pos = lane_lower_bound(B, lenA, c);
        int k = lenA - ((pos < lenA && B[pos] == c) ? 1 : 0);
        if (T && k > T) k = T;
        cnt += k;
        bytes += 4ull * (unsigned long long)(lenA + k);
        ops++;
      } else {
        const uint64_t rb = a.rowptr[c];
        const int deg = (int)(a.rowptr[c + 1] - rb);
        // a one-label mask reads only that label's part of the list
        const bool grouped = LABELED && a.lab_off && __popc(mask) == 1;
        const int2 gr = grouped ? label_range(a, c, __ffs(mask) - 1) : make_int2(0, deg);
        const int32_t* A = PAGED ? nullptr : (grouped ? a.colidx_lab + rb + gr.x : a.colidx + rb);
        int32_t pinned = -1;
        bool cgl = false;  // A sits in an evictable frame
        if (PAGED) {
          // this lane's own list (or label part) when its one page is
          // resident (pinned and read from the frame) or it spans consecutive
          // static frames; a missing page, a list over evictable pages, or a
          // whole sorted list of a labeled graph (host memory) goes to the
          // warp, which reads host memory coalesced, gathers and requests pages
          const uint64_t s0 = rb + (uint64_t)gr.x;
          const int sh = a.pg.page_shift;
          if (LABELED && !grouped) {
            deferred = true;
          } else if (gr.y == 0) {
            A = a.pg.host_colidx + s0;  // nothing is read
          } else {
            const int32_t p0 = (int32_t)(s0 >> sh);
            const int32_t p1 = (int32_t)((s0 + (uint64_t)gr.y - 1) >> sh);
            const int32_t f = (p0 == p1) ? (pinned = try_pin(a.pg, p0)) : static_run(a.pg, p0, p1);
            if (f >= 0) {
              A = a.pg.frames + ((uint64_t)f << sh) + (s0 & ((1ull << sh) - 1));
              cgl = f >= a.pg.n_static;
              lpc.hits++;
            } else if (p0 == p1 && gr.y <= PM_LANE_MAX) {
              // a short list on a missing page: this lane copies it from host
              // memory into its own part of the gather space, 16 reads in
              // flight per round trip, and notes the page for the warp to
              // load after the batch (or posts it to the host thread)
              if (ld_vol(&a.pg.page_frame[p0]) == PAGE_ABSENT) {
                if (a.pg.dev_copy) want = p0;
                else request_page(a.pg, p0, lpc);
              }
              const int32_t* src = a.pg.host_colidx + s0;
              int32_t* stage = S.gather + lane * PM_LANE_MAX;
              for (int x = 0; x < gr.y; x += 16) {
                int v[16];
#pragma unroll
                for (int q = 0; q < 16; q++) v[q] = (x + q < gr.y) ? src[x + q] : 0;
#pragma unroll
                for (int q = 0; q < 16; q++)
                  if (x + q < gr.y) stage[x + q] = v[q];
              }
              A = stage;
              lpc.misses++;
              lpc.zc_bytes += 4ull * (unsigned long long)gr.y;
            } else {
              deferred = true;
            }
          }
        }
        if (deferred) {
          // handled by the warp below
        } else if (kind == SLOT_INTERSECT && !grouped) {
          int lenA = 0;
          int k = lane_intersect<LABELED, PAGED>(A, deg, ub, Bs, lenB, a.labels, mask, &lenA, cgl);
          if (k < 0) {
            deferred = true;
          } else {
            if (T && k > T) k = T;
            cnt += k;
            bytes += 4ull * (unsigned long long)(lenA + lenB + k) + (LABELED ? (unsigned long long)lenA : 0ull);
            ops++;
          }
        } else {
        const int lenA = (ub == INT_MAX) ? deg : lane_lower_bound<PAGED>(A, deg, ub, cgl);
        if (grouped) {
          // the label-l part of the list: a fresh set is its length, an
          // intersection merges only it
          const int32_t* Al = A;
          const int lenl = gr.y;
          int k = 0;
          if (kind == SLOT_FRESH) {
            k = lenl;
          } else if (lenl > PM_LANE_MAX) {
            deferred = true;
          } else {
            int p = 0;
            for (int x = 0; x < lenl && p < lenB; x++) {
              const int v = ld<PAGED>(Al + x, cgl);
              int lo = p, step = 1;
              while (lo + step < lenB && Bs[lo + step] < v) { lo += step; step <<= 1; }
              int hi = min(lo + step + 1, lenB);
              while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (Bs[mid] < v) lo = mid + 1; else hi = mid;
              }
              p = lo;
              k += (p < lenB && Bs[p] == v) ? 1 : 0;
            }
          }
          if (!deferred) {
            if (T && k > T) k = T;
            cnt += k;
            bytes += 4ull * (unsigned long long)(deg + (kind == SLOT_INTERSECT ? lenB : 0) + k) +
                     (unsigned long long)deg;
            ops++;
          }
        } else if (!LABELED && kind == SLOT_FRESH) {
          // first min(lenA, T) elements, minus the path vertices among them
          const int lim = (T && lenA > T) ? T : lenA;
          int k = lim;
          for (int j = 0; j <= L; j++) {
            const int pj = S.path[j];
            const int pos = lane_lower_bound<PAGED>(A, lim, pj, cgl);
            k -= (pos < lim && ld<PAGED>(A + pos, cgl) == pj) ? 1 : 0;
          }
          cnt += k;
          bytes += 4ull * (unsigned long long)(lenA + k);
          ops++;
        } else if (lenA > PM_LANE_MAX) {
          deferred = true;
        } else if (kind == SLOT_FRESH) {  // labeled: label filter only
          int k = 0;
          for (int x = 0; x < lenA; x++) k += (mask >> a.labels[ld<PAGED>(A + x, cgl)]) & 1u;
          if (T && k > T) k = T;
          cnt += k;
          bytes += 4ull * (unsigned long long)(lenA + k) + (unsigned long long)lenA;
          ops++;
        } else {  // intersection with the common operand
          int k = 0, p = 0;
          for (int x = 0; x < lenA && p < lenB; x++) {
            const int v = ld<PAGED>(A + x, cgl);
            int lo = p, step = 1;
            while (lo + step < lenB && Bs[lo + step] < v) { lo += step; step <<= 1; }
            int hi = min(lo + step + 1, lenB);
            while (lo < hi) {
              const int mid = (lo + hi) >> 1;
              if (Bs[mid] < v) lo = mid + 1; else hi = mid;
            }
            p = lo;
            if (p < lenB && Bs[p] == v && (!LABELED || ((mask >> a.labels[v]) & 1u))) k++;
          }
          if (T && k > T) k = T;
          cnt += k;
          bytes += 4ull * (unsigned long long)(lenA + lenB + k) + (LABELED ? (unsigned long long)lenA : 0ull);
          ops++;
        }
        }
        if (PAGED && pinned >= 0) unpin_frame(a.pg, pinned);
      }
    }
    // long first operands: the warp takes them one by one
    unsigned dm = __ballot_sync(FULL, deferred);
    while (dm) {
      const int src = __ffs(dm) - 1;
      dm &= dm - 1;
      const int cc = __shfl_sync(FULL, c, src);
      if (lane == 0) S.path[Lf] = cc;
      __syncwarp();
      cnt_warp += (unsigned long long)run_slot<LABELED, PAGED>(a, P, S, Lf, s, S.top[Lf], true, w);
    }
    if (PAGED) {
      // pages the lanes read around: the warp loads up to two of them per
      // 32 candidates (one page copy each), so later reads hit
      unsigned wm = __ballot_sync(FULL, want >= 0);
      for (int k = 0; k < 2 && wm; k++) {
        const int src = __ffs(wm) - 1;
        wm &= wm - 1;
        warp_load_page(a.pg, __shfl_sync(FULL, want, src), w.pc);
      }
    }
  }
  if (PAGED) {
    unsigned long long v[6] = {lpc.hits, lpc.misses, lpc.zc_bytes, lpc.requests, lpc.evictions, lpc.dropped};
#pragma unroll
    for (int k = 0; k < 6; k++)
      for (int o = 16; o; o >>= 1) v[k] += __shfl_xor_sync(FULL, v[k], o);
    w.pc.hits += v[0];
    w.pc.misses += v[1];
    w.pc.zc_bytes += v[2];
    w.pc.requests += v[3];
    w.pc.evictions += v[4];
    w.pc.dropped += v[5];
  }
  for (int o = 16; o; o >>= 1) {
    cnt += __shfl_xor_sync(FULL, cnt, o);
    bytes += __shfl_xor_sync(FULL, bytes, o);
    ops += __shfl_xor_sync(FULL, ops, o);
  }
  w.setops += ops;
  w.bytes += bytes;
  return cnt + cnt_warp;
}

// The last two levels below candidates [b, e) of level L = nnodes-4, one
// lane per candidate v: the lane computes level L+1's intersection X (and
// its alias Y) for path[L+1] = v into its own part of the free arena, then
// counts the last level over X/Y's candidates -- the small sets of light
// subtrees, where warp-wide set operations leave most lanes idle.  Same set
// operations, counts and accounting as run_level + leaf_batch; unlabeled
// plans of the shape DPlan.l2_x describes, no truncation, X's parent at most
// lane_subtree_max long (it is staged in shared memory).
__device__ unsigned long long lane_subtree(const MatchArgs& a, const DPlan& P, WarpState& S, int L, int b, int e,
                                           Work& w) {
  int32_t* arena = S.arena;
  const int lane = lane_id();
  const int Lq = L + 1;
  const int X = P.l2_x, Y = P.l2_y, M = P.level_begin[Lq], last = P.last_slot;
  const int p1 = P.parent[X];
  const int lenB1 = S.size[p1];
  const int32_t* B1 = arena + S.off[p1];
  const int32_t* Bs = lenB1 > 0 ? stage_bulk(S, B1, lenB1) : B1;
  if (lenB1 > 0 && Bs == B1) w.err |= DEV_TIMEOUT;
  const int32_t* cand = arena + S.off[P.level_begin[L]];
  unsigned long long cnt = 0, bytes = 0, ops = 0;
  const int i = b + lane;
  if (i < e) {
    const int v = cand[i];
    // slot bounds with path[Lq] = v: main slots take the smallest constrained
    // path vertex, helpers the largest (slot_bound)
    auto bound = [&](int s) -> int {
      const bool is_main = (s == M);
      long long ub = is_main ? INT_MAX : -1;
      for (int j = 0; j <= Lq; j++) {
        if (!((P.partial[s] >> j) & 1u)) continue;
        const long long pv = (j == Lq) ? v : S.path[j];
        if (is_main) { if (pv <= ub) ub = pv; }
        else if (ub < pv) ub = pv;
      }
      return ub == -1 ? INT_MAX : (int)ub;
    };
    const uint64_t rb = a.rowptr[v];
    const int deg = (int)(a.rowptr[v + 1] - rb);
    const int32_t* A = a.colidx + rb;
    // X = N(v) below its bound, intersected with its parent
    const int ubX = bound(X);
    const int lenAX = (ubX == INT_MAX) ? deg : lane_lower_bound(A, deg, ubX);
    int32_t* buf = arena + S.top[Lq] + lane * lenB1;
    int sizeX = 0, p = 0;
    for (int x = 0; x < lenAX && p < lenB1; x++) {
      const int val = A[x];
      int lo = p, step = 1;
      while (lo + step < lenB1 && Bs[lo + step] < val) { lo += step; step <<= 1; }
      int hi = min(lo + step + 1, lenB1);
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (Bs[mid] < val) lo = mid + 1; else hi = mid;
      }
      p = lo;
      if (p < lenB1 && Bs[p] == val) buf[sizeX++] = val;
    }
    bytes += 4ull * (unsigned long long)(lenAX + lenB1 + sizeX);
    ops++;
    w.reads++;
    // Y: X itself or its prefix below Y's bound, charged as its own operation
    int sizeY = sizeX;
    if (Y >= 0) {
      const int ubY = bound(Y);
      if (P.alias_prefix[Y] && ubY != INT_MAX) sizeY = lane_lower_bound(buf, sizeX, ubY);
      const int lenAY = (ubY == INT_MAX) ? deg : lane_lower_bound(A, deg, ubY);
      bytes += 4ull * (unsigned long long)(lenAY + lenB1 + sizeY);
      ops++;
    }
    const int sizeM = (M == X) ? sizeX : sizeY;
    const int sizeB = (P.parent[last] == X) ? sizeX : sizeY;
    // the last level over the main slot's candidates c
    int common = INT_MAX;
    for (int j = 0; j <= Lq; j++)
      if ((P.partial[last] >> j) & 1u) common = min(common, (j == Lq) ? v : S.path[j]);
    const bool self_ub = (P.partial[last] >> (Lq + 1)) & 1u;
    for (int k = 0; k < sizeM; k++) {
      const int c = buf[k];
      const int ub = self_ub ? min(common, c) : common;
      const uint64_t rc = a.rowptr[c];
      const int dc = (int)(a.rowptr[c + 1] - rc);
      int lenA = 0;
      const int kk = lane_intersect<false, false>(a.colidx + rc, dc, ub, buf, sizeB, a.labels, 0u, &lenA, false,
                                                  INT_MAX);
      cnt += (unsigned long long)kk;
      bytes += 4ull * (unsigned long long)(lenA + sizeB + kk);
      ops++;
    }
  }
  for (int o = 16; o; o >>= 1) {
    cnt += __shfl_xor_sync(FULL, cnt, o);
    bytes += __shfl_xor_sync(FULL, bytes, o);
    ops += __shfl_xor_sync(FULL, ops, o);
  }
  w.setops += ops;
  w.bytes += bytes;
  return cnt;
}

// A donated piece of a DFS: candidates [begin, end) of level `level`'s main
// slot under the path root(v0, v1), path[2..level].
struct Donation {
  int plan, root, level, begin, end;
  int path[7];  // path[2..level] used
};

// Hands the upper half of the shallowest level range that is long enough to
// the donation ring, when some warps are idle and fewer pieces are queued
// than idle warps.  A range whose candidates head whole subtrees is long
// enough from 2 candidates on; one whose candidates only lead to the last
// level (one set operation each) needs split_min.  Lane 0 decides.
__device__ __forceinline__ void maybe_donate(const MatchArgs& a, WarpState& S, int n, int L0, int L, int plan_id,
                                             int root_id) {
  const int lane = lane_id();
  if (lane == 0) {
    const unsigned int act = *((volatile unsigned int*)a.active);
    const unsigned long long head = *((volatile unsigned long long*)a.don_head);
    const unsigned long long tail = *((volatile unsigned long long*)a.don_tail);
    if (act < a.total_warps && head - tail < (unsigned long long)(a.total_warps - act) &&
        head - tail < (unsigned long long)a.don_mask) {
      for (int k = L0; k <= L; k++) {
        const int it = S.iter[k], iend = S.iend[k];
        if (iend - it < ((k + 1 == n - 2) ? max(S.split, 2) : 2)) continue;
        const int mid = it + (iend - it) / 2;  // it < mid < iend
        const unsigned long long slot = atomicAdd(a.don_head, 1ull);
        int4* dst = a.don_items + 3 * (slot & a.don_mask);
        dst[0] = make_int4(plan_id, root_id, k, mid);
        dst[1] = make_int4(iend, S.path[2], S.path[3], S.path[4]);
        dst[2] = make_int4(S.path[5], S.path[6], 0, 0);
        st_release(&a.don_ready[slot & a.don_mask], slot + 1);
        atomicAdd(&a.stats[ST_SPLITS], 1ull);
        S.iend[k] = mid;
        break;
      }
    }
  }
  __syncwarp();
}

// Depth-first enumeration below a fixed path prefix.  path[0..L0] must be
// set; levels 1..L0 are computed here (for a donated piece this repeats the
// donor's work and is kept out of the counters), then candidates [b, e) of
// level L0's main slot (e < 0: all) are enumerated to the last level.
// Restates match() (src/gpu_match.cu:855-1047) without deferral: every
// branch is finished where it starts.
template <bool LABELED, bool PAGED>
__device__ unsigned long long dfs_from(const MatchArgs& a, const DPlan& P, WarpState& S, int L0, int b, int e,
                                       bool counted_prefix, int plan_id, int root_id, Work& w) {
  const int lane = lane_id();
  const int n = P.nnodes;
  if (lane == 0) S.top[1] = 0;
  __syncwarp();
  if (n == 3) return (unsigned long long)run_slot<LABELED, PAGED>(a, P, S, 1, P.level_begin[1], 0, true, w);
  {
    const unsigned long long so = w.setops, by = w.bytes, rd = w.reads;
    const long long c0 = clock64();
    for (int k = 1; k <= L0 && !w.err; k++) run_level<LABELED, PAGED>(a, P, S, k, w);
    if (!counted_prefix) {
      w.setops = so;
      w.bytes = by;
      w.reads = rd;
      w.prefix_cyc += (unsigned long long)(clock64() - c0);
    } else {
      w.level_cyc += (unsigned long long)(clock64() - c0);
    }
  }
  if (w.err) return 0;
  unsigned long long cnt = 0;
  {
    int end0 = S.size[P.level_begin[L0]];
    if (e >= 0 && e < end0) end0 = e;
    if (lane == 0) { S.iter[L0] = b; S.iend[L0] = end0; }
    __syncwarp();
  }
  int L = L0;
  while (true) {
    // liveness signal for idle warps and the launch-wide deadline, then the
    // periodic look for idle warps to hand work to
    if (w.setops >= S.next_beat) {
      int late = 0;
      if (lane == 0) {
        atomicAdd(a.heartbeat, 1ull);
        S.next_beat = w.setops + 1024;
        late = (global_ns() - S.t_start) > a.timeout_ns;
      }
      if (__shfl_sync(FULL, late, 0)) {
        w.err |= DEV_TIMEOUT;
        return 0;
      }
    }
    if (a.split_min > 0 && w.setops >= S.next_split) {
      if (lane == 0) S.next_split = w.setops + 64;
      maybe_donate(a, S, n, L0, L, plan_id, root_id);
    }
    const int m = P.level_begin[L];
    const int it = S.iter[L];
    const int iend = S.iend[L];
    bool subtree = false;
    if constexpr (!LABELED && !PAGED)
      subtree = P.l2_x >= 0 && L + 4 == n && it < iend && a.lane_subtree_max > 0 &&
                S.size[P.parent[P.l2_x]] <= a.lane_subtree_max &&
                S.top[L + 1] + 32ll * S.size[P.parent[P.l2_x]] <= S.cap;
    if (subtree) {
      const int e2 = min(iend, it + 32);
      const long long c0 = clock64();
      cnt += lane_subtree(a, P, S, L, it, e2, w);
      w.leaf_cyc += (unsigned long long)(clock64() - c0);
      if (lane == 0) S.iter[L] = e2;
      __syncwarp();
    } else if (it < iend && L + 1 == n - 2) {
      const int e2 = min(iend, it + PM_LEAF_BATCH);
      const long long c0 = clock64();
      cnt += leaf_batch<LABELED, PAGED>(a, P, S, L, it, e2, w);
      w.leaf_cyc += (unsigned long long)(clock64() - c0);
      if (lane == 0) S.iter[L] = e2;
      __syncwarp();
      if (w.err) return 0;
    } else if (it < iend) {
      const int v = S.arena[S.off[m] + it];
      if (lane == 0) { S.iter[L] = it + 1; S.path[L + 1] = v; }
      __syncwarp();
      const long long c0 = clock64();
      if (L + 1 == n - 2) {
        cnt += (unsigned long long)run_slot<LABELED, PAGED>(a, P, S, L + 1, P.last_slot, S.top[L + 1], true, w);
        w.leaf_cyc += (unsigned long long)(clock64() - c0);
      } else {
        L++;
        run_level<LABELED, PAGED>(a, P, S, L, w);
        w.level_cyc += (unsigned long long)(clock64() - c0);
        if (lane == 0) { S.iter[L] = 0; S.iend[L] = S.size[P.level_begin[L]]; }
        __syncwarp();
      }
      if (w.err) return 0;
    } else {
      L--;
      if (L < L0) break;
    }
  }
  return cnt;
}

// Takes one donated piece if any is queued.  The caller is counted as active
// before it claims, so "no active warp and nothing queued" is a safe exit
// test for everyone.  Returns false if nothing was taken.
__device__ bool take_donation(const MatchArgs& a, Donation& d) {
  int got = 0;
  int v[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (lane_id() == 0) {
    const unsigned long long tail = *((volatile unsigned long long*)a.don_tail);
    const unsigned long long head = *((volatile unsigned long long*)a.don_head);
    if (tail < head) {
      // counted as active before claiming (no fence: if another warp reads
      // the claim before the count it may leave early, never lose work)
      atomicAdd(a.active, 1u);
      if (atomicCAS(a.don_tail, tail, tail + 1) == tail) {
        // bounded wait for the donor to finish writing this slot
        for (int spin = 0; spin < (1 << 22); spin++) {
          if (ld_acquire(&a.don_ready[tail & a.don_mask]) == tail + 1) { got = 1; break; }
          __nanosleep(64);
        }
        if (got) {
          const volatile int* src = (const volatile int*)(a.don_items + 3 * (tail & a.don_mask));
          for (int i = 0; i < 12; i++) v[i] = src[i];
        } else {
          atomicOr(a.status, (unsigned)DEV_TIMEOUT);
          atomicSub(a.active, 1u);
        }
      } else {
        atomicSub(a.active, 1u);
      }
    }
  }
  got = __shfl_sync(FULL, got, 0);
  int u[12];
#pragma unroll
  for (int i = 0; i < 12; i++) u[i] = __shfl_sync(FULL, v[i], 0);
  d.plan = u[0];
  d.root = u[1];
  d.level = u[2];
  d.begin = u[3];
  d.end = u[4];
  d.path[0] = 0;
  d.path[1] = 0;
  d.path[2] = u[5];
  d.path[3] = u[6];
  d.path[4] = u[7];
  d.path[5] = u[8];
  d.path[6] = u[9];
  return got != 0;
}

// MINB = 4: 64 registers, four 256-thread blocks per SM (more warps in flight,
// some spills); MINB = 3: 85 registers, three blocks; MINB = 1: up to 128
// registers, no spills, fewer warps.
template <bool LABELED, bool PAGED, int MINB>
__global__ void __launch_bounds__(MINB == 1 ? 512 : 256, MINB) match_kernel(const __grid_constant__ MatchArgs a) {
  extern __shared__ WarpState smem_state[];
  const int lane = lane_id();
  const int wib = threadIdx.x >> 5;
  WarpState& S = smem_state[wib];
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + wib;
  int32_t* own = a.arena + gw * a.arena_words;
  if (lane == 0) {
    S.next_beat = 0;
    S.next_split = 0;
    S.t_start = global_ns();
    S.arena = own;
    S.cap = a.slot_words;
    S.gather = own + a.slot_words;
    S.ghalf = (int32_t)(a.gather_words / 2);
    S.big = -1;
    S.mphase = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&S.mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  Work w;
  memset(&w, 0, sizeof(w));
  unsigned long long roots = 0;
  const int np = a.nplans;
  int p = (int)(gw % np);
  int exhausted = 0;
  // phase 1: root chunks from the per-plan cursors
  while (exhausted < np && !w.err) {
    const DPlan& P = a.plans[p];
    const unsigned long long nchunks = (unsigned long long)((P.nroots + a.chunk - 1) / a.chunk);
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(&a.cursors[p], 1ull);
    c = __shfl_sync(FULL, c, 0);
    const unsigned long long gc = c * (unsigned long long)a.shard_count + (unsigned long long)a.shard_rank;
    if (gc >= nchunks) {
      exhausted++;
      p = (p + 1 == np) ? 0 : p + 1;
      continue;
    }
    exhausted = 0;
    if (PAGED && a.pf_off && p == 0) {
      // post the predicted pages of a chunk this warp's successors will reach
      const long long pc = (long long)gc + (long long)a.pf_ahead * a.shard_count;
      // only while the host's queue is short: a page posted behind a long
      // queue stays LOADING, and warps that miss on it meanwhile can neither
      // read it from a frame nor load it themselves
      unsigned long long queued = 0;
      if (lane == 0) queued = *(volatile unsigned long long*)a.pg.ring_head - *(volatile unsigned long long*)a.pg.host_tail;
      queued = __shfl_sync(FULL, queued, 0);  // one decision for the warp (the block below shuffles)
      if (pc < a.pf_chunks && queued < 64) {
        PageCounters lpc = {};
        for (int k = a.pf_off[pc] + lane; k < a.pf_off[pc + 1]; k += 32) {
          const int32_t pg = a.pf_pages[k];
          if (pg >= 0 && pg < a.pg.n_pages && ld_vol(&a.pg.page_frame[pg]) == PAGE_ABSENT) request_page(a.pg, pg, lpc);
        }
        unsigned long long v[3] = {lpc.requests, lpc.evictions, lpc.dropped};
#pragma unroll
        for (int q = 0; q < 3; q++)
          for (int o = 16; o; o >>= 1) v[q] += __shfl_xor_sync(FULL, v[q], o);
        w.pc.requests += v[0];
        w.pc.evictions += v[1];
        w.pc.dropped += v[2];
        w.prefetched += v[0];
      }
    }
    const long long rb = (long long)gc * a.chunk;
    const long long re = min((long long)P.nroots, rb + a.chunk);
    unsigned long long local = 0;
    for (long long r = rb; r < re && !w.err; r++) {
      // position r of the range; with an order, the order's entry there
      const long long pos = P.rbase + r;
      const long long rid = a.root_order ? (long long)a.root_order[pos] : pos;
      const int2 e = P.roots[rid];
      const unsigned long long b0 = w.bytes, r0 = w.reads;
      if (lane == 0) {
        S.path[0] = e.x;
        S.path[1] = e.y;
        S.split = (a.root_split && p == 0) ? a.root_split[rid] : a.split_min;
      }
      __syncwarp();
      const unsigned long long c0 = dfs_from<LABELED, PAGED>(a, P, S, 1, 0, -1, true, p, (int)rid, w);
      return_arena(a, S, own);
      local += c0;
      roots++;
      if (lane == 0 && p == 0) {
        if (a.root_counts) atomicAdd(&a.root_counts[rid], c0);
        if (a.root_cost) atomicAdd(&a.root_cost[rid], (float)(w.bytes - b0 + 8));
        if (a.root_reads) atomicAdd(&a.root_reads[rid], (float)(w.reads - r0));
      }
    }
    if (lane == 0 && local) atomicAdd(&a.counts[p], local);
    p = (p + 1 == np) ? 0 : p + 1;  // interleave plans chunk by chunk
  }
  // phase 2: drain donated ranges until no warp holds work
  __threadfence();
  if (lane == 0) atomicSub(a.active, 1u);
  __syncwarp();
  unsigned long long last_beat = 0, last_change = global_ns();
  const unsigned long long t_drain = last_change;
  unsigned long long busy_ns = 0;
  while (!w.err) {
    Donation item;
    if (take_donation(a, item)) {
      const unsigned long long t_item = global_ns();
      const DPlan& P = a.plans[item.plan];
      const int2 e = P.roots[item.root];
      if (lane == 0) {
        S.path[0] = e.x;
        S.path[1] = e.y;
        for (int k = 2; k <= item.level; k++) S.path[k] = item.path[k];
        S.split = (a.root_split && item.plan == 0) ? a.root_split[item.root] : a.split_min;
      }
      __syncwarp();
      const unsigned long long b0 = w.bytes, r0 = w.reads;
      const unsigned long long c0 = dfs_from<LABELED, PAGED>(a, P, S, item.level, item.begin, item.end, false,
                                                             item.plan, item.root, w);
      return_arena(a, S, own);
      if (lane == 0) {
        if (c0) atomicAdd(&a.counts[item.plan], c0);
        if (item.plan == 0) {
          if (a.root_counts) atomicAdd(&a.root_counts[item.root], c0);
          if (a.root_cost) atomicAdd(&a.root_cost[item.root], (float)(w.bytes - b0));
          if (a.root_reads) atomicAdd(&a.root_reads[item.root], (float)(w.reads - r0));
        }
        // no fence: a warp that reads this decrement before this warp's
        // donations can only leave early; this warp drains them itself
        atomicSub(a.active, 1u);
      }
      __syncwarp();
      last_change = global_ns();
      busy_ns += last_change - t_item;
      continue;
    }
    unsigned int act = 0;
    unsigned long long head = 0, tail = 0, beat = 0;
    // no fence between these reads: a stale pair can only make a warp leave
    // early, and the warp holding the work finishes (and drains) it itself
    if (lane == 0) {
      act = *((volatile unsigned int*)a.active);
      head = *((volatile unsigned long long*)a.don_head);
      tail = *((volatile unsigned long long*)a.don_tail);
      beat = *((volatile unsigned long long*)a.heartbeat);
    }
    act = __shfl_sync(FULL, act, 0);
    head = __shfl_sync(FULL, head, 0);
    tail = __shfl_sync(FULL, tail, 0);
    beat = __shfl_sync(FULL, beat, 0);
    if (act == 0 && tail >= head) break;
    // bounded wait: give up (and report DEV_TIMEOUT) when no warp has made
    // progress for timeout_ns
    const unsigned long long now = global_ns();
    if (beat != last_beat) { last_beat = beat; last_change = now; }
    else if (now - last_change > a.timeout_ns) {
      if (lane == 0) atomicOr(a.status, (unsigned)DEV_TIMEOUT);
      break;
    }
    __nanosleep(1000);
  }
  if (lane == 0) {
    const unsigned long long t_end = global_ns();
    atomicAdd(&a.stats[ST_WARP_NS], t_end - S.t_start);
    atomicAdd(&a.stats[ST_IDLE_NS], t_end - t_drain - min(busy_ns, t_end - t_drain));
    atomicAdd(&a.stats[ST_SETOPS], w.setops);
    atomicAdd(&a.stats[ST_BYTES], w.bytes + 8ull * roots);
    atomicAdd(&a.stats[ST_ROOTS], roots);
    if (w.borrows) atomicAdd(&a.stats[ST_BORROWS], w.borrows);
    atomicAdd(&a.stats[ST_LEAF_CYC], w.leaf_cyc);
    atomicAdd(&a.stats[ST_LEVEL_CYC], w.level_cyc);
    atomicAdd(&a.stats[ST_PREFIX_CYC], w.prefix_cyc);
    if (w.prefetched) atomicAdd(&a.stats[ST_PREFETCH], w.prefetched);
    if (PAGED) {
      atomicAdd(&a.stats[ST_HITS], w.pc.hits);
      atomicAdd(&a.stats[ST_MISSES], w.pc.misses);
      atomicAdd(&a.stats[ST_ZC_BYTES], w.pc.zc_bytes);
      atomicAdd(&a.stats[ST_REQUESTS], w.pc.requests);
      atomicAdd(&a.stats[ST_EVICTIONS], w.pc.evictions);
      atomicAdd(&a.stats[ST_DROPPED], w.pc.dropped);
      if (w.pc.dev_loads) {
        atomicAdd(&a.stats[ST_DEV_LOADS], w.pc.dev_loads);
        atomicAdd(&a.stats[ST_DEV_BYTES], w.pc.dev_bytes);
      }
    }
    if (w.err) atomicOr(a.status, w.err);
  }
}

// =====================================================================
// Root filter (restates JobQueuePreprocessor, src/job_queue.h:39-64, as
// three passes: per-vertex max neighbour degree, per-vertex root counts +
// scan, ordered write).  Root order = reference order (r ascending, then
// adjacency order), so root ids match the reference's Job[] indices.
// =====================================================================

__global__ void maxnbrdeg_kernel(const uint64_t* rowptr, const int32_t* colidx, int64_t n, int32_t* out) {
  const int lane = lane_id();
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long v = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); v < n; v += warps) {
    const uint64_t b = rowptr[v], e = rowptr[v + 1];
    int m = 0;
    for (uint64_t i = b + lane; i < e; i += 32) {
      const int u = colidx[i];
      m = max(m, (int)(rowptr[u + 1] - rowptr[u]));
    }
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(FULL, m, o));
    if (lane == 0) out[v] = m;
  }
}

// Regroups each list by label, keeping id order within a label (a stable
// partition): one warp per vertex, ranks from __match_any_sync.  Vertices
// [v_begin, v_end); entry i of the adjacency array lands at out[i - out_base].
__global__ void label_group_kernel(const uint64_t* rowptr, const int32_t* colidx, const uint8_t* labels,
                                   int64_t v_begin, int64_t v_end, int nl1, int32_t* out, uint64_t out_base,
                                   int32_t* off) {
  __shared__ int base_s[16][33];
  const int lane = lane_id();
  const int wib = threadIdx.x >> 5;
  int* base = base_s[wib];
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long v = v_begin + (long long)blockIdx.x * (blockDim.x >> 5) + wib; v < v_end; v += warps) {
    const uint64_t b = rowptr[v], e = rowptr[v + 1];
    // per-label counts: lane l counts label l
    int mine = 0;
    for (uint64_t i0 = b; i0 < e; i0 += 32) {
      const uint64_t i = i0 + lane;
      const int lb = i < e ? labels[colidx[i]] : -1;
      for (int l = 0; l < nl1 - 1; l++) {
        const unsigned bal = __ballot_sync(FULL, lb == l);
        if (lane == l) mine += __popc(bal);
      }
    }
    // exclusive scan over labels
    int incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    const int excl = incl - mine;
    if (lane < nl1 - 1) {
      off[v * nl1 + lane] = excl;
      base[lane] = excl;
    }
    if (lane == 0) off[v * nl1 + nl1 - 1] = (int)(e - b);  // up to 32 labels: entry 32 needs its own store
    __syncwarp();
    for (uint64_t i0 = b; i0 < e; i0 += 32) {
      const uint64_t i = i0 + lane;
      const bool valid = i < e;
      const int x = valid ? colidx[i] : 0;
      const int lb = valid ? (int)labels[x] : 32 + lane;  // invalid lanes match only themselves
      const unsigned same = __match_any_sync(FULL, lb);
      if (valid) out[b - out_base + base[lb] + __popc(same & lanemask_lt())] = x;
      __syncwarp();
      if (valid && (same & lanemask_lt()) == 0) base[lb] += __popc(same);
      __syncwarp();
    }
  }
}

struct RootFilter {
  int labeled;
  int need_gt;   // unlabeled with partial[0]==1: keep r > c only
  int lab0, lab1;
  int d0, d1, d2;
};

template <bool WRITE>
__global__ void roots_kernel(const uint64_t* rowptr, const int32_t* colidx, const uint8_t* labels,
                             const int32_t* maxnbrdeg, int64_t n, RootFilter f, int32_t* counts,
                             const int64_t* offsets, int2* out) {
  const int lane = lane_id();
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
    const uint64_t b = rowptr[r], e = rowptr[r + 1];
    int total = 0;
    const bool rok = (long long)(e - b) >= f.d0 && (!f.labeled || labels[r] == f.lab0);
    if (rok) {
      long long base = WRITE ? offsets[r] : 0;
      for (uint64_t i0 = b; i0 < e; i0 += 32) {
        const uint64_t i = i0 + lane;
        bool keep = false;
        if (i < e) {
          const int c = colidx[i];
          keep = (!f.need_gt || r > c) && (!f.labeled || labels[c] == f.lab1) &&
                 (int)(rowptr[c + 1] - rowptr[c]) >= f.d1 && maxnbrdeg[c] >= f.d2;
        }
        const unsigned bal = __ballot_sync(FULL, keep);
        if (WRITE && keep) out[base + total + __popc(bal & lanemask_lt())] = make_int2((int)r, colidx[i]);
        total += __popc(bal);
      }
    }
    if (!WRITE && lane == 0) counts[r] = total;
  }
}

// =====================================================================
// Host glue
// =====================================================================

namespace {

void free_dev(void* p) { if (p) cudaFree(p); }

pm_status ensure(void** p, size_t* have, size_t want) {
  if (*have >= want && *p) return PM_OK;
  free_dev(*p);
  *p = nullptr;
  *have = 0;
  if (want == 0) return PM_OK;
  cudaError_t e = cudaMalloc(p, want);
  if (e != cudaSuccess) {
    *p = nullptr;
    return fail(PM_ERR_OOM, "cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
  }
  *have = want;
  return PM_OK;
}

pm_status check_device(int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return fail(PM_ERR_NO_DEVICE, "no CUDA device available (%s); libpumatch_b200 has no CPU path",
                e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
  if (device < 0 || device >= count) return fail(PM_ERR_INVALID, "device %d out of range", device);
  CK(cudaSetDevice(device));
  return PM_OK;
}

DPlan to_dplan(const Plan& p) {
  DPlan d;
  memset(&d, 0, sizeof(d));
  d.nnodes = p.nnodes;
  d.nslots = p.nslots;
  d.labeled = p.labeled;
  d.last_slot = p.level_begin[p.nnodes - 2];
  for (int i = 0; i <= PM_MAX_PAT; i++) d.level_begin[i] = p.level_begin[i];
  for (int s = 0; s < 16; s++) d.alias[s] = -1;
  for (int s = 0; s < p.nslots; s++) {
    d.slot_labels[s] = p.slot_labels[s];
    d.partial[s] = p.partial[s];
    d.kind[s] = (uint8_t)slot_kind(p.set_ops[s]);
    d.parent[s] = (uint8_t)slot_parent(p.set_ops[s]);
  }
  // Slots of one level with the same operation, operands, labels and partial
  // order differ only in how their bound combines the constrained path
  // vertices: the main slot takes the smallest, helpers the largest.  A
  // helper equal to an earlier helper is that helper; the main slot is the
  // prefix of such a helper below its own (smaller) bound -- also under
  // truncation, since both keep their first survivors in the same order.
  for (int L = 1; L + 2 < p.nnodes; L++) {
    const int b = p.level_begin[L], e = p.level_begin[L + 1];
    for (int i = b + 1; i <= e; i++) {
      const int s = (i == e) ? b : i;  // helpers first, the main slot last
      for (int t = b + 1; t < e; t++) {
        if (t == s || (s != b && t >= s)) continue;
        if (p.set_ops[s] != p.set_ops[t] || p.slot_labels[s] != p.slot_labels[t] || p.partial[s] != p.partial[t])
          continue;
        if (d.alias[t] >= 0) continue;  // alias a computed slot only
        d.alias[s] = (int8_t)t;
        d.alias_prefix[s] = (s == b) ? 1 : 0;
        break;
      }
    }
  }
  // Shape for lane_subtree (unlabeled): level n-3 is one intersection X with
  // a parent at an earlier level, plus at most one alias Y of it; the last
  // slot intersects with X or Y.
  d.l2_x = d.l2_y = -1;
  const int n = p.nnodes;
  if (!p.labeled && n >= 5) {
    const int b = p.level_begin[n - 3], e = p.level_begin[n - 2];
    int x = -1, y = -1, others = 0;
    for (int s = b; s < e; s++) {
      if (d.alias[s] < 0) { if (x < 0) x = s; else others++; }
      else if (y < 0) y = s;
      else others++;
    }
    const int last = d.last_slot;
    if (x >= 0 && !others && (y < 0 || d.alias[y] == x) && d.kind[x] == SLOT_INTERSECT && d.parent[x] < b &&
        d.kind[last] == SLOT_INTERSECT && (d.parent[last] == x || (y >= 0 && d.parent[last] == y))) {
      d.l2_x = (int8_t)x;
      d.l2_y = (int8_t)y;
    }
  }
  return d;
}

RootFilter to_filter(const Plan& p) {
  RootFilter f;
  f.labeled = p.labeled;
  f.need_gt = (!p.labeled && p.partial[0] == 1);
  f.lab0 = p.vertex_label[0];
  f.lab1 = p.vertex_label[1];
  f.d0 = p.degree[0];
  f.d1 = p.degree[1];
  f.d2 = p.degree[2];
  return f;
}

// Parent-set limit of the two-level lane scheme from the run options: 0 =
// default (64), negative = never, else capped at the shared staging size.
int lane_subtree_limit(const pm_run_opts& o) {
  return o.lane_subtree_max < 0 ? 0 : (o.lane_subtree_max == 0 ? 64 : std::min(o.lane_subtree_max, PM_SB_MAX));
}

// Worst-case arena words one warp needs for a plan: every materialised slot
// is at most its first operand, itself at most a max-degree list.
int64_t arena_words_for(const Plan& p, int32_t maxdeg, int T) {
  const int64_t per = (T > 0) ? std::min<int64_t>(maxdeg, T) : maxdeg;
  const int materialised = p.nslots - 2;  // minus the root slot and the counted last slot
  return std::max<int64_t>(materialised, 1) * per + 64;
}

}  // namespace

namespace pm {
// Fills g->d_maxnbrdeg from an adjacency array the device can read (HBM or
// mapped host memory).
pm_status compute_maxnbrdeg(pm_graph* g, const int32_t* colidx) {
  if (g->n > 0) {
    PM_CK_PENDING("max neighbour degree");
    maxnbrdeg_kernel<<<2048, 256>>>(g->d_rowptr, colidx, g->n, g->d_maxnbrdeg);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
  }
  return PM_OK;
}
}  // namespace pm

static pm_status graph_finish(pm_graph* g) {
  // per-vertex max neighbour degree, used by the root filter
  CK(cudaMalloc(&g->d_maxnbrdeg, sizeof(int32_t) * std::max<int64_t>(g->n, 1)));
  g->device_bytes += sizeof(int32_t) * g->n;
  if (g->n > 0 && g->residency == PM_RESIDENT_HBM) {
    PM_CK_PENDING("max neighbour degree");
    maxnbrdeg_kernel<<<2048, 256>>>(g->d_rowptr, g->d_colidx, g->n, g->d_maxnbrdeg);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
  }
  if (g->labeled && g->residency == PM_RESIDENT_HBM && g->n > 0) {
    g->nl1 = (g->nlabels > 0 ? g->nlabels : 32) + 1;
    CK(cudaMalloc(&g->d_colidx_lab, sizeof(int32_t) * std::max<int64_t>(g->nadj, 1)));
    CK(cudaMalloc(&g->d_lab_off, sizeof(int32_t) * (size_t)g->n * g->nl1));
    g->device_bytes += sizeof(int32_t) * ((size_t)g->nadj + (size_t)g->n * g->nl1);
    PM_CK_PENDING("label grouping");
    label_group_kernel<<<2048, 256>>>(g->d_rowptr, g->d_colidx, g->d_labels, 0, g->n, g->nl1, g->d_colidx_lab, 0,
                                      g->d_lab_off);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
  }
  return PM_OK;
}

// Labeled paged graphs: the label-grouped copy of the adjacency array goes to
// pinned host memory (it is what the frames cache), the group offsets to the
// device.  Grouped on the device from the id-sorted array (h_colidx_dev), a
// vertex range at a time through a bounded device buffer.  With keep_copy
// false only the offsets are kept: the caller's source holds the grouped
// layout already (pm_graph_from_paged_source).
static pm_status paged_group_labels(pm_graph* g, const uint64_t* h_rowptr, bool keep_copy = true) {
  g->nl1 = (g->nlabels > 0 ? g->nlabels : 32) + 1;
  if (keep_copy) {
    CK(cudaHostAlloc((void**)&g->h_colidx_lab, sizeof(int32_t) * std::max<int64_t>(g->nadj, 1),
                     cudaHostAllocMapped | cudaHostAllocPortable));
    CK(cudaHostGetDevicePointer((void**)&g->h_colidx_lab_dev, g->h_colidx_lab, 0));
  }
  CK(cudaMalloc(&g->d_lab_off, sizeof(int32_t) * (size_t)std::max<int64_t>(g->n, 1) * g->nl1));
  g->device_bytes += sizeof(int32_t) * (size_t)g->n * g->nl1;
  const int64_t chunk = std::max<int64_t>(g->maxdeg, std::min<int64_t>(std::max<int64_t>(g->nadj, 1), 64ll << 20));
  int32_t* tmp = nullptr;
  PM_CK_PENDING("label grouping");
  CK(cudaMalloc(&tmp, sizeof(int32_t) * (size_t)std::max<int64_t>(chunk, 1)));
  pm_status st = PM_OK;
  for (int64_t v0 = 0; v0 < g->n && st == PM_OK;) {
    int64_t v1 = v0;
    while (v1 < g->n && (int64_t)(h_rowptr[v1 + 1] - h_rowptr[v0]) <= chunk) v1++;
    const uint64_t b0 = h_rowptr[v0], len = h_rowptr[v1] - b0;
    label_group_kernel<<<2048, 256>>>(g->d_rowptr, g->h_colidx_dev, g->d_labels, v0, v1, g->nl1, tmp, b0,
                                      g->d_lab_off);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && len && keep_copy)
      e = cudaMemcpy(g->h_colidx_lab + b0, tmp, sizeof(int32_t) * len, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && !keep_copy) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) st = fail(PM_ERR_CUDA, "label grouping: %s", cudaGetErrorString(e));
    v0 = v1;
  }
  cudaFree(tmp);
  if (st != PM_OK) return st;
  if (keep_copy) {
    g->h_paged = g->h_colidx_lab;
    g->h_paged_dev = g->h_colidx_lab_dev;
  }
  return PM_OK;
}

namespace pm {
pm_status paged_place(pm_graph* g, const int32_t* colidx, const pm_graph_opts* o, const int32_t* src_dev);
pm_status paged_maxnbrdeg(pm_graph* g);
void paged_release(pm_graph* g);
pm_status paged_prepare(pm_ctx* ctx, pm_graph* g, bool cold, DPaging* out);
pm_status paged_service_start(pm_ctx* ctx, pm_graph* g);
pm_status paged_service_stop(pm_ctx* ctx, pm_graph* g, pm_stats* st);
int64_t paged_static_frames(const pm_graph* g);
}  // namespace pm

extern "C" void pm_graph_opts_default(pm_graph_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->labeled = 0;
  o->device = 0;
  o->residency = PM_RESIDENT_HBM;
  o->page_bytes = 64 * 1024;
  o->frame_pool_bytes = 4ull << 30;
}

// The row offsets and labels of a graph placed from host arrays, on the
// device (every residency).
static pm_status place_rows(pm_graph* g, int64_t n, int64_t nadj, const uint64_t* rowptr, const uint32_t* labels,
                            const pm_graph_opts& o) {
  g->device = o.device;
  g->n = n;
  g->nadj = nadj;
  g->labeled = o.labeled ? 1 : 0;
  g->residency = o.residency;
  int32_t maxd = 0;
  for (int64_t v = 0; v < n; v++) maxd = std::max<int32_t>(maxd, (int32_t)(rowptr[v + 1] - rowptr[v]));
  g->maxdeg = maxd;
  CK(cudaMalloc(&g->d_rowptr, sizeof(uint64_t) * (n + 1)));
  CK(cudaMemcpy(g->d_rowptr, rowptr, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice));
  g->device_bytes += sizeof(uint64_t) * (n + 1);
  if (g->labeled) {
    std::vector<uint8_t> lab((size_t)std::max<int64_t>(n, 1));
    int nl = 0;
    for (int64_t v = 0; v < n; v++) {
      if (labels[v] >= 32) return fail(PM_ERR_FORMAT, "label %u of vertex %lld >= 32", labels[v], (long long)v);
      lab[v] = (uint8_t)labels[v];
      nl = std::max<int>(nl, (int)labels[v] + 1);
    }
    g->nlabels = nl;
    CK(cudaMalloc(&g->d_labels, std::max<int64_t>(n, 1)));
    CK(cudaMemcpy(g->d_labels, lab.data(), n, cudaMemcpyHostToDevice));
    g->device_bytes += n;
  }
  return PM_OK;
}

extern "C" pm_status pm_graph_from_host(int64_t n, int64_t nadj, const uint64_t* rowptr, const int32_t* colidx,
                                        const uint32_t* labels, const pm_graph_opts* opts, pm_graph** out) {
  if (!rowptr || (nadj > 0 && !colidx) || !out || n < 0 || n > INT32_MAX - 1)
    return fail(PM_ERR_INVALID, "pm_graph_from_host: bad arguments");
  pm_graph_opts o;
  pm_graph_opts_default(&o);
  if (opts) o = *opts;
  pm_status st = check_device(o.device);
  if (st != PM_OK) return st;
  if (o.labeled && !labels) return fail(PM_ERR_INVALID, "labeled graph without labels");
  std::unique_ptr<pm_graph> g(new pm_graph);
  st = place_rows(g.get(), n, nadj, rowptr, labels, o);
  if (st != PM_OK) return st;
  if (o.residency == PM_RESIDENT_PAGED) {
    st = paged_place(g.get(), colidx, &o, nullptr);
    if (st != PM_OK) return st;
    CK(cudaMalloc(&g->d_maxnbrdeg, sizeof(int32_t) * std::max<int64_t>(g->n, 1)));
    g->device_bytes += sizeof(int32_t) * g->n;
    st = paged_maxnbrdeg(g.get());
    if (st != PM_OK) return st;
    if (g->labeled && n > 0) {
      st = paged_group_labels(g.get(), rowptr);
      if (st != PM_OK) return st;
    }
  } else {
    CK(cudaMalloc(&g->d_colidx, sizeof(int32_t) * std::max<int64_t>(nadj, 1)));
    if (nadj) CK(cudaMemcpy(g->d_colidx, colidx, sizeof(int32_t) * nadj, cudaMemcpyHostToDevice));
    g->device_bytes += sizeof(int32_t) * nadj;
    st = graph_finish(g.get());
    if (st != PM_OK) return st;
  }
  *out = g.release();
  return PM_OK;
}

extern "C" pm_status pm_graph_from_paged_source(int64_t n, int64_t nadj, const uint64_t* rowptr,
                                                const uint32_t* labels, const int32_t* src, const int32_t* sorted,
                                                const pm_graph_opts* opts, pm_graph** out) {
  if (!rowptr || !out || n < 0 || n > INT32_MAX - 1 || nadj < 0 || (nadj > 0 && !src))
    return fail(PM_ERR_INVALID, "pm_graph_from_paged_source: bad arguments");
  pm_graph_opts o;
  pm_graph_opts_default(&o);
  if (opts) o = *opts;
  o.residency = PM_RESIDENT_PAGED;
  if (o.labeled && (!labels || (nadj > 0 && !sorted)))
    return fail(PM_ERR_INVALID, "a labeled graph needs labels and the id-sorted array");
  if (!o.labeled) sorted = src;
  if (rowptr[n] != (uint64_t)nadj)
    return fail(PM_ERR_INVALID, "rowptr[n] = %llu but n_adj = %lld", (unsigned long long)rowptr[n], (long long)nadj);
  if (((uintptr_t)src & 15) || ((uintptr_t)sorted & 15))
    return fail(PM_ERR_INVALID, "the source arrays must be 16-byte aligned");
  pm_status st = check_device(o.device);
  if (st != PM_OK) return st;
  std::unique_ptr<pm_graph> g(new pm_graph);
  st = place_rows(g.get(), n, nadj, rowptr, labels, o);
  if (st != PM_OK) return st;
  st = paged_place(g.get(), nullptr, &o, src);
  if (st != PM_OK) return st;
  // the id-sorted lists: root filter, features, and a labeled graph's whole
  // lists (read in place)
  g->h_colidx_dev = const_cast<int32_t*>(sorted);
  CK(cudaMalloc(&g->d_maxnbrdeg, sizeof(int32_t) * std::max<int64_t>(g->n, 1)));
  g->device_bytes += sizeof(int32_t) * g->n;
  st = paged_maxnbrdeg(g.get());
  if (st != PM_OK) return st;
  if (g->labeled && n > 0) {
    st = paged_group_labels(g.get(), rowptr, false);
    if (st != PM_OK) return st;
  }
  *out = g.release();
  return PM_OK;
}

extern "C" pm_status pm_graph_from_device(int64_t n, int64_t nadj, int32_t maxdeg, const uint64_t* d_rowptr,
                                          const int32_t* d_colidx, const uint8_t* d_labels, int device,
                                          pm_graph** out) {
  if (!d_rowptr || (nadj > 0 && !d_colidx) || !out || n < 0 || maxdeg < 0)
    return fail(PM_ERR_INVALID, "pm_graph_from_device: bad arguments");
  pm_status st = check_device(device);
  if (st != PM_OK) return st;
  std::unique_ptr<pm_graph> g(new pm_graph);
  g->device = device;
  g->n = n;
  g->nadj = nadj;
  g->maxdeg = maxdeg;
  g->labeled = d_labels != nullptr;
  g->nlabels = d_labels ? 32 : 0;
  g->owns = false;
  g->d_rowptr = const_cast<uint64_t*>(d_rowptr);
  g->d_colidx = const_cast<int32_t*>(d_colidx);
  g->d_labels = const_cast<uint8_t*>(d_labels);
  st = graph_finish(g.get());
  if (st != PM_OK) return st;
  *out = g.release();
  return PM_OK;
}

extern "C" pm_status pm_graph_open(const char* prefix, const pm_graph_opts* opts, pm_graph** out) {
  pm_graph_opts o;
  pm_graph_opts_default(&o);
  if (opts) o = *opts;
  int64_t n = 0, nadj = 0;
  int32_t maxd = 0;
  uint64_t* rowptr = nullptr;
  int32_t* colidx = nullptr;
  uint32_t* labels = nullptr;
  pm_status st = pm_graph_read(prefix, o.labeled, &n, &nadj, &maxd, &rowptr, &colidx, &labels);
  if (st != PM_OK) return st;
  st = pm_graph_from_host(n, nadj, rowptr, colidx, labels, &o, out);
  free(rowptr);
  free(colidx);
  free(labels);
  return st;
}

extern "C" pm_status pm_graph_get_info(const pm_graph* g, pm_graph_info* info) {
  if (!g || !info) return fail(PM_ERR_INVALID, "pm_graph_get_info: null argument");
  memset(info, 0, sizeof(*info));
  info->n_vertices = g->n;
  info->n_adj = g->nadj;
  info->max_degree = g->maxdeg;
  info->labeled = g->labeled;
  info->n_labels = g->nlabels;
  info->residency = g->residency;
  info->device_bytes = g->device_bytes;
  info->n_pages = (uint64_t)g->n_pages;
  info->n_frames = (uint64_t)g->n_frames;
  info->n_static_frames = (uint64_t)paged_static_frames(g);
  return PM_OK;
}

extern "C" void pm_graph_close(pm_graph* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->owns) {
    free_dev(g->d_rowptr);
    free_dev(g->d_colidx);
    free_dev(g->d_labels);
  }
  free_dev(g->d_maxnbrdeg);
  free_dev(g->d_colidx_lab);
  free_dev(g->d_lab_off);
  paged_release(g);
  delete g;
}

extern "C" pm_status pm_ctx_create(int device, pm_ctx** out) {
  if (!out) return fail(PM_ERR_INVALID, "pm_ctx_create: null argument");
  pm_status st = check_device(device);
  if (st != PM_OK) return st;
  std::unique_ptr<pm_ctx> c(new pm_ctx);
  c->device = device;
  CK(cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
  CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  for (auto& e : c->ev) CK(cudaEventCreate(&e));
  *out = c.release();
  return PM_OK;
}

extern "C" void* pm_ctx_stream(pm_ctx* c) { return c ? (void*)c->stream : nullptr; }

extern "C" void pm_ctx_destroy(pm_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaStreamSynchronize(c->copy_stream);
  free_dev(c->d_arena);
  free_dev(c->d_ctl);
  free_dev(c->d_roots);
  free_dev(c->d_tmp);
  free_dev(c->d_vcount);
  free_dev(c->d_voff);
  for (auto& e : c->ev) if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  delete c;
}

extern "C" void pm_run_opts_default(pm_run_opts* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->root_begin = -1;
  o->root_end = -1;
}

// Builds the root list of plan p into ctx->d_roots + offset; returns count.
static pm_status build_roots(pm_ctx* c, const pm_graph* g, const Plan& p, size_t offset_roots,
                             int64_t* count, bool count_only, int2** roots_buf = nullptr,
                             size_t* roots_bytes = nullptr) {
  if (!roots_buf) { roots_buf = &c->d_roots; roots_bytes = &c->roots_bytes; }
  const int64_t n = g->n;
  if (n == 0) { *count = 0; return PM_OK; }
  if (c->vbuf_n < (size_t)n + 1) {
    free_dev(c->d_vcount);
    free_dev(c->d_voff);
    c->d_vcount = nullptr;
    c->d_voff = nullptr;
    c->vbuf_n = 0;
    CK(cudaMalloc(&c->d_vcount, sizeof(int32_t) * (n + 1)));
    CK(cudaMalloc(&c->d_voff, sizeof(int64_t) * (n + 1)));
    c->vbuf_n = (size_t)n + 1;
  }
  const RootFilter f = to_filter(p);
  const int32_t* colidx = g->residency == PM_RESIDENT_HBM ? g->d_colidx : g->h_colidx_dev;
  PM_CK_PENDING("root filter");
  roots_kernel<false><<<4 * c->nsm, 256, 0, c->stream>>>(g->d_rowptr, colidx, g->d_labels, g->d_maxnbrdeg, n, f,
                                                          c->d_vcount, nullptr, nullptr);
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(c->d_vcount + n, 0, sizeof(int32_t), c->stream));
  size_t need = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, need, c->d_vcount, c->d_voff, n + 1, c->stream));
  pm_status st = ensure(&c->d_tmp, &c->tmp_bytes, need);
  if (st != PM_OK) return st;
  CK(cub::DeviceScan::ExclusiveSum(c->d_tmp, need, c->d_vcount, c->d_voff, n + 1, c->stream));
  int64_t total = 0;
  CK(cudaMemcpyAsync(&total, c->d_voff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *count = total;
  if (count_only) return PM_OK;
  const size_t want = sizeof(int2) * (offset_roots + (size_t)total) + sizeof(int2);
  if (*roots_bytes < want) {
    // grow, keeping the roots of earlier plans
    int2* nr = nullptr;
    CK(cudaMalloc(&nr, want + want / 4));
    if (*roots_buf && offset_roots)
      CK(cudaMemcpyAsync(nr, *roots_buf, sizeof(int2) * offset_roots, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    free_dev(*roots_buf);
    *roots_buf = nr;
    *roots_bytes = want + want / 4;
  }
  PM_CK_PENDING("root filter");
  roots_kernel<true><<<4 * c->nsm, 256, 0, c->stream>>>(g->d_rowptr, colidx, g->d_labels, g->d_maxnbrdeg, n, f,
                                                         nullptr, c->d_voff, *roots_buf + offset_roots);
  CK(cudaGetLastError());
  return PM_OK;
}

extern "C" pm_status pm_count_roots(pm_ctx* c, const pm_graph* g, const pm_plan* ph, int64_t* n_roots) {
  if (!c || !g || !ph || !n_roots) return fail(PM_ERR_INVALID, "pm_count_roots: null argument");
  const Plan& p = *plan_of(ph);
  if (p.labeled && !g->labeled) return fail(PM_ERR_INVALID, "labeled plan on an unlabeled graph");
  CK(cudaSetDevice(c->device));
  return build_roots(c, g, p, 0, n_roots, true);
}

namespace pm {
// Root list of one plan in the context's root buffer (valid until the next
// call that builds roots on this context).
pm_status root_list_for(pm_ctx* c, const pm_graph* g, const pm_plan* ph, const int2** roots, int64_t* n) {
  const Plan* p = plan_of(ph);
  if (p->labeled && !g->labeled) return fail(PM_ERR_INVALID, "labeled plan on an unlabeled graph");
  CK(cudaSetDevice(c->device));
  pm_status st = build_roots(c, g, *p, 0, n, false);
  if (st != PM_OK) return st;
  CK(cudaStreamSynchronize(c->stream));
  *roots = c->d_roots;
  return PM_OK;
}

// Exposed for tests through pm_debug_roots: copies the root list of one plan.
pm_status debug_roots(pm_ctx* c, const pm_graph* g, const Plan& p, int32_t* out_pairs, int64_t cap, int64_t* count) {
  pm_status st = build_roots(c, g, p, 0, count, false);
  if (st != PM_OK) return st;
  const int64_t m = std::min<int64_t>(cap, *count);
  if (m > 0) CK(cudaMemcpyAsync(out_pairs, c->d_roots, sizeof(int2) * m, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PM_OK;
}
}  // namespace pm

extern "C" pm_status pm_debug_roots(pm_ctx* c, const pm_graph* g, const pm_plan* ph, int32_t* out_pairs,
                                    int64_t cap, int64_t* count) {
  if (!c || !g || !ph || !count) return fail(PM_ERR_INVALID, "pm_debug_roots: null argument");
  CK(cudaSetDevice(c->device));
  return debug_roots(c, g, *plan_of(ph), out_pairs, cap, count);
}

// One prepared persistent launch: plans, roots, geometry, kernel arguments.
struct Launch {
  bool labeled = false, paged = false, cold = false, host_copy = false;
  int64_t n_big = 0;          // borrowed arenas
  size_t own_bytes = 0, big_bytes = 0;
  int nplans = 0;
  const Plan* plans[PM_MAX_BATCH];
  DPlan dp[PM_MAX_BATCH];
  MatchArgs a;
  int blocks = 0, threads = 0;
  size_t smem = 0;
  void (*kfn)(const MatchArgs) = nullptr;
  int64_t warps = 0;
  size_t ctl_words = 0;
  unsigned int active0 = 0;  // initial active-warp count (host staging)
};

static constexpr unsigned kDonSlots = 1u << 15;
// a warp's own arena: at most this many slot words and gather words
static constexpr int64_t kOwnSlotWords = 1 << 16;
static constexpr int64_t kOwnGatherWords = 1 << 15;
static constexpr size_t kBigPoolMaxBytes = 48ull << 30;
static constexpr int kCtlRead = 32 + 32 + kStatWords + 1;  // cursors, counts, stats, status word

// Validates the plans and options, builds the root lists into *roots,
// sizes the persistent grid and the arenas, and fills L.  Buffers are grown
// as needed (they belong to the caller: the context for pm_match, the query
// for pm_query_prepare).
static pm_status setup_launch(pm_ctx* c, const pm_graph* g, const pm_plan* const* plans, int nplans,
                              const pm_run_opts& o, int2** roots, size_t* roots_bytes, int32_t** arena,
                              size_t* arena_bytes, unsigned long long** ctl, size_t* ctl_bytes, Launch* L) {
  if (nplans < 1 || nplans > PM_MAX_BATCH) return fail(PM_ERR_INVALID, "between 1 and %d plans per launch", PM_MAX_BATCH);
  CK(cudaSetDevice(c->device));
  L->labeled = plan_of(plans[0]) && plan_of(plans[0])->labeled != 0;
  for (int i = 0; i < nplans; i++) {
    const Plan* p = plan_of(plans[i]);
    if (!p) return fail(PM_ERR_INVALID, "null plan %d", i);
    if ((p->labeled != 0) != L->labeled) return fail(PM_ERR_INVALID, "plans mix labeled and unlabeled modes");
    if (p->labeled && !g->labeled) return fail(PM_ERR_INVALID, "labeled plan on an unlabeled graph");
    L->plans[i] = p;
  }
  L->nplans = nplans;
  if (o.root_order && nplans != 1) return fail(PM_ERR_INVALID, "root_order needs a single plan");
  const int T = std::max(0, o.truncate);
  const int wpb = o.warps_per_block > 0 ? o.warps_per_block : 8;
  if (wpb > 16 || (wpb & (wpb - 1))) return fail(PM_ERR_INVALID, "warps_per_block must be 1,2,4,8 or 16");
  const int chunk = o.chunk > 0 ? o.chunk : 16;
  const int shard_count = o.shard_count > 1 ? o.shard_count : 1;
  if (o.shard_rank < 0 || o.shard_rank >= shard_count) return fail(PM_ERR_INVALID, "bad shard_rank");
  L->paged = g->residency == PM_RESIDENT_PAGED;
  L->cold = o.cold_cache != 0;
  L->host_copy = o.host_page_copy != 0;

  // root lists, concatenated
  size_t off = 0;
  int64_t arena_words = 64;
  for (int i = 0; i < nplans; i++) {
    const Plan& p = *L->plans[i];
    int64_t cnt = 0;
    pm_status st = build_roots(c, g, p, off, &cnt, false, roots, roots_bytes);
    if (st != PM_OK) return st;
    L->dp[i] = to_dplan(p);
    L->dp[i].nroots = cnt;
    arena_words = std::max(arena_words, arena_words_for(p, g->maxdeg, T));
    off += (size_t)cnt;
  }
  off = 0;
  for (int i = 0; i < nplans; i++) {
    int64_t b = 0, e = L->dp[i].nroots;
    if (o.root_begin >= 0) b = std::min<int64_t>(o.root_begin, e);
    if (o.root_end >= 0) e = std::min<int64_t>(o.root_end, e);
    if (e < b) e = b;
    L->dp[i].roots = *roots + off;
    off += (size_t)L->dp[i].nroots;
    L->dp[i].nroots = e - b;
    L->dp[i].rbase = b;
  }
  // Candidate storage.  worst_* hold every materialised slot at its largest
  // possible size (and, paged, two gathered max-degree lists); each warp's own
  // arena holds that when it is small, else a bounded part of it, and warps
  // that outgrow theirs borrow one of a pool of worst-case arenas.
  const int64_t worst_slots = arena_words;
  const int64_t worst_gather =
      L->paged ? ((std::max<int64_t>(2 * (int64_t)g->maxdeg + 64, 32 * PM_LANE_MAX) + 1) & ~1ll) : 0;
  const int64_t own_slots = std::min<int64_t>(worst_slots, o.own_arena_words > 0 ? o.own_arena_words : kOwnSlotWords);
  const int64_t own_gather =
      L->paged ? ((std::max<int64_t>(std::min<int64_t>(worst_gather, kOwnGatherWords), 32 * PM_LANE_MAX) + 1) & ~1ll)
               : 0;
  const bool borrowing = own_slots < worst_slots || own_gather < worst_gather;
  const int64_t slot_words = own_slots;
  arena_words = own_slots + own_gather;

  // launch geometry: persistent, occupancy-limited
  L->threads = wpb * 32;
  L->smem = sizeof(WarpState) * wpb;
  // kernel variant by register cap: 85 registers (three 256-thread blocks per
  // SM) measures fastest; 16-warp blocks need the uncapped variant
  int variant = o.high_occupancy;
  if (variant == 0) variant = (wpb <= 8) ? 2 : 3;
  if (variant < 0 || variant > 3) return fail(PM_ERR_INVALID, "high_occupancy must be 0..3");
  if ((variant == 1 || variant == 2) && wpb > 8)
    return fail(PM_ERR_INVALID, "warps_per_block 16 needs the uncapped kernel variant (high_occupancy 3)");
  if (variant == 1) {
    L->kfn = L->labeled ? (L->paged ? match_kernel<true, true, 4> : match_kernel<true, false, 4>)
                        : (L->paged ? match_kernel<false, true, 4> : match_kernel<false, false, 4>);
  } else if (variant == 2) {
    L->kfn = L->labeled ? (L->paged ? match_kernel<true, true, 3> : match_kernel<true, false, 3>)
                        : (L->paged ? match_kernel<false, true, 3> : match_kernel<false, false, 3>);
  } else {
    L->kfn = L->labeled ? (L->paged ? match_kernel<true, true, 1> : match_kernel<true, false, 1>)
                        : (L->paged ? match_kernel<false, true, 1> : match_kernel<false, false, 1>);
  }
  int per_sm = 0;
  // per-warp state is ~4 KB: 16-warp blocks need more than the default 48 KB
  CK(cudaFuncSetAttribute(L->kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L->smem));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, L->kfn, L->threads, L->smem));
  if (o.blocks_per_sm > 0) per_sm = std::min(per_sm, o.blocks_per_sm);
  per_sm = std::max(per_sm, 1);
  L->blocks = c->nsm * per_sm;
  L->warps = (int64_t)L->blocks * wpb;
  // keep the arenas within half of the free memory by trimming resident warps
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  free_b += *arena_bytes;
  while (L->blocks > c->nsm && (size_t)(L->warps * arena_words * 4) > free_b / 2) {
    L->blocks -= c->nsm;
    L->warps = (int64_t)L->blocks * wpb;
  }
  // borrowed arenas: as many as a quarter of the free memory holds (capped),
  // at least one, at most one per warp
  const int64_t big_words = borrowing ? worst_slots + worst_gather : 0;
  int64_t n_big = 0;
  if (borrowing) {
    const size_t own_b = (size_t)(L->warps * arena_words * 4);
    const size_t room = free_b / 2 > own_b ? free_b / 2 - own_b : 0;
    const size_t budget = std::min(room / 2, kBigPoolMaxBytes);
    n_big = std::max<int64_t>(1, std::min<int64_t>(L->warps, (int64_t)(budget / ((size_t)big_words * 4))));
    if (o.max_borrowed > 0) n_big = std::min<int64_t>(n_big, o.max_borrowed);
  }
  const size_t own_bytes = (size_t)(L->warps * arena_words * 4);
  const size_t big_bytes = (size_t)n_big * (size_t)big_words * 4;
  pm_status st = ensure((void**)arena, arena_bytes, own_bytes + big_bytes + 4 * (size_t)n_big + 256);
  if (st != PM_OK) return st;
  L->n_big = n_big;
  L->own_bytes = own_bytes;
  L->big_bytes = big_bytes;
  // control block: cursors[32] counts[32] stats[16] status/active head tail
  // heartbeat, donation ready[] and items[]
  L->ctl_words = 32 + 32 + kStatWords + 8 + kDonSlots + 6 * kDonSlots;
  st = ensure((void**)ctl, ctl_bytes, L->ctl_words * 8);
  if (st != PM_OK) return st;

  MatchArgs& a = L->a;
  memset(&a, 0, sizeof(a));
  a.rowptr = g->d_rowptr;
  a.colidx = g->d_colidx;
  a.labels = g->d_labels;
  a.colidx_lab = g->d_colidx_lab;
  a.lab_off = g->d_lab_off;
  a.host_sorted = (g->residency == PM_RESIDENT_PAGED && g->d_lab_off) ? g->h_colidx_dev : nullptr;
  a.leaf_flat = o.leaf_per_lane == 1 ? 0 : (o.leaf_per_lane == 2 ? 2 : 1);
  a.lane_subtree_max = lane_subtree_limit(o);
  a.nl1 = g->nl1;
  a.n = (int32_t)g->n;
  a.nplans = nplans;
  a.T = T;
  a.chunk = chunk;
  a.shard_rank = o.shard_rank;
  a.shard_count = shard_count;
  a.split_min = o.split_level1 == 0 ? 64 : (o.split_level1 < 0 ? 0 : o.split_level1);
  a.maxdeg = g->maxdeg;
  unsigned long long* w = *ctl;
  a.cursors = w; w += 32;
  a.counts = w; w += 32;
  a.stats = w; w += kStatWords;
  a.status = (unsigned int*)w;
  a.active = (unsigned int*)w + 1; w += 1;
  a.don_head = w; w += 1;
  a.don_tail = w; w += 1;
  a.heartbeat = w; w += 5;
  a.don_ready = w; w += kDonSlots;
  a.don_items = (int4*)w; w += 6 * kDonSlots;
  a.don_mask = kDonSlots - 1;
  a.total_warps = (unsigned int)L->warps;
  a.arena = *arena;
  a.arena_words = arena_words;
  a.slot_words = slot_words;
  a.gather_words = arena_words - slot_words;
  a.n_big = (int32_t)n_big;
  a.big_arena = n_big ? (int32_t*)((char*)*arena + own_bytes) : nullptr;
  a.big_slot_words = worst_slots;
  a.big_gather_words = worst_gather;
  a.big_owner = n_big ? (unsigned int*)((char*)*arena + own_bytes + big_bytes) : nullptr;
  a.root_counts = (unsigned long long*)o.root_counts;
  a.root_cost = o.root_cost;
  a.root_reads = o.root_reads;
  a.root_order = o.root_order;
  if (o.root_split && nplans != 1) return fail(PM_ERR_INVALID, "root_split needs a single plan");
  a.root_split = o.root_split;
  a.timeout_ns = (unsigned long long)(o.timeout_ms > 0 ? o.timeout_ms : 600000) * 1000000ull;
  if (o.prefetch_off || o.prefetch_pages || o.prefetch_chunks) {
    if (!L->paged) return fail(PM_ERR_INVALID, "prefetch lists need a paged graph");
    if (nplans != 1 || !o.prefetch_off || !o.prefetch_pages || o.prefetch_chunks < 0)
      return fail(PM_ERR_INVALID, "prefetch lists need one plan, both arrays and a chunk count");
    a.pf_off = o.prefetch_off;
    a.pf_pages = o.prefetch_pages;
    a.pf_chunks = o.prefetch_chunks;
    a.pf_ahead = o.prefetch_ahead > 0 ? o.prefetch_ahead : 2;
  }
  for (int i = 0; i < nplans; i++) a.plans[i] = L->dp[i];
  L->active0 = (unsigned int)L->warps;
  if (L->paged) {
    st = paged_prepare(c, const_cast<pm_graph*>(g), L->cold, &a.pg);
    if (st != PM_OK) return st;
    a.pg.dev_copy = L->host_copy ? 0 : 1;
  }
  return PM_OK;
}

// Enqueues one launch on the context stream: control reset, the persistent
// kernel (its plans travel in its parameter block) between events eb/ee, and
// the read-back of counts, stats and status into host_ctl.  Capturable into a
// CUDA graph (host_ctl and active_src must then be pinned).
static pm_status enqueue_launch(pm_ctx* c, Launch& L, const unsigned int* active_src,
                                unsigned long long* host_ctl, cudaEvent_t eb, cudaEvent_t ee) {
  CK(cudaMemsetAsync(L.a.cursors, 0, L.ctl_words * 8, c->stream));
  if (L.n_big) CK(cudaMemsetAsync(L.a.big_owner, 0, 4 * (size_t)L.n_big, c->stream));
  CK(cudaMemcpyAsync(L.a.active, active_src, sizeof(unsigned int), cudaMemcpyHostToDevice, c->stream));
  if (eb) CK(cudaEventRecord(eb, c->stream));
  PM_CK_PENDING("pm_match");
  L.kfn<<<L.blocks, L.threads, L.smem, c->stream>>>(L.a);
  CK(cudaGetLastError());
  if (ee) CK(cudaEventRecord(ee, c->stream));
  CK(cudaMemcpyAsync(host_ctl, L.a.cursors, sizeof(unsigned long long) * kCtlRead, cudaMemcpyDeviceToHost,
                     c->stream));
  return PM_OK;
}

// Turns the read-back control words into counts, stats and a status.
static pm_status finish_launch(const Launch& L, const unsigned long long* host_ctl, float kernel_ms, float roots_ms,
                               const pm_stats& pst, uint64_t* counts_out, pm_stats* stats_out) {
  const unsigned int status = (unsigned int)(host_ctl[64 + kStatWords] & 0xffffffffu);
  for (int i = 0; i < L.nplans; i++) {
    const Plan& p = *L.plans[i];
    counts_out[i] = host_ctl[32 + i] * (p.labeled ? 1ull : (uint64_t)p.multiplicity);
  }
  if (stats_out) {
    pm_stats& so = *stats_out;
    so = pst;
    const unsigned long long* stt = host_ctl + 64;
    so.set_ops = stt[ST_SETOPS];
    so.alg_bytes = stt[ST_BYTES];
    so.n_roots = stt[ST_ROOTS];
    so.splits = stt[ST_SPLITS];
    so.page_hits = stt[ST_HITS];
    so.page_misses = stt[ST_MISSES];
    so.zero_copy_bytes = stt[ST_ZC_BYTES];
    so.evictions = stt[ST_EVICTIONS];
    so.warp_ns = stt[ST_WARP_NS];
    so.idle_ns = stt[ST_IDLE_NS];
    so.kernel_ms = kernel_ms;
    so.roots_ms = roots_ms;
    so.grid_blocks = L.blocks;
    so.block_threads = L.threads;
    so.arena_bytes = (uint64_t)(L.own_bytes + L.big_bytes);
    so.borrowed_arenas = stt[ST_BORROWS];
    so.leaf_cycles = stt[ST_LEAF_CYC];
    so.level_cycles = stt[ST_LEVEL_CYC];
    so.prefix_cycles = stt[ST_PREFIX_CYC];
    so.prefetch_requests = stt[ST_PREFETCH];
    so.page_requests = stt[ST_REQUESTS];
    so.page_dropped = stt[ST_DROPPED];
    so.device_page_loads = stt[ST_DEV_LOADS];
    so.pages_loaded += stt[ST_DEV_LOADS];  // the service thread's count plus the warps'
    so.h2d_page_bytes += stt[ST_DEV_BYTES];
    so.arena_pool = (uint64_t)L.n_big;
    so.device_status = status;
  }
  if (status & DEV_ARENA_OVERFLOW) return fail(PM_ERR_INTERNAL, "device: candidate set exceeded the warp arena");
  if (status & DEV_TIMEOUT) return fail(PM_ERR_TIMEOUT, "device: the launch hit its time limit or a bounded wait gave up");
  if (status) return fail(PM_ERR_INTERNAL, "device status 0x%x", status);
  return PM_OK;
}

// Runs an enqueued launch to completion, with the page service around it.
template <class Enqueue>
static pm_status run_launch(pm_ctx* c, const pm_graph* g, Launch& L, Enqueue enqueue, pm_stats* pst) {
  memset(pst, 0, sizeof(*pst));
  if (L.paged) {
    pm_status st = paged_service_start(c, const_cast<pm_graph*>(g));
    if (st != PM_OK) return st;
  }
  pm_status est = enqueue();
  cudaError_t sync_err = cudaStreamSynchronize(c->stream);
  if (L.paged) {
    pm_status sst = paged_service_stop(c, const_cast<pm_graph*>(g), pst);
    if (sst != PM_OK && est == PM_OK && sync_err == cudaSuccess) return sst;
  }
  if (est != PM_OK) return est;
  CK(sync_err);
  return PM_OK;
}

extern "C" pm_status pm_match(pm_ctx* c, const pm_graph* g, const pm_plan* const* plans, int nplans,
                              const pm_run_opts* opts, uint64_t* counts_out, pm_stats* stats_out) {
  if (!c || !g || !plans || nplans < 1 || !counts_out) return fail(PM_ERR_INVALID, "pm_match: bad arguments");
  pm_run_opts o;
  pm_run_opts_default(&o);
  if (opts) o = *opts;
  CK(cudaSetDevice(c->device));
  cudaEvent_t e0 = c->ev[0], e1 = c->ev[1], e2 = c->ev[2];
  CK(cudaEventRecord(e0, c->stream));
  std::unique_ptr<Launch> L(new Launch);
  pm_status st = setup_launch(c, g, plans, nplans, o, &c->d_roots, &c->roots_bytes, &c->d_arena, &c->arena_bytes,
                              &c->d_ctl, &c->ctl_bytes, L.get());
  if (st != PM_OK) return st;
  c->h_active = L->active0;
  unsigned long long host_ctl[kCtlRead];
  pm_stats pst;
  st = run_launch(c, g, *L, [&]() { return enqueue_launch(c, *L, &c->h_active, host_ctl, e1, e2); }, &pst);
  if (st != PM_OK) return st;
  float kms = 0, rms = 0;
  CK(cudaEventElapsedTime(&kms, e1, e2));
  CK(cudaEventElapsedTime(&rms, e0, e1));
  return finish_launch(*L, host_ctl, kms, rms, pst, counts_out, stats_out);
}

// ---------------------------------------------------------------------
// Prepared queries: the root lists, arenas and launch sequence are built
// once; each run replays the launch captured in a CUDA graph.
// ---------------------------------------------------------------------
struct pm_query {
  pm_ctx* c = nullptr;
  const pm_graph* g = nullptr;
  Launch L;
  int2* d_roots = nullptr;
  size_t roots_bytes = 0;
  int32_t* d_arena = nullptr;
  size_t arena_bytes = 0;
  unsigned long long* d_ctl = nullptr;
  size_t ctl_bytes = 0;
  unsigned int* h_active = nullptr;   // pinned
  unsigned long long* h_ctl = nullptr;  // pinned
  cudaEvent_t eb = nullptr, ee = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  float roots_ms = 0;
};

extern "C" void pm_query_free(pm_query* q) {
  if (!q) return;
  cudaSetDevice(q->c->device);
  if (q->exec) cudaGraphExecDestroy(q->exec);
  if (q->graph) cudaGraphDestroy(q->graph);
  if (q->eb) cudaEventDestroy(q->eb);
  if (q->ee) cudaEventDestroy(q->ee);
  free_dev(q->d_roots);
  free_dev(q->d_arena);
  free_dev(q->d_ctl);
  if (q->h_active) cudaFreeHost(q->h_active);
  if (q->h_ctl) cudaFreeHost(q->h_ctl);
  delete q;
}

extern "C" pm_status pm_query_prepare(pm_ctx* c, const pm_graph* g, const pm_plan* const* plans, int nplans,
                                      const pm_run_opts* opts, pm_query** out) {
  if (!c || !g || !plans || !out) return fail(PM_ERR_INVALID, "pm_query_prepare: bad arguments");
  pm_run_opts o;
  pm_run_opts_default(&o);
  if (opts) o = *opts;
  CK(cudaSetDevice(c->device));
  std::unique_ptr<pm_query, void (*)(pm_query*)> q(new pm_query, pm_query_free);
  q->c = c;
  q->g = g;
  CK(cudaEventRecord(c->ev[0], c->stream));
  pm_status st = setup_launch(c, g, plans, nplans, o, &q->d_roots, &q->roots_bytes, &q->d_arena, &q->arena_bytes,
                              &q->d_ctl, &q->ctl_bytes, &q->L);
  if (st != PM_OK) return st;
  CK(cudaEventRecord(c->ev[1], c->stream));
  CK(cudaEventSynchronize(c->ev[1]));
  CK(cudaEventElapsedTime(&q->roots_ms, c->ev[0], c->ev[1]));
  CK(cudaMallocHost(&q->h_active, sizeof(unsigned int)));
  CK(cudaMallocHost(&q->h_ctl, sizeof(unsigned long long) * kCtlRead));
  *q->h_active = q->L.active0;
  CK(cudaEventCreate(&q->eb));
  CK(cudaEventCreate(&q->ee));
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  // timing events stay outside the graph (recorded around each replay)
  pm_status est = enqueue_launch(c, q->L, q->h_active, q->h_ctl, nullptr, nullptr);
  cudaError_t cerr = cudaStreamEndCapture(c->stream, &q->graph);
  if (est != PM_OK) return est;
  CK(cerr);
  CK(cudaGraphInstantiate(&q->exec, q->graph, 0));
  *out = q.release();
  return PM_OK;
}

extern "C" pm_status pm_query_run(pm_query* q, uint64_t* counts_out, pm_stats* stats_out) {
  if (!q || !counts_out) return fail(PM_ERR_INVALID, "pm_query_run: bad arguments");
  pm_ctx* c = q->c;
  CK(cudaSetDevice(c->device));
  if (q->L.paged) {
    DPaging pg;
    pm_status st = paged_prepare(c, const_cast<pm_graph*>(q->g), q->L.cold, &pg);  // reset the page table
    if (st != PM_OK) return st;
  }
  pm_stats pst;
  pm_status st = run_launch(c, q->g, q->L, [&]() -> pm_status {
    CK(cudaEventRecord(q->eb, c->stream));
    CK(cudaGraphLaunch(q->exec, c->stream));
    CK(cudaEventRecord(q->ee, c->stream));
    return PM_OK;
  }, &pst);
  if (st != PM_OK) return st;
  float kms = 0;
  CK(cudaEventElapsedTime(&kms, q->eb, q->ee));
  return finish_launch(q->L, q->h_ctl, kms, q->roots_ms, pst, counts_out, stats_out);
}

// ---------------------------------------------------------------------
// Allocation-free entry point: pm_match_static.
//
// For callers that must not allocate device memory -- code running while
// another library holds the device allocator lock, in a process whose
// allocator is owned by a framework with a fixed pool, or in a service that
// has budgeted every byte up front.  The caller provides the graph arrays
// and receives the count; everything the launch needs besides them (control
// block, donation ring, root list, per-warp arenas) lives in one file-scope
// device array of PM_STATIC_SCRATCH_BYTES that each GPU keeps from module
// load until the process exits.  The plan travels in the kernel's parameter
// block like every launch's, so the scratch is the only state it shares.
// ---------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_static_scratch[PM_STATIC_SCRATCH_BYTES];

namespace {
constexpr unsigned kStaticRing = 4096;  // donation slots inside the static scratch
constexpr size_t kStaticCtlWords = 32 + 32 + kStatWords + 8 + kStaticRing + 6 * kStaticRing;

struct StaticScratch {
  bool ready = false;
  unsigned char* base = nullptr;  // device address of g_static_scratch on this device
};
StaticScratch g_static[64];
std::mutex g_static_mu;

// Root filter with unordered, bounded compaction (no scan, no temporary
// buffer): each warp reserves slots with one atomic per 32 edges; writes past
// `cap` are skipped and the host sees the true total afterwards.  The 2-hop
// test scans the neighbour's list for a vertex of sufficient degree.
__global__ void roots_static_kernel(const uint64_t* rowptr, const int32_t* colidx, const uint8_t* labels, int64_t n,
                                    RootFilter f, int2* out, unsigned long long cap, unsigned long long* counter) {
  const int lane = lane_id();
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += warps) {
    const uint64_t b = rowptr[r], e = rowptr[r + 1];
    if ((long long)(e - b) < f.d0 || (f.labeled && labels[r] != f.lab0)) continue;
    for (uint64_t i0 = b; i0 < e; i0 += 32) {
      const uint64_t i = i0 + lane;
      bool keep = false;
      int c = 0;
      if (i < e) {
        c = colidx[i];
        keep = (!f.need_gt || r > c) && (!f.labeled || labels[c] == f.lab1) &&
               (int)(rowptr[c + 1] - rowptr[c]) >= f.d1;
        if (keep) {
          bool two_hop = false;
          for (uint64_t d = rowptr[c]; d < rowptr[c + 1] && !two_hop; d++) {
            const int u = colidx[d];
            two_hop = (int)(rowptr[u + 1] - rowptr[u]) >= f.d2;
          }
          keep = two_hop;
        }
      }
      const unsigned bal = __ballot_sync(FULL, keep);
      unsigned long long base = 0;
      if (lane == 0 && bal) base = atomicAdd(counter, (unsigned long long)__popc(bal));
      base = __shfl_sync(FULL, base, 0);
      if (keep) {
        const unsigned long long pos = base + __popc(bal & lanemask_lt());
        if (pos < cap) out[pos] = make_int2((int)r, c);
      }
    }
  }
}
}  // namespace

extern "C" pm_status pm_match_static(const uint64_t* d_rowptr, const int32_t* d_colidx, const uint8_t* d_labels,
                                     int64_t n, int64_t nadj, int32_t max_degree, const pm_plan* plan,
                                     const pm_run_opts* opts, void* stream, uint64_t* count_out,
                                     pm_stats* stats_out) {
  if (!d_rowptr || (nadj > 0 && !d_colidx) || !plan || !count_out || n < 0 || max_degree < 0)
    return fail(PM_ERR_INVALID, "pm_match_static: bad arguments");
  if (n > INT32_MAX - 1) return fail(PM_ERR_INVALID, "pm_match_static: %lld vertices exceed int32 ids", (long long)n);
  const Plan& p = *plan_of(plan);
  if (p.labeled && !d_labels) return fail(PM_ERR_INVALID, "pm_match_static: labeled plan without labels");
  pm_run_opts o;
  pm_run_opts_default(&o);
  if (opts) o = *opts;
  if (o.root_counts || o.root_cost || o.root_reads || o.root_order || o.root_split || o.shard_count > 1 ||
      o.root_begin >= 0 || o.root_end >= 0 || o.prefetch_off || o.prefetch_pages || o.prefetch_chunks)
    return fail(PM_ERR_INVALID,
                "pm_match_static: per-root inputs and outputs, root orders, ranges, shards and prefetch lists are not "
                "supported");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(PM_ERR_INVALID, "pm_match_static: device %d out of range", dev);
  cudaStream_t st = (cudaStream_t)stream;
  // set-up, once per device, with that device current
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static[dev].ready) {
      unsigned char* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_static_scratch);
      if (e != cudaSuccess)
        return fail(PM_ERR_CUDA, "pm_match_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      g_static[dev].base = ptr;
      g_static[dev].ready = true;
    }
    base = g_static[dev].base;
  }
  int nsm = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int T = std::max(0, o.truncate);
  const int wpb = o.warps_per_block > 0 ? o.warps_per_block : 8;
  if (wpb > 16 || (wpb & (wpb - 1)))
    return fail(PM_ERR_INVALID, "pm_match_static: warps_per_block must be 1,2,4,8 or 16");
  const int64_t slot_words = arena_words_for(p, max_degree, T);
  const size_t warp_bytes = (size_t)slot_words * 4;
  const size_t ctl_bytes = kStaticCtlWords * 8;
  const size_t min_arena = (size_t)wpb * warp_bytes;  // one block
  if (ctl_bytes + 64 + min_arena + 256 > PM_STATIC_SCRATCH_BYTES)
    return fail(PM_ERR_INVALID,
                "pm_match_static: one block of warp arenas needs %zu bytes, beyond the %llu-byte static scratch "
                "(max degree %d is too large for this entry point)",
                min_arena, (unsigned long long)PM_STATIC_SCRATCH_BYTES, max_degree);
  // layout: control block | root counter | roots | arenas
  unsigned long long* ctl = (unsigned long long*)base;
  unsigned long long* rcount = (unsigned long long*)(base + ctl_bytes);
  int2* roots = (int2*)(base + ctl_bytes + 64);
  const size_t after_ctl = PM_STATIC_SCRATCH_BYTES - ctl_bytes - 64;
  const unsigned long long root_cap = (after_ctl - min_arena - 256) / sizeof(int2);

  CK(cudaMemsetAsync(base, 0, ctl_bytes + 64, st));  // previous calls leave their contents behind
  const RootFilter f = to_filter(p);
  PM_CK_PENDING("pm_match_static");
  roots_static_kernel<<<4 * nsm, 256, 0, st>>>(d_rowptr, d_colidx, d_labels, n, f, roots, root_cap, rcount);
  CK(cudaGetLastError());
  unsigned long long nroots = 0;
  CK(cudaMemcpyAsync(&nroots, rcount, sizeof(nroots), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (nroots > root_cap)
    return fail(PM_ERR_INVALID, "pm_match_static: %llu root edges exceed the %llu the static scratch holds",
                nroots, root_cap);
  const size_t roots_bytes = ((size_t)nroots * sizeof(int2) + 255) & ~(size_t)255;
  int32_t* arena = (int32_t*)((unsigned char*)roots + roots_bytes);
  // 256 bytes of slack after the last arena: bulk copies of a slot round its
  // end up to 16 bytes
  const size_t arena_bytes = after_ctl - roots_bytes - 256;
  // kernel variant by register cap, as pm_match chooses it
  int variant = o.high_occupancy;
  if (variant == 0) variant = (wpb <= 8) ? 2 : 3;
  if (variant < 0 || variant > 3) return fail(PM_ERR_INVALID, "pm_match_static: high_occupancy must be 0..3");
  if ((variant == 1 || variant == 2) && wpb > 8)
    return fail(PM_ERR_INVALID, "pm_match_static: warps_per_block 16 needs the uncapped kernel variant");
  void (*kfn)(const MatchArgs) =
      variant == 1 ? (p.labeled ? match_kernel<true, false, 4> : match_kernel<false, false, 4>)
      : variant == 2 ? (p.labeled ? match_kernel<true, false, 3> : match_kernel<false, false, 3>)
                     : (p.labeled ? match_kernel<true, false, 1> : match_kernel<false, false, 1>);
  int per_sm = 0;
  CK(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(WarpState) * wpb)));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, wpb * 32, sizeof(WarpState) * wpb));
  if (o.blocks_per_sm > 0) per_sm = std::min(per_sm, o.blocks_per_sm);
  int64_t blocks = std::max(1, per_sm) * (int64_t)nsm;
  blocks = std::min<int64_t>(blocks, (int64_t)(arena_bytes / ((size_t)wpb * warp_bytes)));
  if (blocks < 1) return fail(PM_ERR_INTERNAL, "pm_match_static: no room for a block of arenas");

  DPlan dp = to_dplan(p);
  dp.roots = roots;
  dp.nroots = (int64_t)nroots;
  MatchArgs a;
  memset(&a, 0, sizeof(a));
  a.plans[0] = dp;
  a.rowptr = d_rowptr;
  a.colidx = d_colidx;
  a.labels = d_labels;
  a.leaf_flat = o.leaf_per_lane == 1 ? 0 : (o.leaf_per_lane == 2 ? 2 : 1);
  a.lane_subtree_max = lane_subtree_limit(o);
  a.n = (int32_t)n;
  a.nplans = 1;
  a.T = T;
  a.chunk = o.chunk > 0 ? o.chunk : 16;
  a.shard_rank = 0;
  a.shard_count = 1;
  a.split_min = o.split_level1 == 0 ? 64 : (o.split_level1 < 0 ? 0 : o.split_level1);
  a.maxdeg = max_degree;
  unsigned long long* w = ctl;
  a.cursors = w; w += 32;
  a.counts = w; w += 32;
  a.stats = w; w += kStatWords;
  a.status = (unsigned int*)w;
  a.active = (unsigned int*)w + 1; w += 1;
  a.don_head = w; w += 1;
  a.don_tail = w; w += 1;
  a.heartbeat = w; w += 5;
  a.don_ready = w; w += kStaticRing;
  a.don_items = (int4*)w; w += 6 * kStaticRing;
  a.don_mask = kStaticRing - 1;
  const int64_t warps = blocks * wpb;
  a.total_warps = (unsigned int)warps;
  a.arena = arena;
  a.arena_words = slot_words;
  a.slot_words = slot_words;
  a.gather_words = 0;
  a.n_big = 0;
  a.timeout_ns = (unsigned long long)(o.timeout_ms > 0 ? o.timeout_ms : 600000) * 1000000ull;
  const unsigned int active0 = (unsigned int)warps;
  CK(cudaMemcpyAsync(a.active, &active0, sizeof(active0), cudaMemcpyHostToDevice, st));
  PM_CK_PENDING("pm_match_static");
  kfn<<<(int)blocks, wpb * 32, sizeof(WarpState) * wpb, st>>>(a);
  CK(cudaGetLastError());
  unsigned long long host_ctl[kCtlRead];
  CK(cudaMemcpyAsync(host_ctl, ctl, sizeof(host_ctl), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  Launch L;
  L.nplans = 1;
  L.plans[0] = &p;
  L.own_bytes = (size_t)warps * (size_t)slot_words * 4;
  L.blocks = (int)blocks;
  L.threads = wpb * 32;
  L.warps = warps;
  L.a = a;
  pm_stats pst;
  memset(&pst, 0, sizeof(pst));
  return finish_launch(L, host_ctl, 0.f, 0.f, pst, count_out, stats_out);
}
