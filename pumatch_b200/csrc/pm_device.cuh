// pm_device.cuh -- device-side structures shared by the CUDA translation units
// of libpumatch_b200.so (matching kernel, root filter, page cache).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "pm_common.h"

#define PM_MAX_BATCH 32  // plans per persistent launch

namespace pm {

// Device status flags (pm_stats.device_status).
enum : uint32_t {
  DEV_ARENA_OVERFLOW = 1u << 0,  // a slot did not fit the warp's arena
  DEV_TIMEOUT = 1u << 1,         // a bounded wait gave up
  DEV_BAD_ROOT = 1u << 2,        // root id out of range
};

// One plan as the kernel reads it (constant memory).
struct DPlan {
  int32_t nnodes;
  int32_t nslots;
  int32_t labeled;
  int32_t last_slot;              // the single slot of level nnodes-2
  int32_t level_begin[PM_MAX_PAT + 1];
  uint32_t slot_labels[16];
  uint32_t partial[16];
  uint8_t kind[16];               // SlotKind
  uint8_t parent[16];
  int8_t alias[16];               // -1, or a slot of the same level with the
                                  // same operation whose result contains this one
  uint8_t alias_prefix[16];       // 1: this slot is the alias's prefix below
                                  // this slot's own bound; 0: equal sets
  // last two levels one lane per candidate (lane_subtree): the computed
  // intersection of level nnodes-3, its alias (or -1); l2_x = -1 when the
  // plan does not have that shape
  int8_t l2_x, l2_y;
  int8_t pad_[6];
  const int2* roots;              // (v0, v1) root edges, reference order (the whole list)
  int64_t nroots;                 // positions this launch processes
  int64_t rbase;                  // first position: root_begin (0 = all)
};

// Page cache of the adjacency array (paged residency).  A page is a fixed
// power-of-two range of colidx; frames are page-sized slots of a device pool.
struct DPaging {
  int32_t page_shift;              // log2(ints per page)
  int32_t n_static;                // frames [0, n_static) are never evicted or pinned
  int64_t n_pages;
  int64_t n_frames;
  int32_t* page_frame;             // [n_pages]: frame, or PAGE_ABSENT/LOADING/EVICTING
  // [n_frames]: (page held << 32) | readers in flight; page all ones when
  // never used.  One word, so a pin and an eviction are ordered by the word
  // itself: an evictor's CAS needs zero pins, a reader's add sees the tag.
  unsigned long long* frame_state;
  uint8_t* frame_ref;              // [n_frames]: CLOCK reference bits
  int32_t* frames;                 // [n_frames << page_shift]
  const int32_t* host_colidx;      // device-visible pointer to the paged host array
  unsigned long long* clock_hand;  // device
  unsigned long long* next_free;   // device: frames handed out so far
  unsigned long long* ring_head;   // device: ring slots reserved
  int2* ring;                      // mapped host: (page, frame) requests
  unsigned long long* ring_seq;    // mapped host: slot + 1 once written
  unsigned long long* host_tail;   // mapped host: slots the host consumed
  unsigned int ring_mask;
  int32_t dev_copy;                // 1: a warp that misses on a one-page list copies the page itself
  int64_t n_ints;                  // length of the paged host array (the last page may be short)
};

enum : int32_t { PAGE_ABSENT = -1, PAGE_LOADING = -2 };

struct PagedState;  // host-side page service state (pm_paging.cu)

// Called before a launch: an error still pending from an earlier call (this
// library's or another's on the same thread) is reported, not silently
// cleared, so the launch's own check afterwards sees only its own error.
// cudaErrorNotReady is a query status, not a failure, and is just cleared.
inline pm_status pending_error(const char* where) {
  const cudaError_t e = cudaPeekAtLastError();
  if (e == cudaSuccess) return PM_OK;
  (void)cudaGetLastError();
  if (e == cudaErrorNotReady) return PM_OK;
  return fail(PM_ERR_CUDA, "%s: an earlier CUDA call left an error pending: %s", where, cudaGetErrorString(e));
}

}  // namespace pm

#define PM_CK_PENDING(where)                           \
  do {                                                 \
    const pm_status s_ = pm::pending_error(where);     \
    if (s_ != PM_OK) return s_;                        \
  } while (0)

// Opaque handles of the C-ABI (pumatch.h), shared by the device TUs.
struct pm_graph {
  int device = 0;
  int64_t n = 0, nadj = 0;
  int32_t maxdeg = 0;
  int labeled = 0;
  int nlabels = 0;
  int residency = PM_RESIDENT_HBM;
  bool owns = true;
  uint64_t* d_rowptr = nullptr;
  int32_t* d_colidx = nullptr;   // HBM residency only
  uint8_t* d_labels = nullptr;
  int32_t* d_maxnbrdeg = nullptr;
  // labeled graphs in HBM: each list regrouped by label (id order kept within
  // a label) and per-vertex label offsets, so a one-label candidate set is a
  // contiguous sub-range
  int32_t* d_colidx_lab = nullptr;
  int32_t* d_lab_off = nullptr;    // [n][nl1]: start of label l within v's list; [n][nl1-1] = deg
  int32_t nl1 = 0;
  uint64_t device_bytes = 0;
  // paged residency (pm_paging.cu)
  int32_t* h_colidx = nullptr;     // pinned, mapped copy of the adjacency array
  int32_t* h_colidx_dev = nullptr; // its device-visible address
  // labeled paged graphs page the label-grouped copy (d_lab_off on the
  // device gives the groups); unlabeled ones page colidx itself
  int32_t* h_colidx_lab = nullptr;     // pinned, mapped
  int32_t* h_colidx_lab_dev = nullptr;
  const int32_t* h_paged = nullptr;    // host array the pages are cut from
  const int32_t* h_paged_dev = nullptr;
  uint32_t page_ints = 0;
  int64_t n_pages = 0, n_frames = 0;
  pm::PagedState* ps = nullptr;
};

struct pm_ctx {
  int device = 0;
  int nsm = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // reusable device scratch
  int32_t* d_arena = nullptr;
  size_t arena_bytes = 0;
  unsigned long long* d_ctl = nullptr;  // cursors, counts, stats, status, donation ring
  size_t ctl_bytes = 0;
  int2* d_roots = nullptr;
  size_t roots_bytes = 0;
  void* d_tmp = nullptr;
  size_t tmp_bytes = 0;
  int32_t* d_vcount = nullptr;
  int64_t* d_voff = nullptr;
  size_t vbuf_n = 0;
  unsigned int h_active = 0;  // staging for the initial active-warp count
};

