// pm_paging.cu -- host side of the paged residency: placement of the
// adjacency array in pinned host memory, the device page table and frame pool,
// and the service thread that turns page requests into H2D copies.
//
// Replaces the reference's host packaging threads (src/buffer.cu:1218-1389
// cpu_process_all_vertices, :1580-1645 cpu_process_multiple_queue, :873-929
// copy_packages_to_gpu; test.cu:160-169).  Differences by design:
//   * one service thread per graph, not one per CUDA block, and it never
//     handshakes with the kernel -- the kernel keeps running on host reads
//     while a page is in flight;
//   * copies come from pinned memory (true async DMA) on a side stream, one
//     cudaMemcpyAsync per page plus one 4-byte copy that publishes the page
//     table entry after it (same stream, so it lands after the data);
//   * eviction is decided on the device (CLOCK over reference bits, skipping
//     pinned frames), so the host never overwrites a frame a warp is reading.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "pm_device.cuh"
#include "pm_paging.cuh"

#define CKP(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(PM_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

namespace pm {

pm_status compute_maxnbrdeg(pm_graph* g, const int32_t* colidx);

struct PagedState {
  int device = 0;
  int32_t* frames = nullptr;
  int32_t* page_frame = nullptr;
  unsigned long long* frame_state = nullptr;  // (page << 32) | pins per frame
  uint8_t* frame_ref = nullptr;
  unsigned long long* dctl = nullptr;  // [0] clock hand, [1] next free, [2] ring head
  // mapped pinned host memory
  int2* ring = nullptr;
  unsigned long long* ring_seq = nullptr;
  unsigned long long* host_tail = nullptr;
  int2* ring_dev = nullptr;
  unsigned long long* ring_seq_dev = nullptr;
  unsigned long long* host_tail_dev = nullptr;
  unsigned int ring_slots = 1u << 16;
  int32_t* stage = nullptr;  // pinned: stage[f] = f, source of page-table publishes
  int64_t prefilled = 0;     // frames 0..prefilled-1 hold the initial resident pages
  int64_t n_static = 0;      // frames 0..n_static-1 are never evicted (<= prefilled)
  int64_t n_static_cap = 0;  // static frames the pool was created with
  bool static_loaded = false;  // the static frames hold their pages already
  int32_t* init_pf = nullptr;  // pinned [n_pages]: page -> frame at the start of a run
  int32_t* init_fp = nullptr;  // pinned [n_frames]: frame -> page at the start of a run
  int32_t* cold_pf = nullptr;  // pinned [n_pages]: the same for a cold run (static frames only)
  int32_t* cold_fp = nullptr;  // pinned [n_frames]
  unsigned long long* fs_host = nullptr;  // pinned [n_frames]: frame states to upload
  // service thread
  std::thread th;
  std::atomic<bool> stop{false};
  cudaStream_t copy_stream = nullptr;
  unsigned long long tail = 0;
  unsigned long long loaded = 0, h2d_bytes = 0, noops = 0;
  cudaError_t err = cudaSuccess;
};

static void release_state(PagedState* s) {
  if (!s) return;
  cudaFree(s->frames);
  cudaFree(s->page_frame);
  cudaFree(s->frame_state);
  cudaFree(s->frame_ref);
  cudaFree(s->dctl);
  cudaFreeHost(s->ring);
  cudaFreeHost(s->ring_seq);
  cudaFreeHost(s->host_tail);
  cudaFreeHost(s->stage);
  cudaFreeHost(s->init_pf);
  cudaFreeHost(s->init_fp);
  cudaFreeHost(s->cold_pf);
  cudaFreeHost(s->cold_fp);
  cudaFreeHost(s->fs_host);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  delete s;
}

// Copies out of the page source: pinned host memory, or (a graph placed on
// an external source) device memory of this or another GPU.
static cudaMemcpyKind source_kind(const pm_graph* g) {
  return g->h_colidx ? cudaMemcpyHostToDevice : cudaMemcpyDefault;
}

// Resets the table to the initial residency (frames 0..prefilled-1 hold the
// pages init_fp names), or, when cold, to the static frames alone.  Evictable
// initial pages are recopied into their frames every time, since the last run
// may have evicted them; static frames are copied once.
static pm_status reset_table(pm_graph* g, cudaStream_t st, bool cold) {
  PagedState* s = g->ps;
  const int64_t pre = cold ? s->n_static : s->prefilled;
  const int32_t* pf = cold ? s->cold_pf : s->init_pf;
  const int32_t* fp = cold ? s->cold_fp : s->init_fp;
  CKP(cudaMemcpyAsync(s->page_frame, pf, sizeof(int32_t) * g->n_pages, cudaMemcpyHostToDevice, st));
  // every frame starts unpinned, tagged with the page it holds (all ones when empty)
  for (int64_t f = 0; f < g->n_frames; f++) s->fs_host[f] = (unsigned long long)(uint32_t)fp[f] << 32;
  CKP(cudaMemcpyAsync(s->frame_state, s->fs_host, sizeof(unsigned long long) * g->n_frames,
                      cudaMemcpyHostToDevice, st));
  const size_t pb = (size_t)g->page_ints * 4;
  const cudaMemcpyKind kind = source_kind(g);
  for (int64_t f = s->static_loaded ? s->n_static : 0; f < pre;) {
    // coalesce runs of consecutive pages in consecutive frames into one copy
    // (a run never crosses the static boundary)
    int64_t e = f + 1;
    while (e < pre && e != s->n_static && fp[e] == fp[e - 1] + 1) e++;
    const int64_t first = (int64_t)fp[f] * g->page_ints;
    const size_t bytes = std::min<size_t>((size_t)(e - f) * pb, sizeof(int32_t) * (size_t)(g->nadj - first));
    CKP(cudaMemcpyAsync((char*)s->frames + (size_t)f * pb, g->h_paged + first, bytes, kind, st));
    f = e;
  }
  CKP(cudaMemsetAsync(s->frame_ref, 0, g->n_frames, st));
  unsigned long long h[4] = {0, (unsigned long long)pre, 0, 0};
  CKP(cudaMemcpyAsync(s->dctl, h, sizeof(h), cudaMemcpyHostToDevice, st));
  CKP(cudaStreamSynchronize(st));
  s->static_loaded = true;
  s->tail = 0;
  *(volatile unsigned long long*)s->host_tail = 0;
  memset(s->ring_seq, 0, sizeof(unsigned long long) * s->ring_slots);
  return PM_OK;
}

// Fills init_* / cold_* from a page list: the first n_static entries, sorted,
// take the static frames; the rest, in the given order, the evictable ones.
static pm_status set_initial(pm_graph* g, std::vector<int64_t> pages) {
  PagedState* s = g->ps;
  const int64_t k = std::min<int64_t>((int64_t)pages.size(), g->n_frames);
  pages.resize((size_t)k);
  std::vector<int32_t> pf((size_t)g->n_pages, PAGE_ABSENT);
  for (int64_t f = 0; f < k; f++) {
    if (pages[f] < 0 || pages[f] >= g->n_pages) return fail(PM_ERR_INVALID, "page %lld out of range", (long long)pages[f]);
    if (pf[pages[f]] != PAGE_ABSENT) return fail(PM_ERR_INVALID, "page %lld listed twice", (long long)pages[f]);
    pf[pages[f]] = 0;
  }
  const int64_t ns = std::min<int64_t>(s->n_static, k);
  std::sort(pages.begin(), pages.begin() + ns);
  for (int64_t p = 0; p < g->n_pages; p++) s->init_pf[p] = s->cold_pf[p] = PAGE_ABSENT;
  for (int64_t f = 0; f < g->n_frames; f++) {
    s->init_fp[f] = f < k ? (int32_t)pages[f] : -1;
    s->cold_fp[f] = f < ns ? (int32_t)pages[f] : -1;
    if (f < k) s->init_pf[pages[f]] = (int32_t)f;
    if (f < ns) s->cold_pf[pages[f]] = (int32_t)f;
  }
  s->prefilled = k;
  s->n_static = ns;
  s->static_loaded = false;
  return PM_OK;
}

// Places a paged graph.  The pages are cut from src_dev when it is given (a
// device-visible array: another GPU's HBM through a pm_parts range, say),
// else from a pinned, mapped host copy of colidx.
pm_status paged_place(pm_graph* g, const int32_t* colidx, const pm_graph_opts* o, const int32_t* src_dev) {
  uint32_t pb = o->page_bytes ? o->page_bytes : (64u << 10);
  if (pb < 4096 || (pb & (pb - 1))) return fail(PM_ERR_INVALID, "page_bytes must be a power of two >= 4096");
  std::unique_ptr<PagedState> s(new PagedState);
  s->device = g->device;
  const int64_t nadj = g->nadj;
  g->page_ints = pb / 4;
  int shift = 0;
  while ((1u << shift) < g->page_ints) shift++;
  g->n_pages = (nadj + g->page_ints - 1) / g->page_ints;
  g->n_frames = std::min<int64_t>((int64_t)(o->frame_pool_bytes / pb), g->n_pages);
  if (g->n_frames < 1 && g->n_pages > 0) g->n_frames = 1;
  if (src_dev) {
    // an external source: nothing to copy; the caller keeps it mapped
    g->h_paged = g->h_paged_dev = src_dev;
  } else {
    // adjacency in pinned, mapped host memory
    CKP(cudaHostAlloc((void**)&g->h_colidx, sizeof(int32_t) * std::max<int64_t>(nadj, 1),
                      cudaHostAllocMapped | cudaHostAllocPortable));
    if (nadj) {
      const int64_t kBlock = 1 << 24;
#pragma omp parallel for schedule(static)
      for (int64_t b = 0; b < (nadj + kBlock - 1) / kBlock; b++) {
        const int64_t e = std::min(nadj, (b + 1) * kBlock);
        memcpy(g->h_colidx + b * kBlock, colidx + b * kBlock, sizeof(int32_t) * (e - b * kBlock));
      }
    }
    CKP(cudaHostGetDevicePointer((void**)&g->h_colidx_dev, g->h_colidx, 0));
    g->h_paged = g->h_colidx;  // a labeled graph switches to its label-grouped copy after placement
    g->h_paged_dev = g->h_colidx_dev;
  }
  // device page table and frame pool
  const size_t fbytes = (size_t)g->n_frames * pb;
  CKP(cudaMalloc(&s->frames, std::max<size_t>(fbytes, 4)));
  CKP(cudaMalloc(&s->page_frame, sizeof(int32_t) * std::max<int64_t>(g->n_pages, 1)));
  CKP(cudaMalloc(&s->frame_state, sizeof(unsigned long long) * std::max<int64_t>(g->n_frames, 1)));
  CKP(cudaMalloc(&s->frame_ref, std::max<int64_t>(g->n_frames, 1)));
  CKP(cudaMalloc(&s->dctl, sizeof(unsigned long long) * 4));
  g->device_bytes += fbytes + 4 * g->n_pages + 9 * g->n_frames;
  // request ring, consumer cursor and publish staging in mapped host memory
  CKP(cudaHostAlloc((void**)&s->ring, sizeof(int2) * s->ring_slots, cudaHostAllocMapped | cudaHostAllocPortable));
  CKP(cudaHostAlloc((void**)&s->ring_seq, sizeof(unsigned long long) * s->ring_slots,
                    cudaHostAllocMapped | cudaHostAllocPortable));
  CKP(cudaHostAlloc((void**)&s->host_tail, 64, cudaHostAllocMapped | cudaHostAllocPortable));
  CKP(cudaHostAlloc((void**)&s->stage, sizeof(int32_t) * std::max<int64_t>(g->n_frames, 1), cudaHostAllocPortable));
  for (int64_t f = 0; f < g->n_frames; f++) s->stage[f] = (int32_t)f;
  CKP(cudaHostGetDevicePointer((void**)&s->ring_dev, s->ring, 0));
  CKP(cudaHostGetDevicePointer((void**)&s->ring_seq_dev, s->ring_seq, 0));
  CKP(cudaHostGetDevicePointer((void**)&s->host_tail_dev, s->host_tail, 0));
  CKP(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
  // warm start: the first pages of the array, the way the reference keeps the
  // first 60% of the edges on the device (test.cu:22-43)
  const size_t pfb = sizeof(int32_t) * std::max<int64_t>(g->n_pages, 1);
  const size_t fpb = sizeof(int32_t) * std::max<int64_t>(g->n_frames, 1);
  CKP(cudaHostAlloc((void**)&s->init_pf, pfb, cudaHostAllocPortable));
  CKP(cudaHostAlloc((void**)&s->init_fp, fpb, cudaHostAllocPortable));
  CKP(cudaHostAlloc((void**)&s->cold_pf, pfb, cudaHostAllocPortable));
  CKP(cudaHostAlloc((void**)&s->cold_fp, fpb, cudaHostAllocPortable));
  CKP(cudaHostAlloc((void**)&s->fs_host, 2 * fpb, cudaHostAllocPortable));
  s->n_static = s->n_static_cap = std::min<int64_t>((int64_t)(o->static_pool_bytes / pb), g->n_frames);
  g->ps = s.release();
  std::vector<int64_t> prefix((size_t)g->n_frames);
  for (int64_t f = 0; f < g->n_frames; f++) prefix[f] = f;
  // the frames are filled by the first run (static_loaded is false), after a
  // labeled graph has switched to its grouped copy
  return set_initial(g, std::move(prefix));
}

int64_t paged_static_frames(const pm_graph* g) { return g->ps ? g->ps->n_static : 0; }

pm_status paged_maxnbrdeg(pm_graph* g) { return compute_maxnbrdeg(g, g->h_colidx_dev); }

void paged_release(pm_graph* g) {
  if (g->ps) {
    if (g->ps->th.joinable()) {
      g->ps->stop = true;
      g->ps->th.join();
    }
    release_state(g->ps);
    g->ps = nullptr;
  }
  if (g->h_colidx) cudaFreeHost(g->h_colidx);
  if (g->h_colidx_lab) cudaFreeHost(g->h_colidx_lab);
  g->h_colidx = g->h_colidx_lab = nullptr;
  g->h_paged = nullptr;
}

pm_status paged_prepare(pm_ctx* c, pm_graph* g, bool cold, DPaging* out) {
  PagedState* s = g->ps;
  if (!s) return fail(PM_ERR_INTERNAL, "paged graph without page state");
  pm_status st = reset_table(g, s->copy_stream, cold);
  if (st != PM_OK) return st;
  (void)c;
  memset(out, 0, sizeof(*out));
  int shift = 0;
  while ((1u << shift) < g->page_ints) shift++;
  out->page_shift = shift;
  out->n_static = (int32_t)s->n_static;
  out->n_pages = g->n_pages;
  out->n_frames = g->n_frames;
  out->page_frame = s->page_frame;
  out->frame_state = s->frame_state;
  out->frame_ref = s->frame_ref;
  out->frames = s->frames;
  out->host_colidx = g->h_paged_dev;
  out->clock_hand = s->dctl;
  out->next_free = s->dctl + 1;
  out->ring_head = s->dctl + 2;
  out->ring = s->ring_dev;
  out->ring_seq = s->ring_seq_dev;
  out->host_tail = s->host_tail_dev;
  out->ring_mask = s->ring_slots - 1;
  out->n_ints = g->nadj;
  out->dev_copy = 1;
  return PM_OK;
}

// Drains posted requests: copy page -> frame, then publish the entry.
static void service_loop(pm_graph* g) {
  PagedState* s = g->ps;
  cudaSetDevice(s->device);
  const size_t pb = (size_t)g->page_ints * 4;
  const int64_t nadj = g->nadj;
  const unsigned mask = s->ring_slots - 1;
  for (;;) {
    int got = 0;
    while (*(volatile unsigned long long*)&s->ring_seq[s->tail & mask] == s->tail + 1) {
      std::atomic_thread_fence(std::memory_order_acquire);
      const volatile int* slot = (const volatile int*)&s->ring[s->tail & mask];
      const int2 req = make_int2(slot[0], slot[1]);
      s->tail++;
      got++;
      if (req.x < 0) { s->noops++; continue; }
      const int64_t first = (int64_t)req.x * g->page_ints;
      const size_t bytes = std::min<size_t>(pb, sizeof(int32_t) * (size_t)(nadj - first));
      cudaError_t e = cudaMemcpyAsync((char*)s->frames + (size_t)req.y * pb, g->h_paged + first, bytes,
                                      source_kind(g), s->copy_stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->page_frame + req.x, s->stage + req.y, sizeof(int32_t), cudaMemcpyHostToDevice,
                            s->copy_stream);
      if (e != cudaSuccess) {
        // the page stays LOADING: readers keep using host reads, counts stay exact
        s->err = e;
        continue;
      }
      s->loaded++;
      s->h2d_bytes += bytes;
    }
    if (got) {
      std::atomic_thread_fence(std::memory_order_release);
      *(volatile unsigned long long*)s->host_tail = s->tail;
      continue;
    }
    if (s->stop.load(std::memory_order_acquire)) break;
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  cudaStreamSynchronize(s->copy_stream);
}

pm_status paged_service_start(pm_ctx* c, pm_graph* g) {
  (void)c;
  PagedState* s = g->ps;
  s->stop = false;
  s->loaded = s->h2d_bytes = s->noops = 0;
  s->err = cudaSuccess;
  s->th = std::thread(service_loop, g);
  return PM_OK;
}

// Called after the kernel finished: every request it posted is already in the
// ring, so draining once more and joining completes all of them.
pm_status paged_service_stop(pm_ctx* c, pm_graph* g, pm_stats* st) {
  (void)c;
  PagedState* s = g->ps;
  s->stop = true;
  if (s->th.joinable()) s->th.join();
  st->pages_loaded = s->loaded;
  st->h2d_page_bytes = s->h2d_bytes;
  if (s->err != cudaSuccess)
    return fail(PM_ERR_CUDA, "page service copy failed: %s", cudaGetErrorString(s->err));
  return PM_OK;
}

}  // namespace pm

// Chooses the pages the frame pool starts each (non-cold) run with -- e.g.
// the pages a cost model predicts the hottest.  The first n_static_frames of
// the list become the static (never evicted) pages; pages beyond the pool
// size are ignored; duplicates are an error.
extern "C" pm_status pm_graph_set_resident_pages(pm_graph* g, const int64_t* pages, int64_t n) {
  using namespace pm;
  if (!g || (n > 0 && !pages) || n < 0) return fail(PM_ERR_INVALID, "pm_graph_set_resident_pages: bad arguments");
  if (g->residency != PM_RESIDENT_PAGED || !g->ps) return fail(PM_ERR_INVALID, "graph is not paged");
  CKP(cudaSetDevice(g->device));
  // the static count is the pool's, not the list's: keep it across calls
  PagedState* s = g->ps;
  const int64_t before = s->n_static;
  s->n_static = s->n_static_cap;
  pm_status st = set_initial(g, std::vector<int64_t>(pages, pages + n));
  if (st != PM_OK) s->n_static = before;
  return st;
}
