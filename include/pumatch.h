/*
 * pumatch.h -- C-ABI of libpumatch_b200.so, a B200-native subgraph matcher.
 *
 * The reference (PUMatch) has no library API: its boundary is the CLI
 * `test <graph-prefix> <pattern.g>` (test.cu:15-21) plus three header-only
 * host classes (GraphPreprocessor, PatternPreprocessor, JobQueuePreprocessor)
 * and one kernel `_parallel_match` (src/gpu_match.cuh:10-13).  Each entry point
 * below names the reference piece it replaces.  All signatures use plain
 * pointers and sizes; no C++ or torch types cross this boundary.
 *
 * Ownership: every handle is owned by the caller and freed by the matching
 * *_close / *_free / *_destroy call.  Output buffers are caller-owned.
 * Errors: every call returns a pm_status; pm_last_error() gives a message for
 * the calling thread.  No call exits the process (the reference calls exit(1)
 * on a missing file, src/graph.h:216-226).
 */
#ifndef PUMATCH_H
#define PUMATCH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  PM_OK = 0,
  PM_ERR_IO = 1,        /* file missing or unreadable                          */
  PM_ERR_FORMAT = 2,    /* malformed .meta/.bin/.g content                     */
  PM_ERR_OOM = 3,       /* host or device allocation failed                    */
  PM_ERR_CUDA = 4,      /* a CUDA runtime call failed                          */
  PM_ERR_TIMEOUT = 5,   /* a bounded device wait gave up (status word)         */
  PM_ERR_INVALID = 6,   /* bad argument                                        */
  PM_ERR_INTERNAL = 7,  /* device-side check failed (arena/overflow/etc.)      */
  PM_ERR_NO_DEVICE = 8  /* no CUDA device; the product has no CPU fallback     */
} pm_status;

typedef struct pm_graph pm_graph; /* CSR graph placed for matching          */
typedef struct pm_plan pm_plan;   /* compiled pattern                        */
typedef struct pm_ctx pm_ctx;     /* device, streams, scratch arenas         */

/* ------------------------------------------------------------------ */
/* Graph                                                                */
/* ------------------------------------------------------------------ */

enum {
  PM_RESIDENT_HBM = 0,   /* whole CSR copied to device memory                  */
  PM_RESIDENT_PAGED = 1  /* adjacency stays in pinned host memory; a device
                            frame pool caches fixed-size pages of it           */
};

typedef struct {
  int labeled;              /* 1: read .label.bin (reference LABELED=true)     */
  int device;               /* CUDA ordinal                                    */
  int residency;            /* PM_RESIDENT_*                                   */
  uint32_t page_bytes;      /* paged mode: page size (multiple of 4 KiB)       */
  uint64_t frame_pool_bytes;/* paged mode: device frame-pool cap               */
  uint64_t static_pool_bytes;/* paged mode: the part of the pool whose pages are
                               placed once and never evicted (the reference's
                               device partition, test.cu:22-43); 0 = none     */
} pm_graph_opts;

typedef struct {
  int64_t n_vertices;
  int64_t n_adj;            /* adjacency entries = 2 x undirected edges        */
  int32_t max_degree;
  int32_t labeled;
  int32_t n_labels;         /* 1 + max label value (labeled graphs)            */
  int32_t residency;
  uint64_t device_bytes;    /* device memory held by the graph                 */
  uint64_t n_pages;         /* paged mode: pages of the adjacency array        */
  uint64_t n_frames;        /* paged mode: frames in the device pool           */
  uint64_t n_static_frames; /* paged mode: frames never evicted               */
} pm_graph_info;

void pm_graph_opts_default(pm_graph_opts* o);

/* Replaces GraphPreprocessor(prefix) + to_gpu()/to_gpu_managed()
 * (src/graph.h:34-41, 169-208, 228-254): reads <prefix>.meta.txt, .vertex.bin,
 * .edge.bin and, when labeled, .label.bin, and places the graph on the device. */
pm_status pm_graph_open(const char* prefix, const pm_graph_opts* opts, pm_graph** out);

/* Same placement from caller-owned HOST arrays (rowptr: n+1 uint64, colidx:
 * n_adj int32 sorted per list, labels: n uint32 or NULL).  The arrays are
 * copied; the caller keeps ownership. */
pm_status pm_graph_from_host(int64_t n, int64_t n_adj, const uint64_t* rowptr,
                             const int32_t* colidx, const uint32_t* labels,
                             const pm_graph_opts* opts, pm_graph** out);

/* Wrap DEVICE arrays already resident in HBM (rowptr uint64[n+1], colidx
 * int32[n_adj], labels uint8[n] or NULL).  Nothing is copied and the graph does
 * not own them; max_degree must be exact. */
pm_status pm_graph_from_device(int64_t n, int64_t n_adj, int32_t max_degree,
                               const uint64_t* d_rowptr, const int32_t* d_colidx,
                               const uint8_t* d_labels, int device, pm_graph** out);

pm_status pm_graph_get_info(const pm_graph* g, pm_graph_info* info);

/* Paged graphs: the pages (indices of page_bytes-sized ranges of the adjacency
 * array) the frame pool holds at the start of every run that is not cold --
 * by default the first n_frames pages.  The first n_static_frames of the list
 * fill the static frames (in ascending page order) and stay there in cold runs
 * too; the rest fill the evictable frames.  Replaces the reference's initial
 * package build over the vertices past the device partition
 * (src/buffer.cu:986-1060 create_buffer_from_graph). */
pm_status pm_graph_set_resident_pages(pm_graph* g, const int64_t* pages, int64_t n);
void pm_graph_close(pm_graph* g);

/* Partitioned residency across the GPUs of one node.  Replaces the
 * reference's placement of the edges beyond its device partition in host
 * memory (test.cu:22-43, src/buffer.cu:986-1060) and its multi-node mode's
 * full copy of the graph on every rank (test_mpi.cu:317-349): the adjacency
 * array is cut into slices, each held once in the HBM of one GPU, and every
 * GPU maps all slices into one device address range, which a paged graph
 * takes its pages from (pm_graph_from_paged_source) instead of pinned host
 * memory -- a miss is copied from the owner's HBM over NVLink.
 *
 * A pm_parts is such a range as one device sees it.  Slice p covers bytes
 * [part_begin[p], part_begin[p+1]) (the last up to total_bytes); every
 * boundary and total_bytes are multiples of pm_parts_granularity.  A slice is
 * backed by new memory on a device of this process (pm_parts_alloc; it can be
 * exported as a POSIX file descriptor for another process) or by memory
 * another process exported (pm_parts_import).  pm_parts_map maps them all;
 * pm_parts_ptr is then the range's device address (NULL before).  Slices
 * allocated here are filled by the caller after mapping (pm_parts_write, or
 * cudaMemcpy to pm_parts_ptr + part_begin[p]).  pm_parts_free unmaps and
 * releases; memory exported to other processes lives until they release it
 * too. */
typedef struct pm_parts pm_parts;
pm_status pm_parts_granularity(int device, uint64_t* bytes);
pm_status pm_parts_create(int device, int n_parts, const uint64_t* part_begin, uint64_t total_bytes,
                          pm_parts** out);
pm_status pm_parts_alloc(pm_parts* r, int p, int owner_device);
pm_status pm_parts_export(const pm_parts* r, int p, int* fd);
pm_status pm_parts_import(pm_parts* r, int p, int fd);
pm_status pm_parts_map(pm_parts* r);
void* pm_parts_ptr(const pm_parts* r);
/* Copies host bytes to [offset, offset + bytes) of a mapped range (a slice of
 * this process, usually). */
pm_status pm_parts_write(pm_parts* r, uint64_t offset, const void* host, uint64_t bytes);
void pm_parts_free(pm_parts* r);

/* A paged graph whose pages are cut from a device-visible array instead of
 * pinned host memory (a pm_parts range; any device address this device can
 * read).  src holds the paged layout: the adjacency array itself when
 * unlabeled, its label-grouped copy when labeled (pm_label_group_host).
 * sorted is the id-sorted array (labeled graphs read whole sorted lists from
 * it in place; NULL for unlabeled graphs, where it is src).  Both must stay
 * mapped until pm_graph_close; the graph does not own them.  opts as for
 * pm_graph_from_host (residency is paged whatever opts says). */
pm_status pm_graph_from_paged_source(int64_t n, int64_t n_adj, const uint64_t* rowptr,
                                     const uint32_t* labels, const int32_t* src,
                                     const int32_t* sorted, const pm_graph_opts* opts,
                                     pm_graph** out);

/* Host copy of the label-grouped layout a labeled paged graph caches: every
 * list stably sorted by label (ids ascending within a label); out: n_adj
 * int32.  labels are < 32.  No counterpart in the reference, which tests
 * each element's label inside its set operation (src/gpu_match.cu:238-319);
 * the grouping changes which elements are read, not the counts. */
pm_status pm_label_group_host(int64_t n, int64_t n_adj, const uint64_t* rowptr, const int32_t* colidx,
                              const uint32_t* labels, int32_t* out);

/* Reader/writer of the reference's on-disk layout (src/graph.h:228-254,
 * graph_converter/compactify.cpp:40-48, labelize.cpp:41-50) for host arrays.
 * pm_graph_read allocates *rowptr/*colidx/*labels with malloc; free with
 * pm_host_free. */
pm_status pm_graph_read(const char* prefix, int labeled, int64_t* n, int64_t* n_adj,
                        int32_t* max_degree, uint64_t** rowptr, int32_t** colidx,
                        uint32_t** labels);
pm_status pm_graph_write(const char* prefix, int64_t n, int64_t n_adj,
                         const uint64_t* rowptr, const int32_t* colidx,
                         const uint32_t* labels);
void pm_host_free(void* p);

/* SNAP edge list (text) -> <out_prefix>.meta.txt/.vertex.bin/.edge.bin and,
 * when n_labels > 0, .label.bin: the reference's converter pipeline
 * (graph_converter/convert.sh:32-65: snapToBin, makeLists, compactify,
 * labelize) in one pass.  Ids are compacted in first-seen order; lists are
 * symmetrised, sorted and deduplicated; self-loops are dropped unless
 * keep_self_loops; labels are std::rand() % n_labels after std::srand(0)
 * (labelize.cpp uses 10). */
pm_status pm_convert_snap(const char* snap_path, const char* out_prefix, int n_labels,
                          int keep_self_loops, int64_t* n_vertices, int64_t* n_adj);

/* Degree order (graph_converter/relabel.cpp:26-63): vertices sorted by
 * (degree, id), highest first, take new ids 0..n-1; lists are rewritten and
 * sorted.  Counts of every pattern are unchanged (the graph is relabelled,
 * not changed); clique searches, whose candidates lie below earlier path
 * vertices, then scan the short lists of heavy vertices' lighter
 * neighbours.  Outputs are caller-allocated: rowptr_out[n+1],
 * colidx_out[n_adj], labels_out[n] (when labels), new_id_out[n] (optional:
 * the new id of each old vertex).  Unlike relabel.cpp, labels move with
 * their vertices. */
pm_status pm_reorder_by_degree(int64_t n, int64_t n_adj, const uint64_t* rowptr, const int32_t* colidx,
                               const uint32_t* labels, uint64_t* rowptr_out, int32_t* colidx_out,
                               uint32_t* labels_out, int32_t* new_id_out);

/* Half graph (graph_converter/halve.cpp:19-30): each undirected edge once,
 * from the endpoint of lower degree to the higher (ties: to the higher id).
 * colidx_out must hold n_adj entries; *n_adj_out receives the number used
 * and *max_degree_out the longest half list. */
pm_status pm_halve(int64_t n, int64_t n_adj, const uint64_t* rowptr, const int32_t* colidx,
                   uint64_t* rowptr_out, int32_t* colidx_out, int64_t* n_adj_out, int32_t* max_degree_out);

/* ------------------------------------------------------------------ */
/* Synthetic inputs (stand-ins for the reference's converted datasets)  */
/* ------------------------------------------------------------------ */

/* Seeded Chung-Lu graph: expected degree w_i = c*(i+i0)^(-1/(gamma-1)) scaled
 * to sum 2*n_edges and capped at max_w; endpoints sampled with probability
 * proportional to w; self-loops and duplicates dropped and topped up until
 * exactly n_edges unique undirected edges.  Output CSR is malloc'd. */
pm_status pm_gen_chung_lu(int64_t n, int64_t n_edges, double gamma, double i0,
                          double max_w, uint64_t seed, uint64_t** rowptr,
                          int32_t** colidx, int64_t* n_adj, int32_t* max_degree);

/* Seeded R-MAT graph (a,b,c,d quadrant probabilities, ids >= n rejected),
 * n_edges unique undirected non-loop edges. */
pm_status pm_gen_rmat(int64_t n, int64_t n_edges, double a, double b, double c,
                      uint64_t seed, uint64_t** rowptr, int32_t** colidx,
                      int64_t* n_adj, int32_t* max_degree);

/* pm_gen_rmat computed on a device (the same arrays: the same draw sequence
 * and the first n_edges distinct edges of it), for graphs whose host-side
 * edge sort is too slow or too large -- the configured 65M-vertex, 1.8e9-edge
 * graph.  Outputs are malloc'd host arrays (pm_host_free).  No counterpart in
 * the reference, whose graphs are converted datasets
 * (graph_converter/convert.sh). */
pm_status pm_gen_rmat_device(int64_t n, int64_t n_edges, double a, double b, double c,
                             uint64_t seed, int device, uint64_t** rowptr, int32_t** colidx,
                             int64_t* n_adj, int32_t* max_degree);

/* Uniform labels in [0, n_labels) (malloc'd uint32[n]). */
pm_status pm_gen_labels(int64_t n, int n_labels, uint64_t seed, uint32_t** labels);

/* ------------------------------------------------------------------ */
/* Pattern plans                                                        */
/* ------------------------------------------------------------------ */

#define PM_MAX_PAT 7
#define PM_MAX_SLOTS 15

/* Flattened plan, the kernel's contract (same content as the reference's
 * `Pattern` struct, src/pattern.h:17-25, plus the multiplicity). */
typedef struct {
  int32_t nnodes;
  int32_t nslots;
  int32_t multiplicity;               /* |Aut(P)| (PatternMultiplicity)     */
  int32_t labeled;
  int32_t level_begin[PM_MAX_PAT + 1];/* rowptr: slots of level L are
                                         [level_begin[L], level_begin[L+1]) */
  int32_t degree[PM_MAX_PAT];
  int32_t vertex_label[PM_MAX_PAT];   /* pattern labels (1 when unlabeled)  */
  uint32_t slot_labels[PM_MAX_SLOTS]; /* one-hot label mask per slot        */
  uint32_t partial[PM_MAX_SLOTS];     /* symmetry-breaking bits per slot    */
  uint8_t set_ops[PM_MAX_SLOTS];      /* 0x20 fresh, 0x40 intersect, else
                                         copy; low 5 bits = parent slot     */
  uint8_t pad_[1];
} pm_plan_desc;

/* Replaces PatternPreprocessor(file) (src/pattern.h:48-58). */
pm_status pm_plan_compile(const char* g_path, int labeled, pm_plan** out);
pm_status pm_plan_compile_text(const char* g_text, int labeled, pm_plan** out);
pm_status pm_plan_describe(const pm_plan* p, pm_plan_desc* out);
void pm_plan_free(pm_plan* p);

/* Replaces JobQueuePreprocessor(g, p) (src/job_queue.h:39-64): counts the
 * root edges that pass the reference's filters (computed on the GPU). */
pm_status pm_count_roots(pm_ctx* ctx, const pm_graph* g, const pm_plan* p, int64_t* n_roots);

/* Copies the root list of one plan (pairs r,c in reference order, up to cap
 * pairs) and its length: the same list JobQueuePreprocessor builds, for
 * parity checks of the GPU root filter. */
pm_status pm_debug_roots(pm_ctx* ctx, const pm_graph* g, const pm_plan* p, int32_t* out_pairs,
                         int64_t cap, int64_t* n_roots);

/* ------------------------------------------------------------------ */
/* Matching                                                             */
/* ------------------------------------------------------------------ */

pm_status pm_ctx_create(int device, pm_ctx** out);
void pm_ctx_destroy(pm_ctx* ctx);
/* The cudaStream_t (as void*) every matching launch of this context uses, so
 * callers can order their own work and time it with events on it. */
void* pm_ctx_stream(pm_ctx* ctx);

typedef struct {
  int32_t truncate;         /* 0: exact.  >0: emulate the reference's
                               GRAPH_DEGREE truncation of every set result
                               (src/gpu_match.cu:302,316); 4096 as shipped    */
  int32_t warps_per_block;  /* 0 = default                                  */
  int32_t blocks_per_sm;    /* 0 = default                                  */
  int32_t chunk;            /* root edges per queue pop; 0 = default         */
  int32_t split_level1;     /* work donation to idle warps: >0 = a range of
                               candidates that only lead to the last level
                               is donated from this length on (ranges heading
                               deeper subtrees from 2 on); 0 = default (64);
                               -1 = never donate                             */
  int32_t shard_rank;       /* multi-GPU root sharding: this shard (0-based) */
  int32_t shard_count;      /* number of shards; 0/1 = no sharding; shard k
                               takes root chunks k, k+count, ...            */
  int32_t use_graph;        /* 1: capture the launch in a CUDA graph         */
  int32_t timeout_ms;       /* bound on every device wait; 0 = default       */
  int64_t root_begin;       /* restrict to positions [root_begin, root_end)
                               of the reference-ordered root list, or of
                               root_order when one is given; -1 = all.
                               Per-root outputs and root_split are indexed
                               by root id (the position in the reference
                               order), whatever the range               */
  int64_t root_end;
  int32_t cold_cache;       /* paged mode: empty the frame pool before the run */
  int32_t high_occupancy;   /* kernel variant by register cap: 0 default (85
                               with <= 8 warps per block, else uncapped); 1
                               capped at 64 registers (four 256-thread
                               blocks per SM); 2 capped at 85 (three blocks
                               per SM); 3 uncapped (up to 128, no spills)    */
  int32_t leaf_per_lane;    /* 1: last-level intersections one candidate per
                               lane (long lists go to the warp); 0 (default):
                               work-balanced across the warp when the common
                               operand fits in shared memory, each lane
                               walking a contiguous part of the candidates'
                               lists; 2: the same, strided (lane l takes
                               every 32nd element)                           */
  int32_t lane_subtree_max; /* unlabeled plans ending in a chain of
                               intersections (cliques): the last two levels
                               run one candidate per lane when the parent set
                               is at most this long; 0 = default (64), -1 =
                               never                                          */
  uint64_t* root_counts;    /* optional device ptr: per-root counts (plan 0) */
  float* root_cost;         /* optional device ptr: per-root set-op bytes    */
  const int32_t* root_order;/* optional device ptr: process roots in this
                               order (learned binning); NULL = natural      */
  float* root_reads;        /* optional device ptr: per-root adjacency-list
                               reads (page touches when paged; plan 0)      */
  int64_t own_arena_words;  /* candidate-set words in each warp's own arena
                               (0 = the plans' worst case up to 65,536);
                               warps that outgrow it borrow a worst-case
                               arena from a pool for the rest of the root
                               (the reference truncates instead,
                               src/gpu_match.cu:302,316)                    */
  int32_t max_borrowed;     /* cap on the pool of borrowed arenas (0 = as
                               many as a quarter of free memory holds)       */
  int32_t prefetch_ahead;   /* paged, one plan: when a warp claims root chunk
                               c (chunk = `chunk` roots in processing order),
                               it posts the pages listed for chunk
                               c + prefetch_ahead (0 = 2) to the copy ring  */
  const int32_t* prefetch_off;   /* optional device ptr [prefetch_chunks+1]:
                                    CSR offsets per chunk into prefetch_pages */
  const int32_t* prefetch_pages; /* optional device ptr: page ids             */
  int64_t prefetch_chunks;  /* chunks the lists cover                         */
  const int32_t* root_split; /* optional device ptr [n_roots], one plan: per
                                root, the fewest last-but-one-level
                                candidates a warp hands to idle warps (the
                                split_level1 of that root; learned: lower
                                for roots predicted heavy)                   */
  int32_t host_page_copy;   /* paged mode: 1 = every page load goes through
                               the host service thread; 0 (default) = a
                               warp that misses on a list within one page
                               copies the page into its frame itself       */
} pm_run_opts;

void pm_run_opts_default(pm_run_opts* o);

typedef struct {
  uint64_t n_roots;         /* root edges processed (all plans)             */
  uint64_t set_ops;         /* executed set operations                      */
  uint64_t alg_bytes;       /* sum over set ops of 4(|A|+|B|+|C|) (+|A|
                               label bytes when labeled) + 8 per root       */
  uint64_t splits;          /* ranges donated between warps (any level)     */
  uint64_t page_hits;       /* paged mode: adjacency reads served from HBM  */
  uint64_t page_misses;     /* paged mode: reads served over the host link  */
  uint64_t h2d_page_bytes;  /* paged mode: bytes copied into frames         */
  uint64_t zero_copy_bytes; /* paged mode: bytes read directly from host    */
  uint64_t pages_loaded;
  uint64_t evictions;
  float kernel_ms;          /* device time of the matching launch(es)       */
  float roots_ms;           /* device time of the root filter               */
  int32_t grid_blocks;
  int32_t block_threads;
  uint64_t arena_bytes;
  uint32_t device_status;   /* 0 ok; else PM_DEV_* flags                     */
  uint32_t pad_;
  uint64_t warp_ns;         /* sum over warps of their time in the launch    */
  uint64_t idle_ns;         /* sum over warps of time spent waiting for
                               donated work once the root queue was empty   */
  uint64_t borrowed_arenas; /* times a warp borrowed a worst-case arena      */
  uint64_t arena_pool;      /* worst-case arenas in the launch's pool        */
  uint64_t leaf_cycles;     /* sum over warps of SM cycles counting the last
                               level(s)                                      */
  uint64_t level_cycles;    /* ... computing the candidate sets of the levels
                               above it                                      */
  uint64_t prefix_cycles;   /* ... recomputing the path prefix of a donated
                               range (the cost of moving work between warps) */
  uint64_t prefetch_requests; /* pages posted from the prefetch lists          */
  uint64_t page_requests;   /* paged mode: page loads posted to the host     */
  uint64_t page_dropped;    /* paged mode: loads not posted (ring full, or
                               every evictable frame pinned or referenced)  */
  uint64_t device_page_loads; /* paged mode: pages a warp copied into a frame
                               itself (included in pages_loaded)            */
} pm_stats;

/* Replaces the `_parallel_match` launch and the host reduction of per-warp
 * counts (test.cu:171-198).  Runs every plan over the graph in one persistent
 * launch and writes one exact count per plan (multiplied by the pattern's
 * automorphism count when unlabeled, as test.cu:198 does). */
pm_status pm_match(pm_ctx* ctx, const pm_graph* g, const pm_plan* const* plans, int nplans,
                   const pm_run_opts* opts, uint64_t* counts_out, pm_stats* stats_out);

/* Prepared query: the batched multi-pattern launch built once -- root lists,
 * arenas, plan upload and the persistent kernel captured in a CUDA graph --
 * and replayed by each pm_query_run.  Same results as pm_match.  The graph
 * and context must outlive the query. */
typedef struct pm_query pm_query;
pm_status pm_query_prepare(pm_ctx* ctx, const pm_graph* g, const pm_plan* const* plans, int nplans,
                           const pm_run_opts* opts, pm_query** out);
pm_status pm_query_run(pm_query* q, uint64_t* counts_out, pm_stats* stats_out);
void pm_query_free(pm_query* q);

/* ------------------------------------------------------------------ */
/* Learned scheduler (no counterpart in the reference)                   */
/* ------------------------------------------------------------------ */

#define PM_MLP_IN 16
#define PM_MLP_HIDDEN 64
#define PM_MLP_OUT 2
#define PM_MLP_PARAMS (PM_MLP_IN * PM_MLP_HIDDEN + PM_MLP_HIDDEN + PM_MLP_HIDDEN * PM_MLP_HIDDEN + \
                       PM_MLP_HIDDEN + PM_MLP_HIDDEN * PM_MLP_OUT + PM_MLP_OUT)

/* PM_MLP_IN features per root edge of plan p, in root-list order, into the
 * device buffer d_features (cap rows); *n_roots gets the root count (call
 * with d_features NULL to size the buffer). */
pm_status pm_root_features(pm_ctx* ctx, const pm_graph* g, const pm_plan* p, float* d_features,
                           int64_t cap, int64_t* n_roots);

/* 16 -> 64 -> 64 -> 2 MLP, ReLU, BF16 weights with FP32 accumulation and FP32
 * master weights (Adam).  Parameters are laid out W1[16][64] b1 W2[64][64] b2
 * W3[64][2] b3 (input-major).  All data pointers are device pointers except
 * the host weight/gradient buffers. */
typedef struct pm_mlp pm_mlp;
pm_status pm_mlp_create(int device, uint64_t seed, pm_mlp** out);
void pm_mlp_free(pm_mlp* m);
pm_status pm_mlp_forward(pm_mlp* m, const float* d_x, int64_t n, float* d_y);
/* Mean-squared-error gradient over n samples into host_grad[PM_MLP_PARAMS]. */
pm_status pm_mlp_gradient(pm_mlp* m, const float* d_x, const float* d_t, int64_t n, float* host_grad,
                          float* loss_out);
/* One Adam step on the batch (gradient, update, BF16 re-quantisation). */
pm_status pm_mlp_train_step(pm_mlp* m, const float* d_x, const float* d_t, int64_t n, float lr,
                            float* loss_out);
pm_status pm_mlp_get_weights(pm_mlp* m, float* host_out);
pm_status pm_mlp_set_weights(pm_mlp* m, const float* host_in);

/* ------------------------------------------------------------------ */
/* Allocation-free matching (no counterpart in the reference)           */
/* ------------------------------------------------------------------ */

/* Bytes of the file-scope device scratch pm_match_static works in.  Every
 * GPU that loads this library holds it from module load until exit. */
#define PM_STATIC_SCRATCH_BYTES (64ull << 20)

/* pm_match for callers that cannot allocate device memory (it has no
 * counterpart in the reference, whose driver allocates everything up front,
 * test.cu:59-154): a region that holds another library's allocator lock, a
 * service whose device memory is budgeted and pooled elsewhere, or a
 * framework that owns the allocator and forbids outside cudaMalloc calls.  It
 * calls no cudaMalloc/cudaFree and no allocating library routine: the caller
 * passes the graph as DEVICE arrays (rowptr uint64[n+1], colidx int32[n_adj],
 * labels uint8[n] or NULL) and gets the count in *count_out (host); the
 * control block, root list and per-warp arenas live in one static device
 * array of PM_STATIC_SCRATCH_BYTES.  The launch's plan travels in its kernel
 * parameters, so the scratch is all it shares with other launches.
 *  - Limits: one plan; n below 2^31; the root list plus one block of warp
 *    arenas (patterns' worst-case candidate sets, sized from max_degree)
 *    must fit the scratch, otherwise PM_ERR_INVALID says so; fewer warps run
 *    when the arenas only partly fit.  Per-root inputs and outputs, root
 *    orders, ranges, shards and prefetch lists are not supported here
 *    (PM_ERR_INVALID); every other pm_run_opts field means what it means for
 *    pm_match.
 *  - The first call on a device looks up the scratch's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture.
 *  - Every call shares the one scratch and clears what must start at zero;
 *    calls that overlap on the GPU (other threads, other streams) race on
 *    it -- serialize them.
 *  - stream: a cudaStream_t (NULL = legacy default stream).  The call
 *    synchronizes that stream: it returns after the work on it is done, so
 *    it is not for use inside a stream callback.  stats_out->kernel_ms is 0. */
pm_status pm_match_static(const uint64_t* d_rowptr, const int32_t* d_colidx, const uint8_t* d_labels,
                          int64_t n, int64_t n_adj, int32_t max_degree, const pm_plan* plan,
                          const pm_run_opts* opts, void* stream, uint64_t* count_out,
                          pm_stats* stats_out);

/* The JSON sidecar of one launch (the reference prints only "ms count";
 * its counters g_total_cpu_m / g_total_cpu_bytes, src/buffer.cu:11-19, are
 * never printed): per-pattern counts, kernel ms, matches/s, set operations,
 * algorithmic bytes and GB/s, page traffic, warp idle share.  Writes at most
 * cap bytes (NUL-terminated) into buf; *len_out (optional) receives the
 * length the whole document needs.  PM_ERR_INVALID when it does not fit. */
pm_status pm_stats_json(const pm_stats* stats, const uint64_t* counts, int n_counts, char* buf, size_t cap,
                        size_t* len_out);

const char* pm_strerror(pm_status s);
const char* pm_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* PUMATCH_H */
