/*
 * pm_oracle.h -- CPU oracle for the subgraph-matching hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is loaded by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and
 * never by the product library (pumatch_b200/), which has no CPU fallback.
 *
 * It restates, in plain single-threaded C, the reference's semantics:
 *   - pattern plan compiler      src/pattern.h:67-355
 *   - root-edge filter           src/job_queue.h:39-64
 *   - DFS + candidate sets       src/gpu_match.cu:386-816 (extend),
 *                                 855-1047 (match), 238-319 (compute_set)
 *   - final count x |Aut|        test.cu:195-198
 * Pinning: tests/golden/ holds plan fixtures produced by the reference's own
 * PatternPreprocessor and JobQueuePreprocessor (compiled untouched from the
 * reference headers by oracle/Makefile into oracle/_ref/), which the oracle is
 * checked against; counts are checked against brute-force enumeration and
 * closed forms on small graphs.
 */
#ifndef PM_ORACLE_H
#define PM_ORACLE_H
#include <stdint.h>

#define ORC_MAX_PAT 7
#define ORC_MAX_SLOTS 15

typedef struct {
  int nnodes, nslots, multiplicity, labeled;
  int level_begin[ORC_MAX_PAT + 1];
  int degree[ORC_MAX_PAT];
  int vertex_label[ORC_MAX_PAT];
  uint32_t slot_labels[ORC_MAX_SLOTS];
  uint32_t partial[ORC_MAX_SLOTS];
  uint8_t set_ops[ORC_MAX_SLOTS];
} orc_plan;

typedef struct {
  int64_t n;
  int64_t n_adj;
  const uint64_t* rowptr;
  const int32_t* colidx;
  const uint32_t* labels; /* NULL when unlabeled */
} orc_graph;

typedef struct {
  uint64_t set_ops;
  uint64_t alg_bytes;
  uint64_t roots;
} orc_stats;

/* 0 on success, negative on a malformed pattern. */
int orc_plan_compile_text(const char* text, int labeled, orc_plan* out);

/* Root edges in reference order (r ascending, adjacency order).  Writes up to
 * cap pairs (r,c) into out (may be NULL to count) and returns the total. */
int64_t orc_roots(const orc_graph* g, const orc_plan* p, int32_t* out_pairs, int64_t cap);

/* Exact DFS count over roots [begin,end) of the given root list.  truncate = 0
 * for exact sets, T > 0 to emulate the reference's GRAPH_DEGREE truncation.
 * per_root (optional) receives the raw per-root count.  The returned total is
 * NOT multiplied by the automorphism count; callers apply it for unlabeled
 * plans (test.cu:198). */
uint64_t orc_count(const orc_graph* g, const orc_plan* p, const int32_t* roots,
                   int64_t begin, int64_t end, int truncate, uint64_t* per_root,
                   orc_stats* st);

/* Same, split over nthreads pthreads by root chunks (CPU baseline timing). */
uint64_t orc_count_mt(const orc_graph* g, const orc_plan* p, const int32_t* roots,
                      int64_t begin, int64_t end, int truncate, int nthreads,
                      orc_stats* st);

/* Per-root counts of roots[0, nroots) with each root's DFS divided over
 * nthreads at the candidates of level 1's main slot (the same DFS per piece,
 * so the counts are orc_count's).  Pieces run in a shuffled order when
 * shuffle_seed != 0; with time_limit_s > 0 the run stops at the limit, also
 * inside a piece, and the counts are the matches found by then
 * (*items_done of *items_total pieces finished). */
uint64_t orc_count_split(const orc_graph* g, const orc_plan* p, const int32_t* roots, int64_t nroots,
                         int truncate, int nthreads, double time_limit_s, uint64_t shuffle_seed,
                         uint64_t* per_root, int64_t* items_done, int64_t* items_total, orc_stats* st);

/* Seeded generators with the workload definitions of the product's
 * generators (same edge sets), for inputs built without the product library.
 * Outputs are malloc'd; release with orc_free.  0 on success. */
int orc_gen_chung_lu(int64_t n, int64_t m, double gamma, double i0, double max_w, uint64_t seed,
                     uint64_t** rowptr, int32_t** colidx, int64_t* nadj);
int orc_gen_rmat(int64_t n, int64_t m, double a, double b, double c, uint64_t seed, uint64_t** rowptr,
                 int32_t** colidx, int64_t* nadj);
int orc_gen_labels(int64_t n, int n_labels, uint64_t seed, uint32_t** labels);
void orc_free(void* p);

/* Knuth's random-probe estimator of the DFS tree: estimates the number of set
 * operations and algorithmic bytes of a full run (workload sizing only). */
void orc_estimate(const orc_graph* g, const orc_plan* p, const int32_t* roots, int64_t nroots,
                  int probes, uint64_t seed, double* est_setops, double* est_bytes,
                  double* est_count);

#endif
