/*
 * pm_oracle.c -- CPU oracle for the subgraph-matching hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see pm_oracle.h): the checker for the CUDA path,
 * never linked or called by the product library.
 *
 * Every function restates the reference's algorithm from its source; the
 * citations give the file:line it follows.  Semantics reproduced exactly:
 *   - LABELED (reference default, src/config.h:14): candidate sets are
 *     filtered by label only, no injectivity beyond what intersections imply,
 *     no symmetry breaking (src/gpu_match.cu:274-277, 454-458);
 *   - unlabeled: fresh neighbour sets are diffed against every path vertex,
 *     copies against the newest one (src/gpu_match.cu:534-568, 730-733),
 *     automorphism partial orders bound candidates from above
 *     (src/gpu_match.cu:426-453) and the final count is multiplied by |Aut|
 *     by the caller (test.cu:198);
 *   - optional truncation of every set result to its first T survivors
 *     (GRAPH_DEGREE, src/gpu_match.cu:302,316).
 * One deliberate difference: at the last level the reference diffs a slot it
 * never wrote (compute_set writes nothing at level n-2, src/gpu_match.cu:292,
 * while the unlabeled diff loop at :534-568 reads that slot back), so its
 * unlabeled count for patterns whose last vertex attaches only to the
 * previous one depends on stale device memory.  The oracle (and the CUDA
 * path) use the intended semantics there: the last vertex's fresh candidates
 * minus every path vertex.
 */
#include "pm_oracle.h"

#include <limits.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <math.h>

/* ------------------------------------------------------------------ */
/* Plan compiler: restates PatternPreprocessor (src/pattern.h:48-355). */
/* ------------------------------------------------------------------ */

typedef struct {
  int n;
  int adj[ORC_MAX_PAT][ORC_MAX_PAT];
  int vlabel[ORC_MAX_PAT + 1];
} pat_src;

/* src/pattern.h:67-100: leading '#' lines skipped, then consecutive 'v id
 * label' lines (labels taken in line order; 1 when unlabeled), then 'e a b
 * label' lines setting both directions of the adjacency matrix. */
static int parse_g(const char* text, int labeled, pat_src* ps) {
  memset(ps, 0, sizeof(*ps));
  const char* s = text;
  int phase = 0; /* 0 = header comments, 1 = vertices, 2 = edges */
  while (*s) {
    const char* e = strchr(s, '\n');
    size_t len = e ? (size_t)(e - s) : strlen(s);
    char line[256];
    if (len >= sizeof(line)) return -1;
    memcpy(line, s, len);
    line[len] = 0;
    s = e ? e + 1 : s + len;
    if (len && line[len - 1] == '\r') line[--len] = 0;
    if (len == 0) continue;
    if (phase == 0 && line[0] == '#') continue;
    if (phase <= 1 && line[0] == 'v') {
      phase = 1;
      int id, lab;
      if (sscanf(line, "v %d %d", &id, &lab) != 2) return -1;
      if (ps->n >= ORC_MAX_PAT) return -2;
      if (labeled && (lab < 0 || lab >= 32)) return -3;
      ps->vlabel[ps->n++] = labeled ? lab : 1;
      continue;
    }
    if (phase == 0) return -1;
    phase = 2;
    if (line[0] == '#') continue;
    int a, b, lab;
    if (sscanf(line, "e %d %d %d", &a, &b, &lab) != 3) return -1;
    if (a < 0 || b < 0 || a >= ps->n || b >= ps->n) return -4;
    ps->adj[a][b] = lab;
    ps->adj[b][a] = lab;
  }
  if (ps->n < 3) return -5;
  return 0;
}

/* Heap-free permutation walk over all n! orders (src/pattern.h:124-141
 * enumerates the same set recursively; only the set matters here). */
static int next_perm(int* a, int n) {
  int i = n - 2;
  while (i >= 0 && a[i] >= a[i + 1]) i--;
  if (i < 0) return 0;
  int j = n - 1;
  while (a[j] <= a[i]) j--;
  int t = a[i]; a[i] = a[j]; a[j] = t;
  for (int l = i + 1, r = n - 1; l < r; l++, r--) { t = a[l]; a[l] = a[r]; a[r] = t; }
  return 1;
}

int orc_plan_compile_text(const char* text, int labeled, orc_plan* out) {
  pat_src ps;
  int rc = parse_g(text, labeled, &ps);
  if (rc) return rc;
  const int n = ps.n;
  memset(out, 0, sizeof(*out));
  out->nnodes = n;
  out->labeled = labeled;
  for (int i = 0; i < n; i++) out->vertex_label[i] = ps.vlabel[i];

  /* degrees, identity matching order (src/pattern.h:104-122) */
  for (int i = 0; i < n; i++) {
    int d = 0;
    for (int j = 0; j < n; j++) d += ps.adj[i][j] > 0;
    out->degree[i] = d;
  }

  /* automorphisms and the stabiliser-chain order (src/pattern.h:198-262) */
  static const int fact[8] = {1, 1, 2, 6, 24, 120, 720, 5040};
  int* group = (int*)malloc(sizeof(int) * ORC_MAX_PAT * fact[n]);
  int ng = 0;
  int perm[ORC_MAX_PAT];
  for (int i = 0; i < n; i++) perm[i] = i;
  do {
    /* image adjacency: img[perm[i]] = { perm[j] : adj[i][j] != 0 } */
    uint32_t img[ORC_MAX_PAT] = {0};
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++)
        if (ps.adj[i][j] != 0) img[perm[i]] |= 1u << perm[j];
    int ok = 1;
    for (int i = 0; i < n && ok; i++) {
      uint32_t want = 0;
      for (int j = 0; j < n; j++)
        if (ps.adj[i][j] == 1) want |= 1u << j;
      /* every label-1 neighbour present and the sizes equal */
      if ((want & img[i]) != want || __builtin_popcount(want) != __builtin_popcount(img[i])) ok = 0;
    }
    if (ok) memcpy(group + ORC_MAX_PAT * ng++, perm, sizeof(perm));
  } while (next_perm(perm, n));
  out->multiplicity = ng;

  int L[ORC_MAX_PAT][ORC_MAX_PAT];
  memset(L, 0, sizeof(L));
  for (int v = 0; v < n; v++) {
    int keep = 0;
    for (int g = 0; g < ng; g++) {
      int* x = group + ORC_MAX_PAT * g;
      if (x[v] == v) {
        if (keep != g) memcpy(group + ORC_MAX_PAT * keep, x, sizeof(int) * ORC_MAX_PAT);
        keep++;
      } else {
        L[v][x[v]] = 1;
      }
    }
    ng = keep;
  }
  free(group);

  uint32_t partial[ORC_MAX_PAT][ORC_MAX_PAT];
  memset(partial, 0, sizeof(partial));
  for (int lv = 1; lv < n; lv++)
    for (int j = lv - 1; j >= 0; j--)
      if (L[j][lv]) partial[lv - 1][0] |= 1u << j;

  /* slot factoring (src/pattern.h:143-196).  board[i][k]: bit t set when the
   * slot needs N(path vertex i-t).  Level i's slot 0 feeds pattern vertex i+1. */
  int board[ORC_MAX_PAT][ORC_MAX_PAT + 1];
  int ops[ORC_MAX_PAT][ORC_MAX_PAT + 1];
  int length[ORC_MAX_PAT];
  memset(board, 0, sizeof(board));
  memset(ops, 0, sizeof(ops));
  board[0][0] = 1;
  for (int i = 1; i < n - 1; i++) {
    int m = 0;
    for (int j = 0; j <= i; j++)
      if (ps.adj[i + 1][j]) m |= 1 << (i - j);
    board[i][0] = m;
  }
  for (int i = 0; i < n; i++) length[i] = 1;
  for (int j = 0; j < n - 1; j++) {
    for (int i = n - 2 - j; i >= 0; i--) {
      if (board[i][j] == 0) continue;
      int with_newest = board[i][j] & 1;
      int rest = board[i][j] >> 1;
      if (rest > 0) {
        int k;
        for (k = 1; k < length[i - 1]; k++)
          if (board[i - 1][k] == rest) break;
        if (k == length[i - 1]) {
          if (length[i - 1] >= ORC_MAX_PAT) return -6;
          board[i - 1][length[i - 1]++] = rest;
        }
        ops[i][j] += k + (with_newest << 5);
      } else {
        ops[i][j] |= 0x10;
      }
    }
  }

  /* propagate partial orders to helper slots (src/pattern.h:271-300) */
  for (int i = n - 3; i >= 0; i--) {
    for (int j = 1; j < length[i]; j++) {
      uint32_t m = 0;
      for (int k = 0; k < length[i + 1]; k++) {
        if (!(ops[i + 1][k] & 0x20)) { m = 0; break; }
        if ((ops[i + 1][k] & 0xF) == j) {
          if (partial[i + 1][k] == 0) { m = 0; break; }
          m |= partial[i + 1][k] & ((1u << (i + 1)) - 1);
        }
      }
      partial[i][j] = m;
    }
  }

  /* slot label masks = union of the labels the slot feeds (src/pattern.h:302-327) */
  uint32_t lab[ORC_MAX_PAT][ORC_MAX_PAT];
  memset(lab, 0, sizeof(lab));
  for (int i = 0; i + 1 < n; i++) lab[i][0] = 1u << ps.vlabel[i + 1];
  for (int i = n - 3; i >= 0; i--)
    for (int j = 1; j < length[i]; j++) {
      uint32_t m = 0;
      for (int k = 0; k < length[i + 1]; k++)
        if ((ops[i + 1][k] & 0xF) == j) m |= lab[i + 1][k];
      lab[i][j] = m;
    }

  /* flatten (src/pattern.h:329-355) */
  int flat[ORC_MAX_PAT][ORC_MAX_PAT];
  memset(flat, 0, sizeof(flat));
  int count = 1;
  out->level_begin[0] = 0;
  out->level_begin[1] = 1;
  out->partial[0] = partial[0][0];
  for (int i = 1; i < n - 1; i++) {
    for (int j = 0; j < length[i]; j++) {
      if (count >= ORC_MAX_SLOTS) return -7;
      flat[i][j] = count;
      out->slot_labels[count] = lab[i][j];
      out->partial[count] = partial[i][j];
      int parent = (i > 1) ? flat[i - 1][ops[i][j] & 0x0F] : 0;
      out->set_ops[count] = (uint8_t)(((ops[i][j] & 0x30) << 1) + parent);
      count++;
    }
    out->level_begin[i + 1] = count;
  }
  for (int i = n; i <= ORC_MAX_PAT; i++) out->level_begin[i] = count;
  out->nslots = count;
  return 0;
}

/* ------------------------------------------------------------------ */
/* Root filter: restates JobQueuePreprocessor (src/job_queue.h:39-64).  */
/* ------------------------------------------------------------------ */

static inline int64_t deg_of(const orc_graph* g, int64_t v) {
  return (int64_t)(g->rowptr[v + 1] - g->rowptr[v]);
}

int64_t orc_roots(const orc_graph* g, const orc_plan* p, int32_t* out, int64_t cap) {
  int64_t cnt = 0;
  const int need_gt = (!p->labeled && p->partial[0] == 1);
  for (int64_t r = 0; r < g->n; r++) {
    if (p->labeled && g->labels[r] != (uint32_t)p->vertex_label[0]) continue;
    if (deg_of(g, r) < p->degree[0]) continue;
    for (uint64_t e = g->rowptr[r]; e < g->rowptr[r + 1]; e++) {
      int64_t c = g->colidx[e];
      if (need_gt && !(r > c)) continue;
      if (p->labeled && g->labels[c] != (uint32_t)p->vertex_label[1]) continue;
      if (deg_of(g, c) < p->degree[1]) continue;
      int ok = 0;
      for (uint64_t d = g->rowptr[c]; d < g->rowptr[c + 1]; d++)
        if (deg_of(g, g->colidx[d]) >= p->degree[2]) { ok = 1; break; }
      if (!ok) continue;
      if (out && cnt < cap) { out[2 * cnt] = (int32_t)r; out[2 * cnt + 1] = (int32_t)c; }
      cnt++;
    }
  }
  return cnt;
}

/* ------------------------------------------------------------------ */
/* DFS: restates match/extend/compute_set (src/gpu_match.cu).           */
/* ------------------------------------------------------------------ */

typedef struct {
  const orc_graph* g;
  const orc_plan* p;
  int T;
  int32_t* buf[ORC_MAX_SLOTS];
  int64_t size[ORC_MAX_SLOTS];
  int32_t path[ORC_MAX_PAT];
  orc_stats st;
  double deadline; /* CLOCK_MONOTONIC seconds; 0 = none (timed runs stop at it) */
  int stopped;
} dfs_t;

static double mono_s(void);

/* number of elements of a[0,len) strictly below ub (upper_bound with the
 * reference's comparison, src/gpu_match.cu:185-202) */
static int64_t below(const int32_t* a, int64_t len, int64_t ub) {
  int64_t lo = 0, hi = len;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < ub) lo = mid + 1; else hi = mid;
  }
  return lo;
}

static inline int labok(const dfs_t* d, uint32_t mask, int32_t v) {
  return (mask >> d->g->labels[v]) & 1u;
}

/* Computes slot s of level L for the current path; returns the slot size
 * (for the last level: the count, nothing materialised). */
static int64_t compute_slot(dfs_t* d, int L, int s) {
  const orc_plan* p = d->p;
  const orc_graph* g = d->g;
  const int last = (L == p->nnodes - 2);
  const int is_main = (s == p->level_begin[L]);
  const int labeled = p->labeled;

  /* upper bound from partial orders (src/gpu_match.cu:426-458) */
  int64_t ub = INT_MAX;
  if (!labeled && p->partial[s]) {
    ub = is_main ? INT_MAX : -1;
    for (int j = 0; j <= L; j++) {
      if (!(p->partial[s] & (1u << j))) continue;
      int64_t v = d->path[j];
      if (is_main) { if (v <= ub) ub = v; }
      else { if (ub < v) ub = v; }
    }
    if (ub == -1) ub = INT_MAX;
  }

  const uint8_t op = p->set_ops[s];
  const int parent = op & 0x1F;
  const int32_t *A, *B = NULL;
  int64_t lenA, lenB = 0;
  int kind; /* 0 fresh, 1 intersect, 2 copy */
  const int32_t vL = d->path[L];
  if (op & 0x20) {
    kind = 0;
    A = g->colidx + g->rowptr[vL]; lenA = deg_of(g, vL);
  } else if (op & 0x40) {
    kind = 1;
    A = g->colidx + g->rowptr[vL]; lenA = deg_of(g, vL);
    if (L > 1) { B = d->buf[parent]; lenB = d->size[parent]; }
    else { B = g->colidx + g->rowptr[d->path[0]]; lenB = deg_of(g, d->path[0]); }
  } else {
    kind = 2;
    if (L > 1) { A = d->buf[parent]; lenA = d->size[parent]; }
    else { A = g->colidx + g->rowptr[d->path[0]]; lenA = deg_of(g, d->path[0]); }
  }
  lenA = below(A, lenA, ub);

  const uint32_t mask = p->slot_labels[s];
  const int T = d->T;
  int32_t* out = d->buf[s];
  int64_t cnt = 0;
  int64_t bpos = 0;
  for (int64_t i = 0; i < lenA; i++) {
    const int32_t a = A[i];
    if (labeled && !labok(d, mask, a)) continue;
    if (kind == 1) {
      /* membership in the sorted B: advance a monotone cursor (A is sorted) */
      int64_t lo = bpos, step = 1;
      while (lo + step < lenB && B[lo + step] < a) { lo += step; step <<= 1; }
      int64_t hi = lo + step < lenB ? lo + step + 1 : lenB;
      while (lo < hi) { int64_t mid = (lo + hi) >> 1; if (B[mid] < a) lo = mid + 1; else hi = mid; }
      bpos = lo;
      if (!(lo < lenB && B[lo] == a)) continue;
    } else if (kind == 2 && !labeled) {
      if (a == vL) continue;
    }
    if (!last && (T == 0 || cnt < T)) out[cnt] = a;
    cnt++;
  }
  int64_t size = (T && cnt > T) ? T : cnt;

  if (kind == 0 && !labeled) {
    /* diff the fresh set with every path vertex v_L..v_0 */
    int64_t keep = 0;
    const int32_t* src = last ? A : out; /* unlabeled fresh keeps A's prefix */
    for (int64_t i = 0; i < size; i++) {
      int32_t a = src[i];
      int hit = 0;
      for (int j = 0; j <= L; j++) hit |= (a == d->path[j]);
      if (hit) continue;
      if (!last) out[keep] = a;
      keep++;
    }
    size = keep;
  }
  d->st.set_ops++;
  d->st.alg_bytes += 4u * (uint64_t)(lenA + lenB + size) + (labeled ? (uint64_t)lenA : 0u);
  d->size[s] = size;
  return size;
}

static uint64_t extend(dfs_t* d, int L) {
  const orc_plan* p = d->p;
  const int b = p->level_begin[L], e = p->level_begin[L + 1];
  if (L == p->nnodes - 2) return (uint64_t)compute_slot(d, L, b);
  for (int s = b; s < e; s++) compute_slot(d, L, s);
  uint64_t total = 0;
  const int64_t m = d->size[b];
  const int32_t* cand = d->buf[b];
  for (int64_t i = 0; i < m && !d->stopped; i++) {
    d->path[L + 1] = cand[i];
    total += extend(d, L + 1);
    /* timed runs: stop at the deadline, keeping the matches found so far */
    if (d->deadline > 0 && (i & 63) == 63 && mono_s() >= d->deadline) d->stopped = 1;
  }
  return total;
}

static int64_t max_degree(const orc_graph* g) {
  int64_t m = 0;
  for (int64_t v = 0; v < g->n; v++) { int64_t x = deg_of(g, v); if (x > m) m = x; }
  return m;
}

static void dfs_init(dfs_t* d, const orc_graph* g, const orc_plan* p, int T, int64_t maxdeg) {
  memset(d, 0, sizeof(*d));
  d->g = g; d->p = p; d->T = T;
  for (int s = 0; s < ORC_MAX_SLOTS; s++) d->buf[s] = (int32_t*)malloc(sizeof(int32_t) * (size_t)(maxdeg + 1));
}

static void dfs_free(dfs_t* d) {
  for (int s = 0; s < ORC_MAX_SLOTS; s++) free(d->buf[s]);
}

uint64_t orc_count(const orc_graph* g, const orc_plan* p, const int32_t* roots,
                   int64_t begin, int64_t end, int truncate, uint64_t* per_root,
                   orc_stats* st) {
  dfs_t d;
  dfs_init(&d, g, p, truncate, max_degree(g));
  uint64_t total = 0;
  for (int64_t r = begin; r < end; r++) {
    d.path[0] = roots[2 * r];
    d.path[1] = roots[2 * r + 1];
    uint64_t c = extend(&d, 1);
    d.st.alg_bytes += 8;
    d.st.roots++;
    if (per_root) per_root[r - begin] = c;
    total += c;
  }
  if (st) *st = d.st;
  dfs_free(&d);
  return total;
}

typedef struct {
  const orc_graph* g;
  const orc_plan* p;
  const int32_t* roots;
  int64_t end;
  int T;
  int64_t maxdeg;
  volatile int64_t* cursor;
  uint64_t total;
  orc_stats st;
} mt_arg;

static void* mt_worker(void* v) {
  mt_arg* a = (mt_arg*)v;
  dfs_t d;
  dfs_init(&d, a->g, a->p, a->T, a->maxdeg);
  const int64_t chunk = 64;
  for (;;) {
    int64_t b = __atomic_fetch_add(a->cursor, chunk, __ATOMIC_RELAXED);
    if (b >= a->end) break;
    int64_t e = b + chunk < a->end ? b + chunk : a->end;
    for (int64_t r = b; r < e; r++) {
      d.path[0] = a->roots[2 * r];
      d.path[1] = a->roots[2 * r + 1];
      a->total += extend(&d, 1);
      d.st.alg_bytes += 8;
      d.st.roots++;
    }
  }
  a->st = d.st;
  dfs_free(&d);
  return NULL;
}

uint64_t orc_count_mt(const orc_graph* g, const orc_plan* p, const int32_t* roots,
                      int64_t begin, int64_t end, int truncate, int nthreads,
                      orc_stats* st) {
  if (nthreads < 1) nthreads = 1;
  int64_t cursor = begin;
  int64_t md = max_degree(g);
  mt_arg* args = (mt_arg*)calloc((size_t)nthreads, sizeof(mt_arg));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  for (int t = 0; t < nthreads; t++) {
    args[t].g = g; args[t].p = p; args[t].roots = roots; args[t].end = end;
    args[t].T = truncate; args[t].maxdeg = md; args[t].cursor = &cursor;
    pthread_create(&th[t], NULL, mt_worker, &args[t]);
  }
  uint64_t total = 0;
  orc_stats agg = {0, 0, 0};
  for (int t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    total += args[t].total;
    agg.set_ops += args[t].st.set_ops;
    agg.alg_bytes += args[t].st.alg_bytes;
    agg.roots += args[t].st.roots;
  }
  if (st) *st = agg;
  free(args);
  free(th);
  return total;
}

static uint64_t sm64(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

/* ------------------------------------------------------------------ */
/* Split runs: one root's DFS divided over threads at level 1's main    */
/* slot.  Same DFS (extend) per piece, so per-root counts are those of  */
/* orc_count; only the work division differs.                           */
/* ------------------------------------------------------------------ */

typedef struct {
  const orc_graph* g;
  const orc_plan* p;
  const int32_t* roots;
  const int64_t* item_root; /* per item: root index; item_k: level-1 candidate (-1 = whole root) */
  const int32_t* item_k;
  int64_t nitems;
  int T;
  int64_t maxdeg;
  double deadline; /* CLOCK_MONOTONIC seconds, 0 = none */
  volatile int64_t* cursor;
  volatile int64_t* done;
  uint64_t* per_root;
  uint64_t total;
  orc_stats st;
} split_arg;

static double mono_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void* split_worker(void* v) {
  split_arg* a = (split_arg*)v;
  dfs_t d;
  dfs_init(&d, a->g, a->p, a->T, a->maxdeg);
  d.deadline = a->deadline;
  for (;;) {
    if (d.stopped || (a->deadline > 0 && mono_s() >= a->deadline)) break;
    const int64_t i = __atomic_fetch_add(a->cursor, 1, __ATOMIC_RELAXED);
    if (i >= a->nitems) break;
    const int64_t r = a->item_root[i];
    const int k = a->item_k[i];
    d.path[0] = a->roots[2 * r];
    d.path[1] = a->roots[2 * r + 1];
    uint64_t c;
    if (k < 0) {
      c = extend(&d, 1);
    } else {
      /* level 1 again for this root (its set operations were counted once
       * by the caller), then the subtree of candidate k */
      const orc_stats keep = d.st;
      const int b = a->p->level_begin[1], e = a->p->level_begin[2];
      for (int s = b; s < e; s++) compute_slot(&d, 1, s);
      d.st = keep;
      d.path[2] = d.buf[b][k];
      c = extend(&d, 2);
    }
    if (a->per_root) __atomic_fetch_add(&a->per_root[r], c, __ATOMIC_RELAXED);
    a->total += c;
    if (!d.stopped) __atomic_fetch_add(a->done, 1, __ATOMIC_RELAXED);
  }
  a->st = d.st;
  dfs_free(&d);
  return NULL;
}

uint64_t orc_count_split(const orc_graph* g, const orc_plan* p, const int32_t* roots, int64_t nroots,
                         int truncate, int nthreads, double time_limit_s, uint64_t shuffle_seed,
                         uint64_t* per_root, int64_t* items_done, int64_t* items_total, orc_stats* st) {
  if (nthreads < 1) nthreads = 1;
  const int64_t md = max_degree(g);
  const double t0 = mono_s();
  orc_stats agg = {0, 0, 0};
  /* items: (root, level-1 candidate) for plans of 4+ vertices, whole roots otherwise */
  int64_t nitems = 0, cap = nroots > 0 ? nroots : 1;
  int64_t* item_root = (int64_t*)malloc(sizeof(int64_t) * (size_t)cap);
  int32_t* item_k = (int32_t*)malloc(sizeof(int32_t) * (size_t)cap);
  uint64_t* pr = per_root ? per_root : (uint64_t*)calloc((size_t)cap, sizeof(uint64_t));
  if (per_root) memset(per_root, 0, sizeof(uint64_t) * (size_t)nroots);
  {
    dfs_t d;
    dfs_init(&d, g, p, truncate, md);
    const int deep = p->nnodes > 3;
    for (int64_t r = 0; r < nroots; r++) {
      int64_t m = 1;
      if (deep) {
        d.path[0] = roots[2 * r];
        d.path[1] = roots[2 * r + 1];
        const int b = p->level_begin[1], e = p->level_begin[2];
        for (int s = b; s < e; s++) compute_slot(&d, 1, s);
        m = d.size[b];
      }
      d.st.alg_bytes += 8;
      d.st.roots++;
      if (nitems + m > cap) {
        while (nitems + m > cap) cap *= 2;
        item_root = (int64_t*)realloc(item_root, sizeof(int64_t) * (size_t)cap);
        item_k = (int32_t*)realloc(item_k, sizeof(int32_t) * (size_t)cap);
      }
      for (int64_t k = 0; k < m; k++) {
        item_root[nitems] = r;
        item_k[nitems] = deep ? (int32_t)k : -1;
        nitems++;
      }
    }
    agg = d.st;
    dfs_free(&d);
  }
  if (shuffle_seed) {
    uint64_t s = shuffle_seed;
    for (int64_t i = nitems - 1; i > 0; i--) {
      const int64_t j = (int64_t)(sm64(&s) % (uint64_t)(i + 1));
      const int64_t tr = item_root[i]; item_root[i] = item_root[j]; item_root[j] = tr;
      const int32_t tk = item_k[i]; item_k[i] = item_k[j]; item_k[j] = tk;
    }
  }
  int64_t cursor = 0, done = 0;
  split_arg* args = (split_arg*)calloc((size_t)nthreads, sizeof(split_arg));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  for (int t = 0; t < nthreads; t++) {
    split_arg* a = &args[t];
    a->g = g; a->p = p; a->roots = roots; a->item_root = item_root; a->item_k = item_k;
    a->nitems = nitems; a->T = truncate; a->maxdeg = md;
    a->deadline = time_limit_s > 0 ? t0 + time_limit_s : 0;
    a->cursor = &cursor; a->done = &done; a->per_root = pr;
    pthread_create(&th[t], NULL, split_worker, a);
  }
  uint64_t total = 0;
  for (int t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    total += args[t].total;
    agg.set_ops += args[t].st.set_ops;
    agg.alg_bytes += args[t].st.alg_bytes;
  }
  if (items_done) *items_done = done;
  if (items_total) *items_total = nitems;
  if (st) *st = agg;
  if (!per_root) free(pr);
  free(args);
  free(th);
  free(item_root);
  free(item_k);
  return total;
}

/* ------------------------------------------------------------------ */
/* Knuth estimator (workload sizing only).                              */
/* ------------------------------------------------------------------ */

void orc_estimate(const orc_graph* g, const orc_plan* p, const int32_t* roots, int64_t nroots,
                  int probes, uint64_t seed, double* est_setops, double* est_bytes,
                  double* est_count) {
  dfs_t d;
  dfs_init(&d, g, p, 0, max_degree(g));
  double so = 0, by = 0, ct = 0;
  uint64_t rs = seed;
  for (int k = 0; k < probes && nroots > 0; k++) {
    int64_t r = (int64_t)(sm64(&rs) % (uint64_t)nroots);
    d.path[0] = roots[2 * r];
    d.path[1] = roots[2 * r + 1];
    double w = 1.0;
    for (int L = 1; L <= p->nnodes - 2; L++) {
      uint64_t so0 = d.st.set_ops, by0 = d.st.alg_bytes;
      int b = p->level_begin[L], e = p->level_begin[L + 1];
      if (L == p->nnodes - 2) {
        int64_t c = compute_slot(&d, L, b);
        so += w * (double)(d.st.set_ops - so0);
        by += w * (double)(d.st.alg_bytes - by0);
        ct += w * (double)c;
        break;
      }
      for (int s = b; s < e; s++) compute_slot(&d, L, s);
      so += w * (double)(d.st.set_ops - so0);
      by += w * (double)(d.st.alg_bytes - by0);
      int64_t m = d.size[b];
      if (m == 0) break;
      w *= (double)m;
      d.path[L + 1] = d.buf[b][sm64(&rs) % (uint64_t)m];
    }
  }
  dfs_free(&d);
  double f = probes > 0 ? (double)nroots / probes : 0;
  *est_setops = so * f;
  *est_bytes = by * f;
  *est_count = ct * f;
}

/* ------------------------------------------------------------------ */
/* Seeded graph generators.  Restate the workload definitions the       */
/* product's generators implement (splitmix64-seeded xoshiro256**       */
/* streams, one stream per batch of 65,536 draws, the first m distinct  */
/* undirected edges of the draw sequence, sorted CSR), sequentially and */
/* with a hash set instead of sorted rounds: the same edge set.  Used   */
/* by the CPU measurement arm so that it builds its inputs without the  */
/* product library.                                                     */
/* ------------------------------------------------------------------ */

typedef struct { uint64_t s[4]; } orc_rng;

static void rng_init(orc_rng* r, uint64_t seed, uint64_t stream) {
  uint64_t x = seed ^ (stream * 0xD1B54A32D192ED03ull);
  for (int i = 0; i < 4; i++) r->s[i] = sm64(&x);
}
static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t rng_next(orc_rng* r) {
  uint64_t* s = r->s;
  const uint64_t res = rotl64(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
  s[2] ^= t; s[3] = rotl64(s[3], 45);
  return res;
}
static inline double rng_uniform(orc_rng* r) { return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static inline uint32_t rng_below(orc_rng* r, uint32_t n) {
  return (uint32_t)(((rng_next(r) >> 32) * (uint64_t)n) >> 32);
}

/* open-addressing set of edge keys (key + 1 stored, 0 = empty) */
typedef struct { uint64_t* t; uint64_t mask; int64_t size; } keyset;

static int keyset_add(keyset* k, uint64_t key) {
  uint64_t h = (key * 0x9E3779B97F4A7C15ull) >> 20;
  for (;;) {
    h &= k->mask;
    if (k->t[h] == 0) { k->t[h] = key + 1; k->size++; return 1; }
    if (k->t[h] == key + 1) return 0;
    h++;
  }
}

static int cmp_u64(const void* a, const void* b) {
  const uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return x < y ? -1 : x > y;
}
static int cmp_i32(const void* a, const void* b) {
  const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return x < y ? -1 : x > y;
}

/* draw(ctx, rng) returns an edge key (lo << 32 | hi, lo < hi) or UINT64_MAX */
typedef uint64_t (*draw_fn)(void* ctx, orc_rng* r);

static int gen_edges(int64_t n, int64_t m, uint64_t seed, draw_fn draw, void* ctx, uint64_t** rowptr_out,
                     int32_t** colidx_out, int64_t* nadj_out) {
  uint64_t cap = 1;
  while (cap < (uint64_t)(2 * m + 16)) cap <<= 1;
  keyset ks = {(uint64_t*)calloc(cap, sizeof(uint64_t)), cap - 1, 0};
  uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(m > 0 ? m : 1));
  if (!ks.t || !keys) return -1;
  const int64_t kBatch = 1 << 16;
  for (uint64_t batch = 1; ks.size < m; batch++) {
    if (batch > (uint64_t)(64 * (m / kBatch + 2) + 4096)) break; /* too dense */
    orc_rng r;
    rng_init(&r, seed, batch);
    for (int64_t k = 0; k < kBatch && ks.size < m; k++) {
      const uint64_t key = draw(ctx, &r);
      if (key != UINT64_MAX && keyset_add(&ks, key)) keys[ks.size - 1] = key;
    }
  }
  free(ks.t);
  if (ks.size != m) { free(keys); return -2; }
  qsort(keys, (size_t)m, sizeof(uint64_t), cmp_u64);
  uint64_t* rowptr = (uint64_t*)calloc((size_t)n + 1, sizeof(uint64_t));
  for (int64_t e = 0; e < m; e++) { rowptr[(keys[e] >> 32) + 1]++; rowptr[(keys[e] & 0xffffffffu) + 1]++; }
  for (int64_t v = 0; v < n; v++) rowptr[v + 1] += rowptr[v];
  const int64_t nadj = (int64_t)rowptr[n];
  int32_t* colidx = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nadj > 0 ? nadj : 1));
  uint64_t* fill = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
  memcpy(fill, rowptr, sizeof(uint64_t) * (size_t)n);
  for (int64_t e = 0; e < m; e++) {
    const uint32_t lo = (uint32_t)(keys[e] >> 32), hi = (uint32_t)(keys[e] & 0xffffffffu);
    colidx[fill[lo]++] = (int32_t)hi;
    colidx[fill[hi]++] = (int32_t)lo;
  }
  for (int64_t v = 0; v < n; v++)
    qsort(colidx + rowptr[v], (size_t)(rowptr[v + 1] - rowptr[v]), sizeof(int32_t), cmp_i32);
  free(fill);
  free(keys);
  *rowptr_out = rowptr;
  *colidx_out = colidx;
  *nadj_out = nadj;
  return 0;
}

static inline uint64_t edge_key32(uint32_t u, uint32_t v) {
  return u < v ? ((uint64_t)u << 32 | v) : ((uint64_t)v << 32 | u);
}

typedef struct { uint32_t n; const double* prob; const uint32_t* alias; } cl_ctx;

static uint64_t cl_draw(void* c, orc_rng* r) {
  const cl_ctx* x = (const cl_ctx*)c;
  uint32_t e[2];
  for (int q = 0; q < 2; q++) {
    const uint32_t i = rng_below(r, x->n);
    e[q] = rng_uniform(r) < x->prob[i] ? i : x->alias[i];
  }
  return e[0] == e[1] ? UINT64_MAX : edge_key32(e[0], e[1]);
}

/* Chung-Lu: expected degrees w_i ~ (i + i0)^(-1/(gamma-1)) scaled to sum 2m
 * and capped at max_w; both endpoints drawn proportional to w (Vose alias
 * table, built in the same order of operations so the doubles agree). */
int orc_gen_chung_lu(int64_t n, int64_t m, double gamma, double i0, double max_w, uint64_t seed,
                     uint64_t** rowptr, int32_t** colidx, int64_t* nadj) {
  if (n < 2 || n > INT_MAX || m < 0 || gamma <= 1.0) return -1;
  double* w = (double*)malloc(sizeof(double) * (size_t)n);
  double sum = 0;
  for (int64_t i = 0; i < n; i++) { w[i] = pow((double)i + i0, -1.0 / (gamma - 1.0)); sum += w[i]; }
  for (int64_t i = 0; i < n; i++) { w[i] *= 2.0 * (double)m / sum; if (max_w > 0 && w[i] > max_w) w[i] = max_w; }
  double tot = 0;
  for (int64_t i = 0; i < n; i++) tot += w[i];
  double* prob = (double*)malloc(sizeof(double) * (size_t)n);
  uint32_t* alias = (uint32_t*)calloc((size_t)n, sizeof(uint32_t));
  int64_t* small = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  int64_t* large = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
  int64_t ns = 0, nl = 0;
  for (int64_t i = 0; i < n; i++) {
    prob[i] = w[i] * (double)n / tot;
    if (prob[i] < 1.0) small[ns++] = i; else large[nl++] = i;
  }
  while (ns > 0 && nl > 0) {
    const int64_t s = small[--ns];
    const int64_t l = large[nl - 1];
    alias[s] = (uint32_t)l;
    prob[l] = prob[l] + prob[s] - 1.0;
    if (prob[l] < 1.0) { nl--; small[ns++] = l; }
  }
  for (int64_t i = 0; i < nl; i++) prob[large[i]] = 1.0;
  for (int64_t i = 0; i < ns; i++) prob[small[i]] = 1.0;
  free(small);
  free(large);
  free(w);
  cl_ctx c = {(uint32_t)n, prob, alias};
  const int rc = gen_edges(n, m, seed, cl_draw, &c, rowptr, colidx, nadj);
  free(prob);
  free(alias);
  return rc;
}

typedef struct { int scale; uint64_t n; uint32_t ta, tb, tc; } rmat_ctx;

static uint64_t rmat_draw(void* c, orc_rng* r) {
  const rmat_ctx* x = (const rmat_ctx*)c;
  uint64_t u = 0, v = 0, bits = 0;
  for (int l = 0; l < x->scale; l++) {
    if ((l & 3) == 0) bits = rng_next(r);
    const uint32_t q = (uint32_t)(bits & 0xffff);
    bits >>= 16;
    const uint32_t bu = q >= x->tb, bv = (q >= x->ta && q < x->tb) || q >= x->tc;
    u = (u << 1) | bu;
    v = (v << 1) | bv;
  }
  return (u >= x->n || v >= x->n || u == v) ? UINT64_MAX : edge_key32((uint32_t)u, (uint32_t)v);
}

/* R-MAT: per level one 16-bit draw picks the quadrant (a, b, c, d); ids >= n
 * and self-loops are rejected. */
int orc_gen_rmat(int64_t n, int64_t m, double a, double b, double c, uint64_t seed, uint64_t** rowptr,
                 int32_t** colidx, int64_t* nadj) {
  if (n < 2 || n > INT_MAX || m < 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
  rmat_ctx x;
  x.scale = 0;
  while ((1ll << x.scale) < n) x.scale++;
  x.n = (uint64_t)n;
  x.ta = (uint32_t)llround(a * 65536.0);
  x.tb = (uint32_t)llround((a + b) * 65536.0);
  x.tc = (uint32_t)llround((a + b + c) * 65536.0);
  return gen_edges(n, m, seed, rmat_draw, &x, rowptr, colidx, nadj);
}

/* Uniform labels in [0, n_labels): vertex block b of 65,536 from stream b+1. */
int orc_gen_labels(int64_t n, int n_labels, uint64_t seed, uint32_t** labels) {
  if (n < 0 || n_labels < 1 || n_labels > 32) return -1;
  uint32_t* lab = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
  const int64_t kBlock = 1 << 16;
  for (int64_t b = 0; b < (n + kBlock - 1) / kBlock; b++) {
    orc_rng r;
    rng_init(&r, seed, (uint64_t)b + 1);
    const int64_t e = (b + 1) * kBlock < n ? (b + 1) * kBlock : n;
    for (int64_t v = b * kBlock; v < e; v++) lab[v] = rng_below(&r, (uint32_t)n_labels);
  }
  *labels = lab;
  return 0;
}

void orc_free(void* p) { free(p); }
