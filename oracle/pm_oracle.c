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
} dfs_t;

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
  for (int64_t i = 0; i < m; i++) {
    d->path[L + 1] = cand[i];
    total += extend(d, L + 1);
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

/* ------------------------------------------------------------------ */
/* Knuth estimator (workload sizing only).                              */
/* ------------------------------------------------------------------ */

static uint64_t sm64(uint64_t* s) {
  uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

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
