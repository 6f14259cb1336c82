// pm_host.cpp -- host half of libpumatch_b200.so: error plumbing, the pattern
// plan compiler, the CSR file format and the seeded graph generators.
//
// Nothing here touches the GPU; these entry points also work on a machine
// without one (the matching entry points in pm_device.cu do not).
#include <parallel/algorithm>
#include <omp.h>

#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <fstream>
#include <memory>
#include <set>
#include <sstream>

#include "pm_common.h"

namespace pm {

static thread_local std::string g_last_error;

pm_status fail(pm_status s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

// =====================================================================
// Pattern plan compiler.
//
// Produces the same flattened plan as the reference's PatternPreprocessor
// (src/pattern.h:48-58): identity matching order, per-level "which earlier
// vertices must be adjacent" masks factored into reusable slots, automorphism
// partial orders and slot label masks.  The plan is the kernel's contract.
// =====================================================================

namespace {

struct GFile {
  int n = 0;
  int adj[PM_MAX_PAT][PM_MAX_PAT] = {{0}};
  int label[PM_MAX_PAT + 1] = {0};
};

// .g grammar (src/pattern.h:67-100): optional leading '#' lines, then
// consecutive "v <id> <label>" lines whose labels are taken in line order,
// then "e <a> <b> <label>" lines; an edge label of 0 means "no edge".
pm_status parse_g(const std::string& text, bool labeled, GFile* g) {
  std::istringstream in(text);
  std::string line;
  enum { HEAD, VERTS, EDGES } phase = HEAD;
  int lineno = 0;
  while (std::getline(in, line)) {
    lineno++;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty()) continue;
    if (line[0] == '#' && phase != VERTS) continue;
    std::istringstream ls(line);
    char tag = 0;
    ls >> tag;
    if (tag == 'v' && phase != EDGES) {
      phase = VERTS;
      int id = 0, lab = 0;
      if (!(ls >> id >> lab)) return fail(PM_ERR_FORMAT, ".g line %d: bad vertex line", lineno);
      if (g->n >= PM_MAX_PAT) return fail(PM_ERR_FORMAT, ".g: more than %d vertices", PM_MAX_PAT);
      if (labeled && (lab < 0 || lab >= 32))
        return fail(PM_ERR_FORMAT, ".g line %d: label %d outside [0,32)", lineno, lab);
      g->label[g->n++] = labeled ? lab : 1;
      continue;
    }
    if (tag != 'e' || phase == HEAD)
      return fail(PM_ERR_FORMAT, ".g line %d: unexpected '%c'", lineno, tag);
    phase = EDGES;
    int a = 0, b = 0, lab = 0;
    if (!(ls >> a >> b >> lab)) return fail(PM_ERR_FORMAT, ".g line %d: bad edge line", lineno);
    if (a < 0 || b < 0 || a >= g->n || b >= g->n)
      return fail(PM_ERR_FORMAT, ".g line %d: edge endpoint out of range", lineno);
    g->adj[a][b] = g->adj[b][a] = lab;
  }
  if (g->n < 3) return fail(PM_ERR_FORMAT, ".g: patterns need 3..%d vertices (got %d)", PM_MAX_PAT, g->n);
  return PM_OK;
}

// One intermediate set ("slot") of the factored plan, before flattening.
struct SlotSrc {
  int need = 0;         // bit t: must be adjacent to path vertex (level - t)
  int op = 0;           // bit 0x20 intersect-with-newest, 0x10 fresh, low 4 bits parent
  uint32_t partial = 0;
  uint32_t labels = 0;
};

}  // namespace

pm_status compile_plan(const std::string& text, bool labeled, Plan* out) {
  GFile g;
  pm_status st = parse_g(text, labeled, &g);
  if (st != PM_OK) return st;
  const int n = g.n;
  Plan p;
  p.nnodes = n;
  p.labeled = labeled ? 1 : 0;
  for (int i = 0; i < n; i++) {
    p.vertex_label[i] = g.label[i];
    for (int j = 0; j < n; j++) p.degree[i] += g.adj[i][j] > 0;
  }

  // Automorphism group.  A permutation q is kept when the neighbourhood of
  // every vertex under q equals its label-1 neighbourhood (src/pattern.h:207-234).
  std::vector<std::vector<int>> aut;
  std::vector<int> q(n);
  for (int i = 0; i < n; i++) q[i] = i;
  do {
    std::vector<uint32_t> image(n, 0);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++)
        if (g.adj[i][j] != 0) image[q[i]] |= 1u << q[j];
    bool ok = true;
    for (int i = 0; i < n && ok; i++) {
      uint32_t ones = 0;
      for (int j = 0; j < n; j++)
        if (g.adj[i][j] == 1) ones |= 1u << j;
      ok = ((ones & image[i]) == ones) && __builtin_popcount(ones) == __builtin_popcount(image[i]);
    }
    if (ok) aut.push_back(q);
  } while (std::next_permutation(q.begin(), q.end()));
  p.multiplicity = (int)aut.size();

  // Stabiliser chain: vertex v must be ordered against every vertex it can
  // be mapped to while v's predecessors are fixed (src/pattern.h:238-261).
  bool less_than[PM_MAX_PAT][PM_MAX_PAT] = {{false}};
  for (int v = 0; v < n; v++) {
    std::vector<std::vector<int>> fixed;
    for (auto& x : aut) {
      if (x[v] == v) fixed.push_back(x);
      else less_than[v][x[v]] = true;
    }
    aut.swap(fixed);
  }

  // levels[i] = slots computed at level i (candidates for vertex i+1 first).
  std::vector<std::vector<SlotSrc>> levels(n);
  levels[0].push_back(SlotSrc{1, 0, 0, 0});
  for (int i = 1; i + 1 < n; i++) {
    SlotSrc s;
    for (int j = 0; j <= i; j++)
      if (g.adj[i + 1][j]) s.need |= 1 << (i - j);
    levels[i].push_back(s);
  }
  for (int lv = 1; lv < n; lv++)
    for (int j = 0; j < lv; j++)
      if (less_than[j][lv]) levels[lv - 1][0].partial |= 1u << j;

  // Factor: slot k of level i needs N(newest) (bit 0) and the rest, which is
  // a slot of level i-1, shared when an identical one exists (src/pattern.h:159-191).
  for (int k = 0; k + 1 < n; k++) {
    for (int i = n - 2 - k; i >= 0; i--) {
      if (k >= (int)levels[i].size()) continue;
      SlotSrc& s = levels[i][k];
      if (s.need == 0) continue;
      const int newest = s.need & 1, rest = s.need >> 1;
      if (rest == 0) { s.op |= 0x10; continue; }
      auto& prev = levels[i - 1];
      int at = 1;
      while (at < (int)prev.size() && prev[at].need != rest) at++;
      if (at == (int)prev.size()) {
        if ((int)prev.size() >= PM_MAX_PAT) return fail(PM_ERR_FORMAT, ".g: plan too wide");
        SlotSrc ns;
        ns.need = rest;
        prev.push_back(ns);
      }
      // re-fetch: push_back may move levels[i-1] but not levels[i]
      levels[i][k].op += at + (newest << 5);
    }
  }

  // Helper slots inherit the partial order of their consumers when every
  // consumer one level down is an intersection (src/pattern.h:271-300).
  for (int i = n - 3; i >= 0; i--) {
    for (int j = 1; j < (int)levels[i].size(); j++) {
      uint32_t m = 0;
      for (const SlotSrc& c : levels[i + 1]) {
        if (!(c.op & 0x20)) { m = 0; break; }
        if ((c.op & 0xF) != j) continue;
        if (c.partial == 0) { m = 0; break; }
        m |= c.partial & ((1u << (i + 1)) - 1);
      }
      levels[i][j].partial = m;
    }
  }

  // Label masks: a main slot keeps its own vertex's label; a helper slot the
  // union over the slots it feeds (src/pattern.h:302-327).
  for (int i = 0; i + 1 < n; i++) levels[i][0].labels = 1u << g.label[i + 1];
  for (int i = n - 3; i >= 0; i--)
    for (int j = 1; j < (int)levels[i].size(); j++) {
      uint32_t m = 0;
      for (const SlotSrc& c : levels[i + 1])
        if ((c.op & 0xF) == j) m |= c.labels;
      levels[i][j].labels = m;
    }

  // Flatten: level 0 is the root slot; parents become flat indices
  // (src/pattern.h:329-355).
  int flat_of[PM_MAX_PAT][PM_MAX_PAT] = {{0}};
  int next = 1;
  p.level_begin[0] = 0;
  p.level_begin[1] = 1;
  p.partial[0] = levels[0][0].partial;
  for (int i = 1; i + 1 < n; i++) {
    for (int j = 0; j < (int)levels[i].size(); j++) {
      if (next >= PM_MAX_SLOTS) return fail(PM_ERR_FORMAT, ".g: more than %d slots", PM_MAX_SLOTS);
      const SlotSrc& s = levels[i][j];
      flat_of[i][j] = next;
      p.slot_labels[next] = s.labels;
      p.partial[next] = s.partial;
      const int parent = (i > 1) ? flat_of[i - 1][s.op & 0x0F] : 0;
      p.set_ops[next] = (uint8_t)(((s.op & 0x30) << 1) + parent);
      next++;
    }
    p.level_begin[i + 1] = next;
  }
  for (int i = n; i <= PM_MAX_PAT; i++) p.level_begin[i] = next;
  p.nslots = next;
  *out = p;
  return PM_OK;
}

// =====================================================================
// CSR construction shared by the generators.
// =====================================================================

void csr_from_keys(int64_t n, const std::vector<uint64_t>& keys, uint64_t** rowptr_out,
                   int32_t** colidx_out, int64_t* n_adj_out, int32_t* max_degree_out) {
  const int64_t m = (int64_t)keys.size();
  std::vector<std::atomic<uint32_t>> deg(n);
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < n; v++) deg[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; e++) {
    deg[keys[e] >> 32].fetch_add(1, std::memory_order_relaxed);
    deg[keys[e] & 0xffffffffu].fetch_add(1, std::memory_order_relaxed);
  }
  uint64_t* rowptr = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  rowptr[0] = 0;
  int32_t maxd = 0;
  for (int64_t v = 0; v < n; v++) {
    uint32_t d = deg[v].load(std::memory_order_relaxed);
    rowptr[v + 1] = rowptr[v] + d;
    if ((int32_t)d > maxd) maxd = (int32_t)d;
  }
  const int64_t nadj = (int64_t)rowptr[n];
  int32_t* colidx = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(nadj, 1));
#pragma omp parallel for schedule(static)
  for (int64_t v = 0; v < n; v++) deg[v].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m; e++) {
    const uint32_t lo = (uint32_t)(keys[e] >> 32), hi = (uint32_t)(keys[e] & 0xffffffffu);
    colidx[rowptr[lo] + deg[lo].fetch_add(1, std::memory_order_relaxed)] = (int32_t)hi;
    colidx[rowptr[hi] + deg[hi].fetch_add(1, std::memory_order_relaxed)] = (int32_t)lo;
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t v = 0; v < n; v++) std::sort(colidx + rowptr[v], colidx + rowptr[v + 1]);
  *rowptr_out = rowptr;
  *colidx_out = colidx;
  *n_adj_out = nadj;
  *max_degree_out = maxd;
}

namespace {

struct KeyPos {
  uint64_t key;
  uint64_t pos;
};

// Draws candidate edges batch by batch (batch b from its own RNG stream, so
// the result does not depend on the thread count), keeps the first
// occurrence of each new edge in generation order, and stops at exactly m
// unique edges.  gen(rng, out, count) appends count keys, UINT64_MAX for a
// rejected draw (self-loop or out-of-range id).
template <class Gen>
std::vector<uint64_t> sample_unique(int64_t m, uint64_t seed, Gen gen) {
  const int64_t kBatch = 1 << 16;
  std::vector<uint64_t> have;  // sorted unique keys
  uint64_t next_batch = 0;
  for (int round = 0; (int64_t)have.size() < m; round++) {
    if (round > 64) break;  // graph too dense for the requested edge count
    const int64_t need = m - (int64_t)have.size();
    const int64_t want = need + need / 4 + 1024;
    const int64_t nb = (want + kBatch - 1) / kBatch;
    std::vector<uint64_t> cand((size_t)(nb * kBatch));
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < nb; b++) {
      Rng rng(seed, next_batch + (uint64_t)b + 1);
      gen(rng, cand.data() + b * kBatch, kBatch);
    }
    next_batch += (uint64_t)nb;
    std::vector<KeyPos> kp;
    kp.reserve(cand.size());
    for (size_t i = 0; i < cand.size(); i++)
      if (cand[i] != UINT64_MAX) kp.push_back({cand[i], (uint64_t)i});
    std::vector<uint64_t>().swap(cand);
    __gnu_parallel::sort(kp.begin(), kp.end(), [](const KeyPos& a, const KeyPos& b) {
      return a.key != b.key ? a.key < b.key : a.pos < b.pos;
    });
    // first occurrence per key, not already present
    std::vector<KeyPos> fresh;
    size_t h = 0;
    for (size_t i = 0; i < kp.size(); i++) {
      if (i > 0 && kp[i].key == kp[i - 1].key) continue;
      while (h < have.size() && have[h] < kp[i].key) h++;
      if (h < have.size() && have[h] == kp[i].key) continue;
      fresh.push_back(kp[i]);
    }
    std::vector<KeyPos>().swap(kp);
    __gnu_parallel::sort(fresh.begin(), fresh.end(),
                         [](const KeyPos& a, const KeyPos& b) { return a.pos < b.pos; });
    if ((int64_t)fresh.size() > need) fresh.resize((size_t)need);
    std::vector<uint64_t> add(fresh.size());
    for (size_t i = 0; i < fresh.size(); i++) add[i] = fresh[i].key;
    __gnu_parallel::sort(add.begin(), add.end());
    std::vector<uint64_t> merged(have.size() + add.size());
    std::merge(have.begin(), have.end(), add.begin(), add.end(), merged.begin());
    have.swap(merged);
  }
  return have;
}

inline uint64_t edge_key(uint32_t u, uint32_t v) {
  return u < v ? ((uint64_t)u << 32 | v) : ((uint64_t)v << 32 | u);
}

}  // namespace
}  // namespace pm

using namespace pm;

// =====================================================================
// C-ABI: errors, plans, files, generators
// =====================================================================

extern "C" const char* pm_last_error(void) { return g_last_error.c_str(); }

extern "C" pm_status pm_stats_json(const pm_stats* st, const uint64_t* counts, int n_counts, char* buf,
                                   size_t cap, size_t* len_out) {
  if (!st || (n_counts > 0 && !counts) || n_counts < 0 || (cap > 0 && !buf))
    return fail(PM_ERR_INVALID, "pm_stats_json: bad arguments");
  std::string j = "{\"counts\": [";
  uint64_t total = 0;
  for (int i = 0; i < n_counts; i++) {
    j += (i ? ", " : "") + std::to_string((unsigned long long)counts[i]);
    total += counts[i];
  }
  const double s = st->kernel_ms / 1000.0;
  char tmp[768];
  snprintf(tmp, sizeof(tmp),
           "], \"kernel_ms\": %.3f, \"roots_ms\": %.3f, \"matches_per_s\": %.6g, \"n_roots\": %llu, "
           "\"set_ops\": %llu, \"alg_bytes\": %llu, \"alg_gbs\": %.6g, \"splits\": %llu, "
           "\"page_hits\": %llu, \"page_misses\": %llu, \"pages_loaded\": %llu, \"h2d_page_bytes\": %llu, "
           "\"zero_copy_bytes\": %llu, \"evictions\": %llu, \"warp_idle_share\": %.4f, "
           "\"grid_blocks\": %d, \"block_threads\": %d, \"arena_bytes\": %llu, \"borrowed_arenas\": %llu, "
           "\"arena_pool\": %llu, \"device_status\": %u}",
           st->kernel_ms, st->roots_ms, s > 0 ? (double)total / s : 0.0, (unsigned long long)st->n_roots,
           (unsigned long long)st->set_ops, (unsigned long long)st->alg_bytes,
           s > 0 ? (double)st->alg_bytes / s / 1e9 : 0.0, (unsigned long long)st->splits,
           (unsigned long long)st->page_hits, (unsigned long long)st->page_misses,
           (unsigned long long)st->pages_loaded, (unsigned long long)st->h2d_page_bytes,
           (unsigned long long)st->zero_copy_bytes, (unsigned long long)st->evictions,
           st->warp_ns ? (double)st->idle_ns / (double)st->warp_ns : 0.0, st->grid_blocks, st->block_threads,
           (unsigned long long)st->arena_bytes, (unsigned long long)st->borrowed_arenas,
           (unsigned long long)st->arena_pool, st->device_status);
  j += tmp;
  if (len_out) *len_out = j.size() + 1;
  if (j.size() + 1 > cap) return fail(PM_ERR_INVALID, "pm_stats_json: needs %zu bytes", j.size() + 1);
  memcpy(buf, j.c_str(), j.size() + 1);
  return PM_OK;
}

extern "C" const char* pm_strerror(pm_status s) {
  switch (s) {
    case PM_OK: return "ok";
    case PM_ERR_IO: return "i/o error";
    case PM_ERR_FORMAT: return "format error";
    case PM_ERR_OOM: return "out of memory";
    case PM_ERR_CUDA: return "CUDA error";
    case PM_ERR_TIMEOUT: return "device wait timed out";
    case PM_ERR_INVALID: return "invalid argument";
    case PM_ERR_INTERNAL: return "internal error";
    case PM_ERR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

struct pm_plan {
  Plan p;
};

extern "C" pm_status pm_plan_compile_text(const char* text, int labeled, pm_plan** out) {
  if (!text || !out) return fail(PM_ERR_INVALID, "pm_plan_compile_text: null argument");
  std::unique_ptr<pm_plan> h(new pm_plan);
  pm_status st = compile_plan(text, labeled != 0, &h->p);
  if (st != PM_OK) return st;
  *out = h.release();
  return PM_OK;
}

extern "C" pm_status pm_plan_compile(const char* path, int labeled, pm_plan** out) {
  if (!path || !out) return fail(PM_ERR_INVALID, "pm_plan_compile: null argument");
  std::ifstream f(path);
  if (!f.good()) return fail(PM_ERR_IO, "cannot open pattern file %s", path);
  std::stringstream ss;
  ss << f.rdbuf();
  return pm_plan_compile_text(ss.str().c_str(), labeled, out);
}

extern "C" pm_status pm_plan_describe(const pm_plan* h, pm_plan_desc* d) {
  if (!h || !d) return fail(PM_ERR_INVALID, "pm_plan_describe: null argument");
  memset(d, 0, sizeof(*d));
  const Plan& p = h->p;
  d->nnodes = p.nnodes;
  d->nslots = p.nslots;
  d->multiplicity = p.multiplicity;
  d->labeled = p.labeled;
  memcpy(d->level_begin, p.level_begin, sizeof(d->level_begin));
  memcpy(d->degree, p.degree, sizeof(d->degree));
  memcpy(d->vertex_label, p.vertex_label, sizeof(d->vertex_label));
  memcpy(d->slot_labels, p.slot_labels, sizeof(d->slot_labels));
  memcpy(d->partial, p.partial, sizeof(d->partial));
  memcpy(d->set_ops, p.set_ops, sizeof(d->set_ops));
  return PM_OK;
}

extern "C" void pm_plan_free(pm_plan* p) { delete p; }

namespace pm {
const Plan* plan_of(const pm_plan* h) { return h ? &h->p : nullptr; }
}  // namespace pm

extern "C" void pm_host_free(void* p) { free(p); }

// ---------------------------------------------------------------- files

static pm_status read_exact(const std::string& path, void* dst, size_t bytes) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return fail(PM_ERR_IO, "cannot open %s", path.c_str());
  size_t got = bytes ? fread(dst, 1, bytes, f) : 0;
  fclose(f);
  if (got != bytes) return fail(PM_ERR_FORMAT, "%s: expected %zu bytes, read %zu", path.c_str(), bytes, got);
  return PM_OK;
}

extern "C" pm_status pm_graph_read(const char* prefix, int labeled, int64_t* n_out, int64_t* nadj_out,
                                   int32_t* maxdeg_out, uint64_t** rowptr_out, int32_t** colidx_out,
                                   uint32_t** labels_out) {
  if (!prefix || !n_out || !nadj_out || !rowptr_out || !colidx_out)
    return fail(PM_ERR_INVALID, "pm_graph_read: null argument");
  const std::string pre(prefix);
  // .meta.txt: n_vertices n_adj vid_size max_degree (src/graph.h:229-238)
  std::ifstream meta(pre + ".meta.txt");
  if (!meta.good()) return fail(PM_ERR_IO, "cannot open %s.meta.txt", prefix);
  long long n = -1, nadj = -1, vid = -1, maxd = -1;
  if (!(meta >> n >> nadj >> vid >> maxd)) return fail(PM_ERR_FORMAT, "%s.meta.txt: need 4 integers", prefix);
  if (vid != 4) return fail(PM_ERR_FORMAT, "%s.meta.txt: vid_size %lld, only 4 is supported", prefix, vid);
  if (n < 0 || n > INT32_MAX || nadj < 0) return fail(PM_ERR_FORMAT, "%s.meta.txt: bad sizes", prefix);
  uint64_t* rowptr = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n + 1));
  int32_t* colidx = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<long long>(nadj, 1));
  uint32_t* labels = labeled ? (uint32_t*)malloc(sizeof(uint32_t) * (size_t)std::max<long long>(n, 1)) : nullptr;
  if (!rowptr || !colidx || (labeled && !labels)) {
    free(rowptr); free(colidx); free(labels);
    return fail(PM_ERR_OOM, "pm_graph_read: host allocation failed");
  }
  auto bail = [&](pm_status s) { free(rowptr); free(colidx); free(labels); return s; };
  pm_status st;
  if ((st = read_exact(pre + ".vertex.bin", rowptr, sizeof(uint64_t) * (n + 1))) != PM_OK) return bail(st);
  if ((st = read_exact(pre + ".edge.bin", colidx, sizeof(int32_t) * nadj)) != PM_OK) return bail(st);
  if (labeled && (st = read_exact(pre + ".label.bin", labels, sizeof(uint32_t) * n)) != PM_OK) return bail(st);
  if (rowptr[0] != 0 || rowptr[n] != (uint64_t)nadj)
    return bail(fail(PM_ERR_FORMAT, "%s.vertex.bin: offsets do not span [0,%lld]", prefix, nadj));
  int32_t real_max = 0;
  int64_t bad = -1;
#pragma omp parallel for schedule(dynamic, 4096) reduction(max : real_max)
  for (long long v = 0; v < n; v++) {
    if (rowptr[v + 1] < rowptr[v] || rowptr[v + 1] > (uint64_t)nadj) { bad = v; continue; }
    const int32_t d = (int32_t)(rowptr[v + 1] - rowptr[v]);
    if (d > real_max) real_max = d;
    for (uint64_t e = rowptr[v]; e < rowptr[v + 1]; e++) {
      if (colidx[e] < 0 || colidx[e] >= n || (e > rowptr[v] && colidx[e] < colidx[e - 1])) { bad = v; break; }
    }
  }
  if (bad >= 0) return bail(fail(PM_ERR_FORMAT, "%s: adjacency of vertex %lld is unsorted or out of range", prefix, (long long)bad));
  if (labeled)
    for (long long v = 0; v < n; v++)
      if (labels[v] >= 32) return bail(fail(PM_ERR_FORMAT, "%s.label.bin: label %u >= 32", prefix, labels[v]));
  *n_out = n;
  *nadj_out = nadj;
  if (maxdeg_out) *maxdeg_out = real_max;
  *rowptr_out = rowptr;
  *colidx_out = colidx;
  if (labels_out) *labels_out = labels; else free(labels);
  return PM_OK;
}

static pm_status write_all(const std::string& path, const void* src, size_t bytes) {
  FILE* f = fopen(path.c_str(), "wb");
  if (!f) return fail(PM_ERR_IO, "cannot create %s", path.c_str());
  size_t put = bytes ? fwrite(src, 1, bytes, f) : 0;
  int rc = fclose(f);
  if (put != bytes || rc != 0) return fail(PM_ERR_IO, "short write to %s", path.c_str());
  return PM_OK;
}

extern "C" pm_status pm_graph_write(const char* prefix, int64_t n, int64_t nadj, const uint64_t* rowptr,
                                    const int32_t* colidx, const uint32_t* labels) {
  if (!prefix || !rowptr || (nadj > 0 && !colidx)) return fail(PM_ERR_INVALID, "pm_graph_write: null argument");
  const std::string pre(prefix);
  int64_t maxd = 0;
  for (int64_t v = 0; v < n; v++) maxd = std::max<int64_t>(maxd, (int64_t)(rowptr[v + 1] - rowptr[v]));
  // same 4-line layout as graph_converter/compactify.cpp:47-48
  FILE* f = fopen((pre + ".meta.txt").c_str(), "w");
  if (!f) return fail(PM_ERR_IO, "cannot create %s.meta.txt", prefix);
  fprintf(f, "%lld\n%lld\n%d\n%lld\n", (long long)n, (long long)nadj, 4, (long long)maxd);
  fclose(f);
  pm_status st;
  if ((st = write_all(pre + ".vertex.bin", rowptr, sizeof(uint64_t) * (n + 1))) != PM_OK) return st;
  if ((st = write_all(pre + ".edge.bin", colidx, sizeof(int32_t) * nadj)) != PM_OK) return st;
  if (labels && (st = write_all(pre + ".label.bin", labels, sizeof(uint32_t) * n)) != PM_OK) return st;
  return PM_OK;
}

// ------------------------------------------------- degree order and halving

// Checks a CSR's shape: monotone offsets ending at n_adj, ids in range.
static pm_status check_csr(const char* who, int64_t n, int64_t nadj, const uint64_t* rowptr,
                           const int32_t* colidx) {
  if (n < 0 || n > INT32_MAX || nadj < 0 || !rowptr || (nadj > 0 && !colidx))
    return fail(PM_ERR_INVALID, "%s: bad arguments", who);
  if (rowptr[0] != 0 || rowptr[n] != (uint64_t)nadj) return fail(PM_ERR_FORMAT, "%s: offsets do not span the lists", who);
  for (int64_t v = 0; v < n; v++)
    if (rowptr[v + 1] < rowptr[v]) return fail(PM_ERR_FORMAT, "%s: offsets of vertex %lld decrease", who, (long long)v);
  for (int64_t i = 0; i < nadj; i++)
    if (colidx[i] < 0 || colidx[i] >= n) return fail(PM_ERR_FORMAT, "%s: vertex id %d out of range", who, colidx[i]);
  return PM_OK;
}

// Restates graph_converter/relabel.cpp:26-63: vertices sorted by (degree,
// id) descending take the new ids 0, 1, ...; every list is rewritten in new
// ids and sorted.  relabel.cpp copies no label file; here the labels move
// with their vertices, so a labeled graph stays the same graph.
extern "C" pm_status pm_reorder_by_degree(int64_t n, int64_t nadj, const uint64_t* rowptr, const int32_t* colidx,
                                          const uint32_t* labels, uint64_t* rowptr_out, int32_t* colidx_out,
                                          uint32_t* labels_out, int32_t* new_id_out) {
  pm_status st = check_csr("pm_reorder_by_degree", n, nadj, rowptr, colidx);
  if (st != PM_OK) return st;
  if (!rowptr_out || (nadj > 0 && !colidx_out) || (labels && !labels_out))
    return fail(PM_ERR_INVALID, "pm_reorder_by_degree: missing output");
  std::vector<int32_t> order((size_t)n), nid((size_t)n);
  for (int64_t v = 0; v < n; v++) order[v] = (int32_t)v;
  auto deg = [&](int32_t v) { return rowptr[v + 1] - rowptr[v]; };
  std::sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
    const uint64_t dx = deg(x), dy = deg(y);
    return dx != dy ? dx > dy : x > y;
  });
  for (int64_t i = 0; i < n; i++) nid[order[i]] = (int32_t)i;
  rowptr_out[0] = 0;
  for (int64_t i = 0; i < n; i++) rowptr_out[i + 1] = rowptr_out[i] + deg(order[i]);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < n; i++) {
    const int32_t old = order[i];
    int32_t* out = colidx_out + rowptr_out[i];
    const uint64_t b = rowptr[old], d = deg(old);
    for (uint64_t k = 0; k < d; k++) out[k] = nid[colidx[b + k]];
    std::sort(out, out + d);
  }
  if (labels)
    for (int64_t i = 0; i < n; i++) labels_out[i] = labels[order[i]];
  if (new_id_out) std::copy(nid.begin(), nid.end(), new_id_out);
  return PM_OK;
}

// Restates graph_converter/halve.cpp:19-30: vertex u keeps neighbour w when
// w has the higher degree, or the same degree and the higher id -- each
// undirected edge once, towards its heavier end.  colidx_out must hold nadj
// entries (exactly nadj/2 are used for a symmetric graph without loops).
extern "C" pm_status pm_halve(int64_t n, int64_t nadj, const uint64_t* rowptr, const int32_t* colidx,
                              uint64_t* rowptr_out, int32_t* colidx_out, int64_t* nadj_out,
                              int32_t* max_degree_out) {
  pm_status st = check_csr("pm_halve", n, nadj, rowptr, colidx);
  if (st != PM_OK) return st;
  if (!rowptr_out || (nadj > 0 && !colidx_out) || !nadj_out || !max_degree_out)
    return fail(PM_ERR_INVALID, "pm_halve: missing output");
  rowptr_out[0] = 0;
  int64_t maxd = 0;
  for (int64_t u = 0; u < n; u++) {
    const uint64_t b = rowptr[u], e = rowptr[u + 1], du = e - b;
    uint64_t o = rowptr_out[u];
    for (uint64_t i = b; i < e; i++) {
      const int32_t w = colidx[i];
      const uint64_t dw = rowptr[w + 1] - rowptr[w];
      if (dw > du || (dw == du && w > u)) colidx_out[o++] = w;
    }
    rowptr_out[u + 1] = o;
    maxd = std::max<int64_t>(maxd, (int64_t)(o - rowptr_out[u]));
  }
  *nadj_out = (int64_t)rowptr_out[n];
  *max_degree_out = (int32_t)maxd;
  return PM_OK;
}

// ---------------------------------------------------------------- generators

extern "C" pm_status pm_gen_chung_lu(int64_t n, int64_t m, double gamma, double i0, double max_w,
                                     uint64_t seed, uint64_t** rowptr, int32_t** colidx,
                                     int64_t* n_adj, int32_t* max_degree) {
  if (n < 2 || n > INT32_MAX || m < 0 || gamma <= 1.0 || !rowptr || !colidx || !n_adj || !max_degree)
    return fail(PM_ERR_INVALID, "pm_gen_chung_lu: bad arguments");
  if ((double)m > 0.5 * (double)n * (double)(n - 1)) return fail(PM_ERR_INVALID, "pm_gen_chung_lu: too many edges");
  // expected degrees w_i ~ (i + i0)^(-1/(gamma-1)), sum 2m, capped
  std::vector<double> w((size_t)n);
  double sum = 0;
  for (int64_t i = 0; i < n; i++) { w[i] = std::pow((double)i + i0, -1.0 / (gamma - 1.0)); sum += w[i]; }
  for (int64_t i = 0; i < n; i++) { w[i] *= 2.0 * (double)m / sum; if (max_w > 0 && w[i] > max_w) w[i] = max_w; }
  // Vose alias table for O(1) endpoint draws proportional to w
  double tot = 0;
  for (double x : w) tot += x;
  std::vector<double> prob((size_t)n);
  std::vector<uint32_t> alias((size_t)n);
  std::vector<int64_t> small, large;
  for (int64_t i = 0; i < n; i++) {
    prob[i] = w[i] * (double)n / tot;
    (prob[i] < 1.0 ? small : large).push_back(i);
  }
  while (!small.empty() && !large.empty()) {
    int64_t s = small.back(); small.pop_back();
    int64_t l = large.back();
    alias[s] = (uint32_t)l;
    prob[l] = prob[l] + prob[s] - 1.0;
    if (prob[l] < 1.0) { large.pop_back(); small.push_back(l); }
  }
  for (int64_t i : large) prob[i] = 1.0;
  for (int64_t i : small) prob[i] = 1.0;
  auto draw = [&](Rng& r) -> uint32_t {
    uint32_t i = r.below((uint32_t)n);
    return r.uniform() < prob[i] ? i : alias[i];
  };
  std::vector<uint64_t> keys = sample_unique(m, seed, [&](Rng& r, uint64_t* out, int64_t cnt) {
    for (int64_t k = 0; k < cnt; k++) {
      uint32_t a = draw(r), b = draw(r);
      out[k] = (a == b) ? UINT64_MAX : edge_key(a, b);
    }
  });
  if ((int64_t)keys.size() != m) return fail(PM_ERR_INVALID, "pm_gen_chung_lu: could not reach %lld edges", (long long)m);
  csr_from_keys(n, keys, rowptr, colidx, n_adj, max_degree);
  return PM_OK;
}

extern "C" pm_status pm_gen_rmat(int64_t n, int64_t m, double a, double b, double c, uint64_t seed,
                                 uint64_t** rowptr, int32_t** colidx, int64_t* n_adj, int32_t* max_degree) {
  if (n < 2 || n > INT32_MAX || m < 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 || !rowptr || !colidx)
    return fail(PM_ERR_INVALID, "pm_gen_rmat: bad arguments");
  int scale = 0;
  while ((1ll << scale) < n) scale++;
  // quadrant thresholds on 16-bit draws
  const uint32_t ta = (uint32_t)std::lround(a * 65536.0);
  const uint32_t tb = (uint32_t)std::lround((a + b) * 65536.0);
  const uint32_t tc = (uint32_t)std::lround((a + b + c) * 65536.0);
  std::vector<uint64_t> keys = sample_unique(m, seed, [&](Rng& r, uint64_t* out, int64_t cnt) {
    for (int64_t k = 0; k < cnt; k++) {
      uint32_t u, v;
      out[k] = rmat_draw(r, scale, (uint64_t)n, ta, tb, tc, &u, &v) ? edge_key(u, v) : UINT64_MAX;
    }
  });
  if ((int64_t)keys.size() != m) return fail(PM_ERR_INVALID, "pm_gen_rmat: could not reach %lld edges", (long long)m);
  csr_from_keys(n, keys, rowptr, colidx, n_adj, max_degree);
  return PM_OK;
}

extern "C" pm_status pm_gen_labels(int64_t n, int n_labels, uint64_t seed, uint32_t** labels) {
  if (n < 0 || n_labels < 1 || n_labels > 32 || !labels) return fail(PM_ERR_INVALID, "pm_gen_labels: bad arguments");
  uint32_t* lab = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)std::max<int64_t>(n, 1));
  if (!lab) return fail(PM_ERR_OOM, "pm_gen_labels: allocation failed");
  const int64_t kBlock = 1 << 16;
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < (n + kBlock - 1) / kBlock; b++) {
    Rng r(seed, (uint64_t)b + 1);
    const int64_t e = std::min(n, (b + 1) * kBlock);
    for (int64_t v = b * kBlock; v < e; v++) lab[v] = r.below((uint32_t)n_labels);
  }
  *labels = lab;
  return PM_OK;
}

// ---------------------------------------------------------------- converter

// SNAP edge list -> the CSR files (graph_converter/convert.sh:32-65 as one
// step): '#' and empty lines skipped, the first two integers of a line are an
// edge; ids are compacted in first-seen order (snapToBin.cpp:23-32), every
// edge is stored in both directions, each list sorted and deduplicated
// (compactify.cpp:15-21).  Self-loops are dropped unless keep_self_loops (the
// reference keeps them; the matcher assumes none).  n_labels > 0 writes
// labels std::rand() % n_labels after std::srand(0), vertex by vertex, which
// is labelize.cpp:45-49's sequence with n_labels = 10.
extern "C" pm_status pm_convert_snap(const char* snap_path, const char* out_prefix, int n_labels,
                                     int keep_self_loops, int64_t* n_out, int64_t* nadj_out) {
  if (!snap_path || !out_prefix || n_labels < 0 || n_labels > 32)
    return fail(PM_ERR_INVALID, "pm_convert_snap: bad arguments");
  std::ifstream in(snap_path);
  if (!in.good()) return fail(PM_ERR_IO, "cannot open %s", snap_path);
  std::vector<int64_t> id_map;
  int64_t next_id = 0;
  auto map_id = [&](int64_t raw) -> int64_t {
    if (raw < 0) return -1;
    if ((int64_t)id_map.size() <= raw) id_map.resize((size_t)raw + 2048, -1);
    if (id_map[raw] < 0) id_map[raw] = next_id++;
    return id_map[raw];
  };
  std::vector<uint64_t> keys;
  std::vector<uint32_t> loops;
  std::string line;
  int64_t lineno = 0;
  while (std::getline(in, line)) {
    lineno++;
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ls(line);
    long long a = -1, b = -1;
    if (!(ls >> a >> b)) return fail(PM_ERR_FORMAT, "%s line %lld: expected two vertex ids", snap_path, (long long)lineno);
    const int64_t u = map_id(a), v = map_id(b);
    if (u < 0 || v < 0) return fail(PM_ERR_FORMAT, "%s line %lld: negative vertex id", snap_path, (long long)lineno);
    if (u > INT32_MAX - 1 || v > INT32_MAX - 1) return fail(PM_ERR_FORMAT, "%s: more than 2^31 vertices", snap_path);
    if (u == v) {
      if (keep_self_loops) loops.push_back((uint32_t)u);
      continue;
    }
    keys.push_back(edge_key((uint32_t)u, (uint32_t)v));
  }
  const int64_t n = next_id;
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  uint64_t* rowptr = nullptr;
  int32_t* colidx = nullptr;
  int64_t nadj = 0;
  int32_t maxd = 0;
  csr_from_keys(n, keys, &rowptr, &colidx, &nadj, &maxd);
  if (!loops.empty()) {
    // add u to its own list once, keeping lists sorted
    std::sort(loops.begin(), loops.end());
    loops.erase(std::unique(loops.begin(), loops.end()), loops.end());
    uint64_t* rp2 = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
    int32_t* ci2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nadj + (int64_t)loops.size() + 1));
    size_t li = 0;
    rp2[0] = 0;
    for (int64_t v = 0; v < n; v++) {
      const bool self = li < loops.size() && loops[li] == (uint32_t)v;
      int64_t o = (int64_t)rp2[v];
      bool placed = !self;
      for (uint64_t e = rowptr[v]; e < rowptr[v + 1]; e++) {
        if (!placed && colidx[e] > v) { ci2[o++] = (int32_t)v; placed = true; }
        ci2[o++] = colidx[e];
      }
      if (!placed) ci2[o++] = (int32_t)v;
      if (self) li++;
      rp2[v + 1] = (uint64_t)o;
    }
    free(rowptr);
    free(colidx);
    rowptr = rp2;
    colidx = ci2;
    nadj = (int64_t)rp2[n];
  }
  std::vector<uint32_t> labels;
  if (n_labels > 0) {
    labels.resize((size_t)std::max<int64_t>(n, 1));
    std::srand(0);
    for (int64_t v = 0; v < n; v++) labels[v] = (uint32_t)(std::rand() % n_labels);
  }
  pm_status st = pm_graph_write(out_prefix, n, nadj, rowptr, colidx, n_labels > 0 ? labels.data() : nullptr);
  free(rowptr);
  free(colidx);
  if (st != PM_OK) return st;
  if (n_out) *n_out = n;
  if (nadj_out) *nadj_out = nadj;
  return PM_OK;
}
