// pm_cli.cpp -- the drop-in `test` command.
//
//   test <graph-prefix> <pattern.g> [--labeled=0|1] [--truncate=N] [--device=D]
//        [--paged] [--frame-mb=M] [--static-mb=S] [--page-kb=K] [--batch=<list file>]
//        [--warps=W] [--chunk=C] [--split=S] [--variant=V] [--tuned=<autotuner json>]
//        [--json=<path>] [--parts=K] [--parts-device=D]
//
// Same positional arguments and output as the reference's driver
// (test.cu:15-21, 200-209): the last stdout line is "<kernel ms> <count>" and
// "<graph>\t<pattern>\t<ms>\t<count>" is appended to ./result.txt.
// Diagnostics go to stderr.  Defaults follow the reference as shipped:
// labeled matching (src/config.h:14); exact candidate sets unless
// --truncate=4096 asks for the reference's GRAPH_DEGREE cap.
// With --batch, <pattern.g> is ignored and each line of the list file names a
// pattern; all run in one launch and one "<ms> <count>" line is printed per
// pattern in list order (ms is the shared launch time).
// --json writes the launch's statistics (pm_stats_json) to <path>.
// --tuned reads the "best" record the autotuner writes (warps_per_block,
// chunk, split_level1, high_occupancy, page_kb); explicit flags after it
// override it.  --variant picks the kernel's register cap (pm_run_opts
// high_occupancy: 1 = 64, 2 = 85, 3 = uncapped; 0 = the default).
// --parts=K pages the graph (as --paged, with its pool options) from the
// adjacency array cut into K slices of device memory, slice p in the HBM of
// GPU device+p (all on GPU D with --parts-device=D), mapped into one range:
// partitioned residency, misses copied from the owner's HBM over NVLink.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <string>
#include <vector>

#include "pumatch.h"

// Integer value of "key" in the first JSON object that follows "best" (the
// autotuner's output); false when absent or null.
static bool tuned_int(const std::string& text, const char* key, long long* out) {
  size_t at = text.find("\"best\"");
  if (at == std::string::npos) return false;
  const size_t end = text.find('}', at);
  const std::string k = std::string("\"") + key + "\"";
  size_t p = text.find(k, at);
  if (p == std::string::npos || (end != std::string::npos && p > end)) return false;
  p = text.find(':', p + k.size());
  if (p == std::string::npos) return false;
  char* e = nullptr;
  const long long v = strtoll(text.c_str() + p + 1, &e, 10);
  if (e == text.c_str() + p + 1) return false;
  *out = v;
  return true;
}

static int die(const char* what, pm_status s) {
  fprintf(stderr, "test: %s: %s (%s)\n", what, pm_strerror(s), pm_last_error());
  return 1;
}

// Places the graph at `prefix` paged from k slices of device memory (see
// --parts above); the ranges stay mapped until the caller frees them, after
// the graph.  Slice bounds: multiples of the allocation granularity and of the
// page size, equal slices but for the last (pumatch_b200/parts.py does the
// same).
static pm_status place_parts(const char* prefix, const pm_graph_opts& go, int k, int one_device,
                             std::vector<pm_parts*>& ranges, pm_graph** out) {
  int64_t n = 0, nadj = 0;
  int32_t maxd = 0;
  uint64_t* rowptr = nullptr;
  int32_t* colidx = nullptr;
  uint32_t* labels = nullptr;
  pm_status s = pm_graph_read(prefix, go.labeled, &n, &nadj, &maxd, &rowptr, &colidx, &labels);
  if (s != PM_OK) return s;
  std::vector<int32_t> grouped;
  std::vector<const int32_t*> arrays;
  if (go.labeled) {
    grouped.resize((size_t)nadj);
    s = pm_label_group_host(n, nadj, rowptr, colidx, labels, grouped.data());
    arrays = {grouped.data(), colidx};
  } else {
    arrays = {colidx};
  }
  uint64_t gran = 0;
  if (s == PM_OK) s = pm_parts_granularity(go.device, &gran);
  std::vector<uint64_t> begins;
  uint64_t total = 0;
  if (s == PM_OK) {
    const uint64_t align = gran > go.page_bytes ? gran : go.page_bytes;
    const uint64_t bytes = 4ull * (uint64_t)nadj;
    uint64_t units = (bytes + align - 1) / align;
    if (units == 0) units = 1;
    const uint64_t per = (units + (uint64_t)k - 1) / (uint64_t)k;
    for (uint64_t p = 0; p < (uint64_t)k && p * per < units; p++) begins.push_back(p * per * align);
    total = units * align;
  }
  for (size_t a = 0; a < arrays.size() && s == PM_OK; a++) {
    pm_parts* r = nullptr;
    s = pm_parts_create(go.device, (int)begins.size(), begins.data(), total, &r);
    if (s != PM_OK) break;
    ranges.push_back(r);
    for (size_t p = 0; p < begins.size() && s == PM_OK; p++)
      s = pm_parts_alloc(r, (int)p, one_device >= 0 ? one_device : go.device + (int)p);
    if (s == PM_OK) s = pm_parts_map(r);
    for (size_t p = 0; p < begins.size() && s == PM_OK; p++) {
      const uint64_t b = begins[p], e = p + 1 < begins.size() ? begins[p + 1] : total;
      const uint64_t have = 4ull * (uint64_t)nadj;
      if (b < have)
        s = pm_parts_write(r, b, (const char*)arrays[a] + b, (e < have ? e : have) - b);
    }
  }
  if (s == PM_OK)
    s = pm_graph_from_paged_source(n, nadj, rowptr, go.labeled ? labels : nullptr,
                                   (const int32_t*)pm_parts_ptr(ranges[0]),
                                   go.labeled ? (const int32_t*)pm_parts_ptr(ranges[1]) : nullptr, &go, out);
  pm_host_free(rowptr);
  pm_host_free(colidx);
  pm_host_free(labels);
  return s;
}

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: test <graph-prefix> <pattern.g> [--labeled=0|1] [--truncate=N] [--device=D]\n"
                    "            [--paged] [--frame-mb=M] [--static-mb=S] [--page-kb=K] [--batch=<list>]\n"
                    "            [--warps=W] [--chunk=C] [--split=S] [--variant=V] [--tuned=<json>] [--json=<path>]\n"
                    "            [--parts=K] [--parts-device=D]\n");
    return 2;
  }
  const char* prefix = argv[1];
  std::string pattern = argv[2];
  int labeled = 1, truncate = 0, device = 0, paged = 0;
  long long frame_mb = 4096, static_mb = 0, page_kb = 64;
  long long warps = 0, chunk = 0, split = 0, variant = 0;
  int n_parts = 0, parts_device = -1;
  std::string batch, json_path;
  for (int i = 3; i < argc; i++) {
    const char* a = argv[i];
    if (!strncmp(a, "--tuned=", 8)) {
      std::ifstream f(a + 8);
      if (!f.good()) { fprintf(stderr, "test: cannot open %s\n", a + 8); return 1; }
      const std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
      long long v;
      if (text.find("\"best\"") == std::string::npos) { fprintf(stderr, "test: %s has no \"best\" record\n", a + 8); return 1; }
      if (tuned_int(text, "warps_per_block", &v)) warps = v;
      if (tuned_int(text, "chunk", &v)) chunk = v;
      if (tuned_int(text, "split_level1", &v)) split = v;
      if (tuned_int(text, "page_kb", &v)) page_kb = v;
      if (tuned_int(text, "high_occupancy", &v)) variant = v;
    }
    else if (!strncmp(a, "--json=", 7)) json_path = a + 7;
    else if (!strncmp(a, "--warps=", 8)) warps = atoll(a + 8);
    else if (!strncmp(a, "--chunk=", 8)) chunk = atoll(a + 8);
    else if (!strncmp(a, "--split=", 8)) split = atoll(a + 8);
    else if (!strncmp(a, "--variant=", 10)) variant = atoll(a + 10);
    else if (!strncmp(a, "--labeled=", 10)) labeled = atoi(a + 10);
    else if (!strncmp(a, "--truncate=", 11)) truncate = atoi(a + 11);
    else if (!strncmp(a, "--device=", 9)) device = atoi(a + 9);
    else if (!strcmp(a, "--paged")) paged = 1;
    else if (!strncmp(a, "--frame-mb=", 11)) frame_mb = atoll(a + 11);
    else if (!strncmp(a, "--static-mb=", 12)) static_mb = atoll(a + 12);
    else if (!strncmp(a, "--page-kb=", 10)) page_kb = atoll(a + 10);
    else if (!strncmp(a, "--batch=", 8)) batch = a + 8;
    else if (!strncmp(a, "--parts=", 8)) n_parts = atoi(a + 8);
    else if (!strncmp(a, "--parts-device=", 15)) parts_device = atoi(a + 15);
    else { fprintf(stderr, "test: unknown option %s\n", a); return 2; }
  }
  std::vector<std::string> files;
  if (batch.empty()) {
    files.push_back(pattern);
  } else {
    std::ifstream f(batch);
    if (!f.good()) { fprintf(stderr, "test: cannot open %s\n", batch.c_str()); return 1; }
    std::string line;
    while (std::getline(f, line))
      if (!line.empty() && line[0] != '#') files.push_back(line);
  }

  if (n_parts < 0 || n_parts > 1024 || (parts_device >= 0 && n_parts == 0)) {
    fprintf(stderr, "test: --parts takes 1..1024 slices (and --parts-device needs it)\n");
    return 2;
  }
  pm_graph_opts go;
  pm_graph_opts_default(&go);
  go.labeled = labeled;
  go.device = device;
  if (paged || n_parts) {
    go.residency = PM_RESIDENT_PAGED;
    go.frame_pool_bytes = (uint64_t)frame_mb << 20;
    go.page_bytes = (uint32_t)(page_kb << 10);
    go.static_pool_bytes = (uint64_t)static_mb << 20;
  }
  pm_graph* g = nullptr;
  std::vector<pm_parts*> ranges;
  pm_status s = n_parts ? place_parts(prefix, go, n_parts, parts_device, ranges, &g) : pm_graph_open(prefix, &go, &g);
  if (s != PM_OK) return die("graph", s);
  pm_graph_info gi;
  pm_graph_get_info(g, &gi);
  fprintf(stderr, "graph: %lld vertices, %lld adjacency entries, max degree %d, device bytes %llu\n",
          (long long)gi.n_vertices, (long long)gi.n_adj, gi.max_degree, (unsigned long long)gi.device_bytes);

  std::vector<pm_plan*> plans;
  for (auto& f : files) {
    pm_plan* p = nullptr;
    s = pm_plan_compile(f.c_str(), labeled, &p);
    if (s != PM_OK) return die(f.c_str(), s);
    plans.push_back(p);
  }
  pm_ctx* ctx = nullptr;
  s = pm_ctx_create(device, &ctx);
  if (s != PM_OK) return die("context", s);
  pm_run_opts ro;
  pm_run_opts_default(&ro);
  ro.truncate = truncate;
  if (warps) ro.warps_per_block = (int32_t)warps;
  if (chunk) ro.chunk = (int32_t)chunk;
  if (split) ro.split_level1 = (int32_t)split;
  if (variant) ro.high_occupancy = (int32_t)variant;
  std::vector<uint64_t> counts(plans.size(), 0);
  pm_stats st;
  s = pm_match(ctx, g, plans.data(), (int)plans.size(), &ro, counts.data(), &st);
  if (s != PM_OK) return die("match", s);
  fprintf(stderr, "roots %llu, set ops %llu, algorithmic bytes %llu, root filter %.3f ms\n",
          (unsigned long long)st.n_roots, (unsigned long long)st.set_ops,
          (unsigned long long)st.alg_bytes, st.roots_ms);
  if (!json_path.empty()) {
    size_t need = 0;
    pm_stats_json(&st, counts.data(), (int)counts.size(), nullptr, 0, &need);
    std::vector<char> doc(need);
    FILE* jf = fopen(json_path.c_str(), "w");
    if (!jf || pm_stats_json(&st, counts.data(), (int)counts.size(), doc.data(), doc.size(), nullptr) != PM_OK) {
      fprintf(stderr, "test: cannot write %s\n", json_path.c_str());
      if (jf) fclose(jf);
      return 1;
    }
    fprintf(jf, "%s\n", doc.data());
    fclose(jf);
  }
  const float ms = st.kernel_ms;
  for (size_t i = 0; i < plans.size(); i++) {
    std::cout << ms << ' ' << (unsigned long long)counts[i] << std::endl;
    FILE* out = fopen("result.txt", "a");
    if (out) {
      fprintf(out, "%s\t%s\t%f\t%llu\n", prefix, files[i].c_str(), ms, (unsigned long long)counts[i]);
      fclose(out);
    } else {
      fprintf(stderr, "test: cannot append to result.txt\n");
    }
  }
  for (auto* p : plans) pm_plan_free(p);
  pm_ctx_destroy(ctx);
  pm_graph_close(g);
  for (auto* r : ranges) pm_parts_free(r);
  return 0;
}
