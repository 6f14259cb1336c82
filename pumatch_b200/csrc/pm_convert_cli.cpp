// pm_convert_cli.cpp -- the reference's converter steps:
//   convert <snap.txt> [--labels=N] [--keep-self-loops] [--out=prefix]
//       writes <prefix>.meta.txt/.vertex.bin/.edge.bin/.label.bin, the files
//       graph_converter/convert.sh produces for the `test` command;
//   convert --order=degree <graph-prefix>
//       writes <graph-prefix>.ord.* with vertices renumbered by degree
//       (graph_converter/relabel.cpp; labels move with their vertices);
//   convert --halve <graph-prefix>
//       writes <graph-prefix>.half.* with each edge once, towards its
//       heavier end (graph_converter/halve.cpp).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <unistd.h>

#include "pumatch.h"

static int die(const char* what, pm_status s) {
  fprintf(stderr, "convert: %s: %s (%s)\n", what, pm_strerror(s), pm_last_error());
  return 1;
}

static int transform(const char* prefix, bool halve) {
  const std::string pre(prefix);
  const bool labeled = access((pre + ".label.bin").c_str(), R_OK) == 0;
  int64_t n = 0, nadj = 0;
  int32_t maxd = 0;
  uint64_t* rowptr = nullptr;
  int32_t* colidx = nullptr;
  uint32_t* labels = nullptr;
  pm_status s = pm_graph_read(prefix, labeled ? 1 : 0, &n, &nadj, &maxd, &rowptr, &colidx, &labels);
  if (s != PM_OK) return die("read", s);
  std::vector<uint64_t> rp((size_t)n + 1);
  std::vector<int32_t> ci((size_t)(nadj > 0 ? nadj : 1));
  std::vector<uint32_t> lb(labeled ? (size_t)(n > 0 ? n : 1) : 0);
  int rc = 0;
  if (halve) {
    int64_t hadj = 0;
    int32_t hmax = 0;
    s = pm_halve(n, nadj, rowptr, colidx, rp.data(), ci.data(), &hadj, &hmax);
    if (s != PM_OK) rc = die("halve", s);
    else if ((s = pm_graph_write((pre + ".half").c_str(), n, hadj, rp.data(), ci.data(), nullptr)) != PM_OK)
      rc = die("write", s);
    else printf("%lld vertices, %lld half-graph entries, max half degree %d\n", (long long)n, (long long)hadj, hmax);
  } else {
    s = pm_reorder_by_degree(n, nadj, rowptr, colidx, labels, rp.data(), ci.data(), labeled ? lb.data() : nullptr,
                             nullptr);
    if (s != PM_OK) rc = die("reorder", s);
    else if ((s = pm_graph_write((pre + ".ord").c_str(), n, nadj, rp.data(), ci.data(),
                                 labeled ? lb.data() : nullptr)) != PM_OK)
      rc = die("write", s);
    else printf("%lld vertices renumbered by degree\n", (long long)n);
  }
  pm_host_free(rowptr);
  pm_host_free(colidx);
  pm_host_free(labels);
  return rc;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: convert <snap.txt> [--labels=N (default 10, 0 = none)] [--keep-self-loops] [--out=prefix]\n"
                    "       convert --order=degree <graph-prefix>\n"
                    "       convert --halve <graph-prefix>\n");
    return 2;
  }
  if (!strcmp(argv[1], "--order=degree") || !strcmp(argv[1], "--halve")) {
    if (argc != 3) { fprintf(stderr, "convert: %s takes one graph prefix\n", argv[1]); return 2; }
    return transform(argv[2], !strcmp(argv[1], "--halve"));
  }
  int labels = 10, loops = 0;
  const char* out = argv[1];
  for (int i = 2; i < argc; i++) {
    if (!strncmp(argv[i], "--labels=", 9)) labels = atoi(argv[i] + 9);
    else if (!strcmp(argv[i], "--keep-self-loops")) loops = 1;
    else if (!strncmp(argv[i], "--out=", 6)) out = argv[i] + 6;
    else { fprintf(stderr, "convert: unknown option %s\n", argv[i]); return 2; }
  }
  int64_t n = 0, nadj = 0;
  pm_status s = pm_convert_snap(argv[1], out, labels, loops, &n, &nadj);
  if (s != PM_OK) return die("convert", s);
  printf("%lld vertices, %lld adjacency entries\n", (long long)n, (long long)nadj);
  return 0;
}
