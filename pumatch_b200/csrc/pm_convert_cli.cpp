// pm_convert_cli.cpp -- `convert <snap.txt> [--labels=N] [--keep-self-loops]`:
// writes <snap.txt>.meta.txt/.vertex.bin/.edge.bin/.label.bin, the files the
// reference's graph_converter/convert.sh produces for the `test` command.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "pumatch.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    fprintf(stderr, "usage: convert <snap.txt> [--labels=N (default 10, 0 = none)] [--keep-self-loops] [--out=prefix]\n");
    return 2;
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
  if (s != PM_OK) {
    fprintf(stderr, "convert: %s (%s)\n", pm_strerror(s), pm_last_error());
    return 1;
  }
  printf("%lld vertices, %lld adjacency entries\n", (long long)n, (long long)nadj);
  return 0;
}
