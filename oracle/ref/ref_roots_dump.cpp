/* Prints the reference's root-job list for <graph-prefix> <pattern.g>:
 * first line the count, then one "r c" pair per line.  Compiled against the
 * reference's own src/graph.h, src/pattern.h and src/job_queue.h (untouched);
 * used only to generate golden root fixtures under tests/golden/. */
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <unistd.h>
#include "graph.h"
#include "pattern.h"
#include "job_queue.h"

int main(int argc, char** argv) {
  if (argc != 3) { fprintf(stderr, "usage: ref_roots_dump <prefix> <pattern.g>\n"); return 2; }
  GraphPreprocessor g(argv[1]);
  PatternPreprocessor p(argv[2]);
  /* JobQueuePreprocessor prints "vr.size(): N" on stdout; keep it off ours */
  fflush(stdout);
  FILE* keep = fdopen(dup(1), "w");
  freopen("/dev/null", "w", stdout);
  JobQueuePreprocessor q(g.g, p);
  fflush(stdout);
  fprintf(keep, "%d\n", (int)q.q.length);
  for (int i = 0; i < q.q.length; i++) fprintf(keep, "%d %d\n", q.q.q[i].nodes[0], q.q.q[i].nodes[1]);
  fclose(keep);
  return 0;
}
