/* Prints the reference's compiled plan for one .g file as one JSON object.
 * Compiled against the reference's own src/pattern.h (untouched); used only
 * to generate the golden plan fixtures under tests/golden/. */
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include "pattern.h"

int main(int argc, char** argv) {
  if (argc != 2) { fprintf(stderr, "usage: ref_plan_dump <pattern.g>\n"); return 2; }
  PatternPreprocessor p(argv[1]);
  const int n = p.pat.nnodes;
  const int nslots = p.pat.rowptr[n - 1];
  printf("{\"labeled\": %d, \"nnodes\": %d, \"multiplicity\": %d, \"nslots\": %d",
         (int)LABELED, n, p.PatternMultiplicity, nslots);
  printf(", \"level_begin\": [");
  for (int i = 0; i < n; i++) printf("%s%d", i ? ", " : "", p.pat.rowptr[i]);
  printf("], \"degree\": [");
  for (int i = 0; i < n; i++) printf("%s%d", i ? ", " : "", p.pat.degree[i]);
  printf("], \"vertex_label\": [");
  for (int i = 0; i < n; i++) printf("%s%d", i ? ", " : "", p.vertex_labels[i]);
  /* slot 0 is the root slot: only its partial order is defined */
  printf("], \"partial\": [");
  for (int s = 0; s < nslots; s++) printf("%s%u", s ? ", " : "", p.pat.partial[s]);
  printf("], \"slot_labels\": [0");
  for (int s = 1; s < nslots; s++) printf(", %u", p.pat.slot_labels[s]);
  printf("], \"set_ops\": [0");
  for (int s = 1; s < nslots; s++) printf(", %u", (unsigned)(unsigned char)p.pat.set_ops[s]);
  printf("]}\n");
  return 0;
}
