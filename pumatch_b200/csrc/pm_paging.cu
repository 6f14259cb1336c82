// pm_paging.cu -- placeholder for the paged (out-of-HBM) residency.
#include "pm_device.cuh"

namespace pm {
pm_status paged_place(pm_graph*, const int32_t*, const pm_graph_opts*) {
  return fail(PM_ERR_INVALID, "paged residency is not available in this build");
}
pm_status paged_maxnbrdeg(pm_graph*) { return PM_ERR_INVALID; }
void paged_release(pm_graph*) {}
}  // namespace pm
