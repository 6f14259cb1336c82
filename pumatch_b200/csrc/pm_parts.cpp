// pm_parts.cpp -- one device address range over slices of an array that live
// in the HBM of several GPUs (partitioned residency).
//
// The reference keeps the part of the adjacency array that does not fit its
// device partition in host memory and pages it over PCIe (test.cu:22-43,
// src/buffer.cu:986-1060); its multi-node mode copies the whole graph to
// every rank (test_mpi.cu:317-349).  On a node whose GPUs share NVLink, the
// array can instead be cut into slices, each held once in the HBM of one GPU,
// and every GPU maps all slices into one contiguous range with the CUDA
// virtual memory calls: the paged matcher then takes its pages from that
// range (peer HBM over NVLink, or its own) exactly as it takes them from
// pinned host memory, with no change to the kernel.
//
// A slice is a cuMemCreate allocation on its owner's device, exportable as a
// POSIX file descriptor, so the processes of a one-process-per-GPU job can
// pass their slices to each other (over a Unix socket) and import them.  The
// driver entry points are fetched through cudaGetDriverEntryPoint, so the
// library does not link libcuda itself.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include <unistd.h>

#include "pm_common.h"
#include "pumatch.h"

using namespace pm;

namespace {

typedef CUresult (*PFN_reserve)(CUdeviceptr*, size_t, size_t, CUdeviceptr, unsigned long long);
typedef CUresult (*PFN_addr_free)(CUdeviceptr, size_t);
typedef CUresult (*PFN_create)(CUmemGenericAllocationHandle*, size_t, const CUmemAllocationProp*, unsigned long long);
typedef CUresult (*PFN_release)(CUmemGenericAllocationHandle);
typedef CUresult (*PFN_map)(CUdeviceptr, size_t, size_t, CUmemGenericAllocationHandle, unsigned long long);
typedef CUresult (*PFN_unmap)(CUdeviceptr, size_t);
typedef CUresult (*PFN_set_access)(CUdeviceptr, size_t, const CUmemAccessDesc*, size_t);
typedef CUresult (*PFN_export)(void*, CUmemGenericAllocationHandle, CUmemAllocationHandleType, unsigned long long);
typedef CUresult (*PFN_import)(CUmemGenericAllocationHandle*, void*, CUmemAllocationHandleType);
typedef CUresult (*PFN_granularity)(size_t*, const CUmemAllocationProp*, CUmemAllocationGranularity_flags);

struct Vmm {
  PFN_reserve reserve = nullptr;
  PFN_addr_free addr_free = nullptr;
  PFN_create create = nullptr;
  PFN_release release = nullptr;
  PFN_map map = nullptr;
  PFN_unmap unmap = nullptr;
  PFN_set_access set_access = nullptr;
  PFN_export export_fd = nullptr;
  PFN_import import_fd = nullptr;
  PFN_granularity granularity = nullptr;
  bool ok = false;
};

Vmm g_vmm;
std::once_flag g_vmm_once;

template <class F>
bool entry(const char* name, F* out) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess ||
      !p)
    return false;
  *out = reinterpret_cast<F>(p);
  return true;
}

const Vmm* vmm() {
  std::call_once(g_vmm_once, [] {
    Vmm v;
    v.ok = entry("cuMemAddressReserve", &v.reserve) && entry("cuMemAddressFree", &v.addr_free) &&
           entry("cuMemCreate", &v.create) && entry("cuMemRelease", &v.release) && entry("cuMemMap", &v.map) &&
           entry("cuMemUnmap", &v.unmap) && entry("cuMemSetAccess", &v.set_access) &&
           entry("cuMemExportToShareableHandle", &v.export_fd) &&
           entry("cuMemImportFromShareableHandle", &v.import_fd) &&
           entry("cuMemGetAllocationGranularity", &v.granularity);
    g_vmm = v;
  });
  return g_vmm.ok ? &g_vmm : nullptr;
}

CUmemAllocationProp device_prop(int device) {
  CUmemAllocationProp prop;
  memset(&prop, 0, sizeof(prop));
  prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  prop.location.id = device;
  prop.requestedHandleTypes = CU_MEM_HANDLE_TYPE_POSIX_FILE_DESCRIPTOR;
  return prop;
}

}  // namespace

#define CKV(call, what)                                                                  \
  do {                                                                                   \
    CUresult r_ = (call);                                                                \
    if (r_ != CUDA_SUCCESS) return fail(PM_ERR_CUDA, "%s: driver error %d", what, (int)r_); \
  } while (0)

struct pm_parts {
  int device = 0;              // the device that reads the range
  uint64_t total = 0;          // bytes of the range (a multiple of the granularity)
  std::vector<uint64_t> begin; // slice p covers [begin[p], begin[p+1])
  std::vector<CUmemGenericAllocationHandle> handle;
  std::vector<int> backed;     // 0 none, 1 allocated here, 2 imported
  std::vector<int> owner;      // device of the slice's memory (-1 when imported: unknown here)
  CUdeviceptr base = 0;
  bool mapped = false;
};

static pm_status use_device(int device) {
  if (device < 0) return fail(PM_ERR_INVALID, "device %d", device);
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaFree(nullptr);  // the primary context must exist for the driver calls
  if (e != cudaSuccess) return fail(PM_ERR_NO_DEVICE, "device %d: %s", device, cudaGetErrorString(e));
  return PM_OK;
}

extern "C" pm_status pm_parts_granularity(int device, uint64_t* bytes) {
  if (!bytes) return fail(PM_ERR_INVALID, "pm_parts_granularity: bad arguments");
  pm_status st = use_device(device);
  if (st != PM_OK) return st;
  const Vmm* v = vmm();
  if (!v) return fail(PM_ERR_CUDA, "the CUDA virtual memory entry points are unavailable");
  CUmemAllocationProp prop = device_prop(device);
  size_t g = 0;
  CKV(v->granularity(&g, &prop, CU_MEM_ALLOC_GRANULARITY_MINIMUM), "cuMemGetAllocationGranularity");
  *bytes = g;
  return PM_OK;
}

extern "C" pm_status pm_parts_create(int device, int n_parts, const uint64_t* part_begin, uint64_t total_bytes,
                                     pm_parts** out) {
  if (!out || n_parts < 1 || n_parts > 1024 || !part_begin || total_bytes == 0)
    return fail(PM_ERR_INVALID, "pm_parts_create: bad arguments");
  uint64_t gran = 0;
  pm_status st = pm_parts_granularity(device, &gran);
  if (st != PM_OK) return st;
  if (total_bytes % gran) return fail(PM_ERR_INVALID, "range of %llu bytes is not a multiple of the granularity %llu",
                                      (unsigned long long)total_bytes, (unsigned long long)gran);
  if (part_begin[0] != 0) return fail(PM_ERR_INVALID, "the first slice must start at 0");
  for (int p = 0; p < n_parts; p++) {
    const uint64_t e = p + 1 < n_parts ? part_begin[p + 1] : total_bytes;
    if (part_begin[p] % gran || e <= part_begin[p] || e > total_bytes)
      return fail(PM_ERR_INVALID, "slice %d [%llu, %llu) is empty, unordered or not granularity-aligned", p,
                  (unsigned long long)part_begin[p], (unsigned long long)e);
  }
  std::unique_ptr<pm_parts> r(new pm_parts);
  r->device = device;
  r->total = total_bytes;
  r->begin.assign(part_begin, part_begin + n_parts);
  r->begin.push_back(total_bytes);
  r->handle.assign(n_parts, 0);
  r->backed.assign(n_parts, 0);
  r->owner.assign(n_parts, -1);
  CKV(vmm()->reserve(&r->base, total_bytes, gran, 0, 0), "cuMemAddressReserve");
  *out = r.release();
  return PM_OK;
}

static pm_status check_slice(const pm_parts* r, int p) {
  if (!r || p < 0 || p + 1 >= (int)r->begin.size()) return fail(PM_ERR_INVALID, "slice %d out of range", p);
  return PM_OK;
}

extern "C" pm_status pm_parts_alloc(pm_parts* r, int p, int owner_device) {
  pm_status st = check_slice(r, p);
  if (st != PM_OK) return st;
  if (r->backed[p] || r->mapped) return fail(PM_ERR_INVALID, "slice %d is backed already", p);
  st = use_device(owner_device);
  if (st != PM_OK) return st;
  CUmemAllocationProp prop = device_prop(owner_device);
  CKV(vmm()->create(&r->handle[p], r->begin[p + 1] - r->begin[p], &prop, 0), "cuMemCreate");
  r->backed[p] = 1;
  r->owner[p] = owner_device;
  return use_device(r->device);
}

extern "C" pm_status pm_parts_export(const pm_parts* r, int p, int* fd) {
  pm_status st = check_slice(r, p);
  if (st != PM_OK) return st;
  if (!fd || r->backed[p] != 1) return fail(PM_ERR_INVALID, "slice %d was not allocated here", p);
  int h = -1;
  CKV(vmm()->export_fd(&h, r->handle[p], CU_MEM_HANDLE_TYPE_POSIX_FILE_DESCRIPTOR, 0), "cuMemExportToShareableHandle");
  *fd = h;
  return PM_OK;
}

extern "C" pm_status pm_parts_import(pm_parts* r, int p, int fd) {
  pm_status st = check_slice(r, p);
  if (st != PM_OK) return st;
  if (r->backed[p] || r->mapped) return fail(PM_ERR_INVALID, "slice %d is backed already", p);
  if (fd < 0) return fail(PM_ERR_INVALID, "bad file descriptor");
  st = use_device(r->device);
  if (st != PM_OK) return st;
  CKV(vmm()->import_fd(&r->handle[p], (void*)(uintptr_t)fd, CU_MEM_HANDLE_TYPE_POSIX_FILE_DESCRIPTOR),
      "cuMemImportFromShareableHandle");
  r->backed[p] = 2;
  return PM_OK;
}

extern "C" pm_status pm_parts_map(pm_parts* r) {
  if (!r || r->mapped) return fail(PM_ERR_INVALID, "pm_parts_map: bad arguments");
  const int k = (int)r->handle.size();
  for (int p = 0; p < k; p++)
    if (!r->backed[p]) return fail(PM_ERR_INVALID, "slice %d has no memory", p);
  pm_status st = use_device(r->device);
  if (st != PM_OK) return st;
  int done = 0;
  CUresult err = CUDA_SUCCESS;
  for (; done < k; done++) {
    err = vmm()->map(r->base + r->begin[done], r->begin[done + 1] - r->begin[done], 0, r->handle[done], 0);
    if (err != CUDA_SUCCESS) break;
  }
  if (err == CUDA_SUCCESS) {
    CUmemAccessDesc acc;
    memset(&acc, 0, sizeof(acc));
    acc.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
    acc.location.id = r->device;
    acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
    err = vmm()->set_access(r->base, r->total, &acc, 1);
  }
  if (err != CUDA_SUCCESS) {
    for (int p = 0; p < done; p++) vmm()->unmap(r->base + r->begin[p], r->begin[p + 1] - r->begin[p]);
    return fail(PM_ERR_CUDA, "mapping the slices: driver error %d", (int)err);
  }
  r->mapped = true;
  return PM_OK;
}

extern "C" void* pm_parts_ptr(const pm_parts* r) { return r && r->mapped ? (void*)r->base : nullptr; }

extern "C" pm_status pm_parts_write(pm_parts* r, uint64_t offset, const void* host, uint64_t bytes) {
  if (!r || !r->mapped || (bytes && !host) || offset > r->total || bytes > r->total - offset)
    return fail(PM_ERR_INVALID, "pm_parts_write: bad arguments or range not mapped");
  pm_status st = use_device(r->device);
  if (st != PM_OK) return st;
  if (bytes) {
    cudaError_t e = cudaMemcpy((void*)(r->base + offset), host, bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return fail(PM_ERR_CUDA, "pm_parts_write: %s", cudaGetErrorString(e));
  }
  return PM_OK;
}

extern "C" void pm_parts_free(pm_parts* r) {
  if (!r) return;
  const Vmm* v = vmm();
  if (v) {
    cudaSetDevice(r->device);
    if (r->mapped)
      for (size_t p = 0; p + 1 < r->begin.size(); p++) v->unmap(r->base + r->begin[p], r->begin[p + 1] - r->begin[p]);
    for (size_t p = 0; p < r->handle.size(); p++)
      if (r->backed[p]) v->release(r->handle[p]);
    if (r->base) v->addr_free(r->base, r->total);
  }
  delete r;
}

// Stable counting sort of every list by label (ids stay ascending within a
// label): the layout a labeled paged graph caches, the same as the device's
// label_group_kernel writes.
extern "C" pm_status pm_label_group_host(int64_t n, int64_t n_adj, const uint64_t* rowptr, const int32_t* colidx,
                                         const uint32_t* labels, int32_t* out) {
  if (n < 0 || !rowptr || !labels || (n_adj > 0 && (!colidx || !out)))
    return fail(PM_ERR_INVALID, "pm_label_group_host: bad arguments");
  if (rowptr[n] != (uint64_t)n_adj) return fail(PM_ERR_INVALID, "rowptr[n] != n_adj");
  for (int64_t v = 0; v < n; v++)
    if (labels[v] >= 32) return fail(PM_ERR_FORMAT, "label %u of vertex %lld >= 32", labels[v], (long long)v);
  bool bad = false;
#pragma omp parallel for schedule(dynamic, 4096) reduction(|| : bad)
  for (int64_t v = 0; v < n; v++) {
    const uint64_t b = rowptr[v], e = rowptr[v + 1];
    int start[33] = {0};
    for (uint64_t i = b; i < e; i++) {
      const int32_t x = colidx[i];
      if (x < 0 || x >= n) { bad = true; break; }
      start[labels[x] + 1]++;
    }
    if (bad) continue;
    for (int l = 0; l < 32; l++) start[l + 1] += start[l];
    for (uint64_t i = b; i < e; i++) out[b + start[labels[colidx[i]]]++] = colidx[i];
  }
  if (bad) return fail(PM_ERR_FORMAT, "an adjacency entry is not a vertex id");
  return PM_OK;
}
