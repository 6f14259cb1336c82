// pm_gen.cu -- R-MAT generation on the device, for graphs whose host-side
// edge sort would take too long or too much memory (the configured 65M-vertex
// graph has 1.8e9 undirected edges, 3.6e9 adjacency entries).
//
// Same definition as pm_gen_rmat (pm_host.cpp), so both return the same
// arrays: batch t (t = 1, 2, ...) is 65,536 draws from the xoshiro256** stream
// Rng(seed, t) through the shared rmat_draw; the graph is the first n_edges
// distinct undirected non-loop edges of that draw sequence, as a sorted CSR.
//
// Steps (all on the device, CUB radix sorts with 64-bit item counts):
//   1. one thread per batch draws its 65,536 keys (lo << scale | hi);
//   2. sort (key, draw index) by key: each key's first draw comes first;
//   3. keep the first draw of every key; if fewer than n_edges are distinct,
//      draw more batches and start over;
//   4. sort the distinct keys by their first draw index and keep n_edges;
//   5. both directions of every kept edge, sorted by (row, column): colidx,
//      and row counts scanned into rowptr.
// The reference has no generator (its graphs are converted datasets,
// graph_converter/convert.sh); this is workload tooling for the benchmarks.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "pm_common.h"
#include "pm_device.cuh"

using namespace pm;

namespace {

constexpr int64_t kBatch = 1 << 16;

struct RmatParams {
  int scale;
  uint64_t n;
  uint32_t ta, tb, tc;
  uint64_t reject;  // key of a rejected draw: sorts after every valid key
};

__global__ void draw_kernel(uint64_t seed, int64_t nbatch, RmatParams p, uint64_t* keys, uint32_t* pos) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbatch) return;
  Rng r(seed, (uint64_t)b + 1);
  uint64_t* out = keys + b * kBatch;
  uint32_t* po = pos + b * kBatch;
  for (int64_t k = 0; k < kBatch; k++) {
    uint32_t u, v;
    const bool ok = rmat_draw(r, p.scale, p.n, p.ta, p.tb, p.tc, &u, &v);
    const uint64_t lo = min(u, v), hi = max(u, v);
    out[k] = ok ? (lo << p.scale | hi) : p.reject;
    po[k] = (uint32_t)(b * kBatch + k);
  }
}

// flag[i] = key i is the first draw of its key and not a rejection
__global__ void first_flags(const uint64_t* keys, int64_t cnt, uint64_t reject, uint8_t* flags) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x)
    flags[i] = keys[i] != reject && (i == 0 || keys[i] != keys[i - 1]);
}

// both directions of edge e as (row << 32 | column)
__global__ void directed_kernel(const uint64_t* keys, int64_t m, int scale, uint64_t* out) {
  const uint64_t mask = (1ull << scale) - 1;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t lo = keys[e] >> scale, hi = keys[e] & mask;
    out[2 * e] = lo << 32 | hi;
    out[2 * e + 1] = hi << 32 | lo;
  }
}

__global__ void split_kernel(const uint64_t* pairs, int64_t cnt, int32_t* colidx, uint32_t* deg) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
    colidx[i] = (int32_t)(pairs[i] & 0xffffffffu);
    atomicAdd(&deg[pairs[i] >> 32], 1u);
  }
}

// RAII device buffer for the generator's temporaries
struct DBuf {
  void* p = nullptr;
  ~DBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t bytes) {
    if (p) cudaFree(p);
    p = nullptr;
    return cudaMalloc(&p, std::max<size_t>(bytes, 1));
  }
  void release() { if (p) cudaFree(p); p = nullptr; }
  template <class T> T* as() const { return (T*)p; }
};

#define CKG(call)                                                                              \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      return fail(e_ == cudaErrorMemoryAllocation ? PM_ERR_OOM : PM_ERR_CUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                          \
  } while (0)

}  // namespace

extern "C" pm_status pm_gen_rmat_device(int64_t n, int64_t m, double a, double b, double c, uint64_t seed,
                                        int device, uint64_t** rowptr_out, int32_t** colidx_out, int64_t* n_adj,
                                        int32_t* max_degree) {
  if (n < 2 || n > INT32_MAX || m < 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 || !rowptr_out || !colidx_out ||
      !n_adj || !max_degree)
    return fail(PM_ERR_INVALID, "pm_gen_rmat_device: bad arguments");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return fail(PM_ERR_NO_DEVICE, "no CUDA device available; pm_gen_rmat_device has no CPU path");
  if (device < 0 || device >= count) return fail(PM_ERR_INVALID, "device %d out of range", device);
  CKG(cudaSetDevice(device));
  PM_CK_PENDING("pm_gen_rmat_device");
  RmatParams p;
  p.scale = 0;
  while ((1ll << p.scale) < n) p.scale++;
  if (p.scale > 31) return fail(PM_ERR_INVALID, "pm_gen_rmat_device: n too large");
  p.n = (uint64_t)n;
  p.ta = (uint32_t)std::lround(a * 65536.0);
  p.tb = (uint32_t)std::lround((a + b) * 65536.0);
  p.tc = (uint32_t)std::lround((a + b + c) * 65536.0);
  p.reject = (1ull << (2 * p.scale)) - 1;
  const int key_bits = 2 * p.scale;

  // 1-4: the first m distinct keys of the draw sequence
  DBuf edges;  // uint64[m], sorted by first draw
  int64_t want = m + m / 4 + 1024;
  for (int attempt = 0;; attempt++) {
    const int64_t nb = (want + kBatch - 1) / kBatch;
    const int64_t draws = nb * kBatch;
    if (attempt > 8 || draws >= (int64_t)UINT32_MAX)
      return fail(PM_ERR_INVALID, "pm_gen_rmat_device: cannot reach %lld distinct edges", (long long)m);
    DBuf keys, keys2, pos, pos2, tmp, flags, nsel;
    CKG(keys.alloc(8 * (size_t)draws));
    CKG(pos.alloc(4 * (size_t)draws));
    draw_kernel<<<(unsigned)((nb + 127) / 128), 128>>>(seed, nb, p, keys.as<uint64_t>(), pos.as<uint32_t>());
    CKG(cudaGetLastError());
    CKG(keys2.alloc(8 * (size_t)draws));
    CKG(pos2.alloc(4 * (size_t)draws));
    // ping-pong buffers: the sort needs no copy of its input
    cub::DoubleBuffer<uint64_t> dk(keys.as<uint64_t>(), keys2.as<uint64_t>());
    cub::DoubleBuffer<uint32_t> dv(pos.as<uint32_t>(), pos2.as<uint32_t>());
    size_t tb = 0;
    CKG(cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, draws, 0, key_bits));
    CKG(tmp.alloc(tb));
    CKG(cub::DeviceRadixSort::SortPairs(tmp.p, tb, dk, dv, draws, 0, key_bits));
    tmp.release();
    uint64_t* sk = dk.Current();
    uint32_t* sv = dv.Current();
    uint64_t* ok = dk.Alternate();
    uint32_t* ov = dv.Alternate();
    CKG(flags.alloc((size_t)draws));
    first_flags<<<4096, 256>>>(sk, draws, p.reject, flags.as<uint8_t>());
    CKG(cudaGetLastError());
    // distinct keys and their first draws (into the other buffers)
    CKG(nsel.alloc(sizeof(int64_t)));
    tb = 0;
    size_t tbv = 0;
    CKG(cub::DeviceSelect::Flagged(nullptr, tb, sk, flags.as<uint8_t>(), ok, nsel.as<int64_t>(), draws));
    CKG(cub::DeviceSelect::Flagged(nullptr, tbv, sv, flags.as<uint8_t>(), ov, nsel.as<int64_t>(), draws));
    tb = std::max(tb, tbv);
    CKG(tmp.alloc(tb));
    CKG(cub::DeviceSelect::Flagged(tmp.p, tb, sk, flags.as<uint8_t>(), ok, nsel.as<int64_t>(), draws));
    CKG(cub::DeviceSelect::Flagged(tmp.p, tb, sv, flags.as<uint8_t>(), ov, nsel.as<int64_t>(), draws));
    int64_t distinct = 0;
    CKG(cudaMemcpy(&distinct, nsel.p, sizeof(int64_t), cudaMemcpyDeviceToHost));
    tmp.release();
    flags.release();
    if (distinct < m) {
      want = std::max<int64_t>(want + want / 2, (int64_t)((double)draws * (double)m / std::max<int64_t>(distinct, 1) * 1.1));
      continue;
    }
    // by first draw: the first m distinct edges
    cub::DoubleBuffer<uint32_t> ek(ov, sv);
    cub::DoubleBuffer<uint64_t> ev(ok, sk);
    tb = 0;
    CKG(cub::DeviceRadixSort::SortPairs(nullptr, tb, ek, ev, distinct, 0, 32));
    CKG(tmp.alloc(tb));
    CKG(cub::DeviceRadixSort::SortPairs(tmp.p, tb, ek, ev, distinct, 0, 32));
    CKG(edges.alloc(8 * (size_t)std::max<int64_t>(m, 1)));
    if (m) CKG(cudaMemcpy(edges.p, ev.Current(), 8 * (size_t)m, cudaMemcpyDeviceToDevice));
    break;
  }

  // 5: both directions sorted by (row, column) -> colidx and rowptr
  const int64_t nadj = 2 * m;
  DBuf dir, dir2, tmp, col, deg, rp, mx;
  CKG(dir.alloc(8 * (size_t)std::max<int64_t>(nadj, 1)));
  directed_kernel<<<4096, 256>>>(edges.as<uint64_t>(), m, p.scale, dir.as<uint64_t>());
  CKG(cudaGetLastError());
  edges.release();
  CKG(dir2.alloc(8 * (size_t)std::max<int64_t>(nadj, 1)));
  cub::DoubleBuffer<uint64_t> dd(dir.as<uint64_t>(), dir2.as<uint64_t>());
  size_t tb = 0;
  CKG(cub::DeviceRadixSort::SortKeys(nullptr, tb, dd, nadj, 0, 32 + p.scale));
  CKG(tmp.alloc(tb));
  CKG(cub::DeviceRadixSort::SortKeys(tmp.p, tb, dd, nadj, 0, 32 + p.scale));
  tmp.release();
  const uint64_t* sorted = dd.Current();
  CKG(col.alloc(4 * (size_t)std::max<int64_t>(nadj, 1)));
  CKG(deg.alloc(4 * (size_t)(n + 1)));
  CKG(cudaMemset(deg.p, 0, 4 * (size_t)(n + 1)));
  split_kernel<<<4096, 256>>>(sorted, nadj, col.as<int32_t>(), deg.as<uint32_t>());
  CKG(cudaGetLastError());
  dir.release();
  dir2.release();
  CKG(rp.alloc(8 * (size_t)(n + 1)));
  CKG(mx.alloc(sizeof(uint32_t)));
  tb = 0;
  CKG(cub::DeviceScan::ExclusiveSum(nullptr, tb, deg.as<uint32_t>(), rp.as<uint64_t>(), n + 1));
  size_t tb2 = 0;
  CKG(cub::DeviceReduce::Max(nullptr, tb2, deg.as<uint32_t>(), mx.as<uint32_t>(), n));
  CKG(tmp.alloc(std::max(tb, tb2)));
  CKG(cub::DeviceScan::ExclusiveSum(tmp.p, tb, deg.as<uint32_t>(), rp.as<uint64_t>(), n + 1));
  CKG(cub::DeviceReduce::Max(tmp.p, tb2, deg.as<uint32_t>(), mx.as<uint32_t>(), n));
  uint32_t maxd = 0;
  CKG(cudaMemcpy(&maxd, mx.p, sizeof(maxd), cudaMemcpyDeviceToHost));
  uint64_t* h_rp = (uint64_t*)malloc(8 * (size_t)(n + 1));
  int32_t* h_ci = (int32_t*)malloc(4 * (size_t)std::max<int64_t>(nadj, 1));
  if (!h_rp || !h_ci) {
    free(h_rp);
    free(h_ci);
    return fail(PM_ERR_OOM, "pm_gen_rmat_device: host allocation of %lld entries failed", (long long)nadj);
  }
  cudaError_t e = cudaMemcpy(h_rp, rp.p, 8 * (size_t)(n + 1), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && nadj) e = cudaMemcpy(h_ci, col.p, 4 * (size_t)nadj, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    free(h_rp);
    free(h_ci);
    return fail(PM_ERR_CUDA, "pm_gen_rmat_device: copy-out failed: %s", cudaGetErrorString(e));
  }
  *rowptr_out = h_rp;
  *colidx_out = h_ci;
  *n_adj = nadj;
  *max_degree = (int32_t)maxd;
  return PM_OK;
}
