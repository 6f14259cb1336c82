// pm_learn.cu -- the learned scheduler's device code: per-root features and
// a 16 -> 64 -> 64 -> 2 MLP (ReLU) with BF16 weights and FP32 accumulation,
// trained with hand-written forward, backward and Adam kernels.
//
// The network predicts, per root edge, log(1 + DFS cost) and log(1 + adjacency
// reads) of the root's subtree.  Predictions only reorder work (heavy roots
// first) and choose which pages to keep resident; they never prune, so every
// count stays exact.  Nothing here exists in the reference.
//
// The layers are far too small for tensor cores to matter (5,378 parameters;
// a 64-wide layer is one 64x64 product per sample), so they run on the FMA
// pipes: one thread per sample forward, and a tiled backward where each block
// stages 64 samples' activations in shared memory and each thread then owns a
// slice of the weight gradients (an outer-product accumulation over the tile).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "pm_device.cuh"

using namespace pm;
namespace pm {
const Plan* plan_of(const pm_plan* h);
}

#define CKL(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(PM_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

namespace {

constexpr int NIN = PM_MLP_IN, NH = PM_MLP_HIDDEN, NOUT = PM_MLP_OUT;
// parameter layout (row-major, input-major): W1[NIN][NH] b1[NH] W2[NH][NH] b2[NH] W3[NH][NOUT] b3[NOUT]
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + NIN * NH;
constexpr int OFF_W2 = OFF_B1 + NH;
constexpr int OFF_B2 = OFF_W2 + NH * NH;
constexpr int OFF_W3 = OFF_B2 + NH;
constexpr int OFF_B3 = OFF_W3 + NH * NOUT;
constexpr int NPARAM = OFF_B3 + NOUT;
static_assert(NPARAM == PM_MLP_PARAMS, "parameter count");

__device__ __forceinline__ float bf(const __nv_bfloat16 v) { return __bfloat162float(v); }

// ---------------------------------------------------------------- forward
__global__ void mlp_forward_kernel(const __nv_bfloat16* __restrict__ wq, const float* __restrict__ x, int64_t n,
                                   float* __restrict__ y) {
  __shared__ float w[NPARAM];
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) w[i] = bf(wq[i]);
  __syncthreads();
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    float xin[NIN];
#pragma unroll
    for (int i = 0; i < NIN; i++) xin[i] = x[s * NIN + i];
    float h1[NH];
#pragma unroll 8
    for (int j = 0; j < NH; j++) {
      float z = w[OFF_B1 + j];
#pragma unroll
      for (int i = 0; i < NIN; i++) z = fmaf(xin[i], w[OFF_W1 + i * NH + j], z);
      h1[j] = fmaxf(z, 0.f);
    }
    float o0 = w[OFF_B3], o1 = w[OFF_B3 + 1];
    for (int k = 0; k < NH; k++) {
      float z = w[OFF_B2 + k];
#pragma unroll 8
      for (int j = 0; j < NH; j++) z = fmaf(h1[j], w[OFF_W2 + j * NH + k], z);
      const float a = fmaxf(z, 0.f);
      o0 = fmaf(a, w[OFF_W3 + k * NOUT], o0);
      o1 = fmaf(a, w[OFF_W3 + k * NOUT + 1], o1);
    }
    y[s * NOUT] = o0;
    y[s * NOUT + 1] = o1;
  }
}

// ---------------------------------------------------------------- backward
// Mean-squared-error gradients over the batch, accumulated in FP32.
constexpr int TILE = 64;

struct BackwardSmem {
  float w[NPARAM];
  float sx[TILE][NIN];
  float sh1[TILE][NH];    // relu(z1)
  float sdz1[TILE][NH];   // dL/dz1
  float sa2[TILE][NH];    // relu(z2)
  float sdz2[TILE][NH];   // dL/dz2
  float sdo[TILE][NOUT];  // dL/dout
  float sloss[TILE];
};

__global__ void __launch_bounds__(256) mlp_backward_kernel(const __nv_bfloat16* __restrict__ wq,
                                                           const float* __restrict__ x, const float* __restrict__ t,
                                                           int64_t n, float* __restrict__ grad,
                                                           float* __restrict__ loss) {
  extern __shared__ float4 smem_raw[];
  BackwardSmem& S = *reinterpret_cast<BackwardSmem*>(smem_raw);
  float* w = S.w;
  auto& sx = S.sx;
  auto& sh1 = S.sh1;
  auto& sdz1 = S.sdz1;
  auto& sa2 = S.sa2;
  auto& sdz2 = S.sdz2;
  auto& sdo = S.sdo;
  auto& sloss = S.sloss;
  for (int i = threadIdx.x; i < NPARAM; i += blockDim.x) w[i] = bf(wq[i]);
  __syncthreads();
  float g[(NPARAM + 255) / 256];  // this thread's slice of the gradient
  for (int i = 0; i < (NPARAM + 255) / 256; i++) g[i] = 0.f;
  float lsum = 0.f;
  const float inv_n = 1.f / (float)(n * NOUT);
  for (int64_t base = (int64_t)blockIdx.x * TILE; base < n; base += (int64_t)gridDim.x * TILE) {
    // phase A: one thread per sample -- forward and backward of the activations
    if (threadIdx.x < TILE) {
      const int r = threadIdx.x;
      const int64_t s = base + r;
      if (s < n) {
        for (int i = 0; i < NIN; i++) sx[r][i] = x[s * NIN + i];
        float z1[NH];
        for (int j = 0; j < NH; j++) {
          float z = w[OFF_B1 + j];
          for (int i = 0; i < NIN; i++) z = fmaf(sx[r][i], w[OFF_W1 + i * NH + j], z);
          z1[j] = z;
          sh1[r][j] = fmaxf(z, 0.f);
        }
        float o0 = w[OFF_B3], o1 = w[OFF_B3 + 1];
        for (int k = 0; k < NH; k++) {
          float z = w[OFF_B2 + k];
          for (int j = 0; j < NH; j++) z = fmaf(sh1[r][j], w[OFF_W2 + j * NH + k], z);
          const float a = fmaxf(z, 0.f);
          sa2[r][k] = a;
          sdz2[r][k] = z > 0.f ? 1.f : 0.f;  // mask, scaled below
          o0 = fmaf(a, w[OFF_W3 + k * NOUT], o0);
          o1 = fmaf(a, w[OFF_W3 + k * NOUT + 1], o1);
        }
        const float e0 = o0 - t[s * NOUT], e1 = o1 - t[s * NOUT + 1];
        sloss[r] = e0 * e0 + e1 * e1;
        const float d0 = 2.f * e0 * inv_n, d1 = 2.f * e1 * inv_n;
        sdo[r][0] = d0;
        sdo[r][1] = d1;
        for (int k = 0; k < NH; k++)
          sdz2[r][k] *= fmaf(w[OFF_W3 + k * NOUT], d0, w[OFF_W3 + k * NOUT + 1] * d1);
        for (int j = 0; j < NH; j++) {
          float d = 0.f;
          for (int k = 0; k < NH; k++) d = fmaf(w[OFF_W2 + j * NH + k], sdz2[r][k], d);
          sdz1[r][j] = z1[j] > 0.f ? d : 0.f;
        }
      } else {
        for (int i = 0; i < NIN; i++) sx[r][i] = 0.f;
        for (int j = 0; j < NH; j++) { sh1[r][j] = 0.f; sdz1[r][j] = 0.f; sa2[r][j] = 0.f; sdz2[r][j] = 0.f; }
        sdo[r][0] = sdo[r][1] = 0.f;
        sloss[r] = 0.f;
      }
    }
    __syncthreads();
    // phase B: each thread accumulates its parameters over the tile
    for (int q = 0; q < (NPARAM + 255) / 256; q++) {
      const int pidx = threadIdx.x + q * 256;
      if (pidx >= NPARAM) break;
      float acc = 0.f;
      if (pidx < OFF_B1) {
        const int i = pidx / NH, j = pidx % NH;
        for (int r = 0; r < TILE; r++) acc = fmaf(sx[r][i], sdz1[r][j], acc);
      } else if (pidx < OFF_W2) {
        const int j = pidx - OFF_B1;
        for (int r = 0; r < TILE; r++) acc += sdz1[r][j];
      } else if (pidx < OFF_B2) {
        const int j = (pidx - OFF_W2) / NH, k = (pidx - OFF_W2) % NH;
        for (int r = 0; r < TILE; r++) acc = fmaf(sh1[r][j], sdz2[r][k], acc);
      } else if (pidx < OFF_W3) {
        const int k = pidx - OFF_B2;
        for (int r = 0; r < TILE; r++) acc += sdz2[r][k];
      } else if (pidx < OFF_B3) {
        const int k = (pidx - OFF_W3) / NOUT, o = (pidx - OFF_W3) % NOUT;
        for (int r = 0; r < TILE; r++) acc = fmaf(sa2[r][k], sdo[r][o], acc);
      } else {
        const int o = pidx - OFF_B3;
        for (int r = 0; r < TILE; r++) acc += sdo[r][o];
      }
      g[q] += acc;
    }
    if (threadIdx.x == 0)
      for (int r = 0; r < TILE; r++) lsum += sloss[r];
    __syncthreads();
  }
  for (int q = 0; q < (NPARAM + 255) / 256; q++) {
    const int pidx = threadIdx.x + q * 256;
    if (pidx < NPARAM) atomicAdd(&grad[pidx], g[q]);
  }
  if (threadIdx.x == 0) atomicAdd(loss, lsum * inv_n);
}

// ---------------------------------------------------------------- Adam
__global__ void adam_kernel(float* __restrict__ w, __nv_bfloat16* __restrict__ wq, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NPARAM) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  wq[i] = __float2bfloat16_rn(wi);
}

__global__ void quantize_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NPARAM) wq[i] = __float2bfloat16_rn(w[i]);
}

// ---------------------------------------------------------------- features
// 16 features of a root edge (v0, v1); f[15] depends on the plan (how many
// neighbours of v1 carry pattern vertex 2's label, as a fraction of deg v1).
// What the first two levels of a root's DFS will see, for the cost features:
// v2's candidates are v1's neighbours with v2's label (labeled) or below v0
// (unlabeled, when the plan bounds v2 by v0); each contributes its neighbours
// with v3's label (the label-group offsets give them directly) or its degree.
struct FeatPlan {
  int lab2, lab3;      // pattern labels of v2 and v3 (labeled; -1 when absent)
  int bound_v0;        // unlabeled: v2 < v0
  int nl1;             // label-group stride of lab_off, 0 without groups
  const int32_t* lab_off;
};

__global__ void features_kernel(const uint64_t* __restrict__ rowptr, const int32_t* __restrict__ colidx,
                                const uint8_t* __restrict__ labels, const int32_t* __restrict__ maxnbrdeg,
                                const float* __restrict__ deg_rank, int nlabels, FeatPlan fp, const int2* roots,
                                int64_t nroots, float* __restrict__ out) {
  const int lab2 = fp.lab2;
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < nroots; r += warps) {
    const int2 e = roots[r];
    const uint64_t b1 = rowptr[e.y], e1 = rowptr[e.y + 1];
    float two_hop = 0.f, pairs = 0.f;
    int hist[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int match2 = 0, cand2 = 0;
    for (uint64_t i = b1 + lane; i < e1; i += 32) {
      const int u = colidx[i];
      const float du = (float)(rowptr[u + 1] - rowptr[u]);
      two_hop += du;
      bool is_cand;
      if (labels) {
        const int l = labels[u];
        hist[l & 7]++;
        match2 += (l == lab2);
        is_cand = (l == lab2);
      } else {
        is_cand = !fp.bound_v0 || u < e.x;
      }
      if (is_cand) {
        cand2++;
        if (labels && fp.lab_off && fp.lab3 >= 0 && fp.lab3 < fp.nl1 - 1) {
          const int32_t* o = fp.lab_off + (int64_t)u * fp.nl1;
          pairs += (float)(o[fp.lab3 + 1] - o[fp.lab3]);
        } else {
          pairs += du;
        }
      }
    }
    for (int o = 16; o; o >>= 1) {
      two_hop += __shfl_xor_sync(0xffffffffu, two_hop, o);
      pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
      match2 += __shfl_xor_sync(0xffffffffu, match2, o);
      cand2 += __shfl_xor_sync(0xffffffffu, cand2, o);
#pragma unroll
      for (int k = 0; k < 8; k++) hist[k] += __shfl_xor_sync(0xffffffffu, hist[k], o);
    }
    if (lane == 0) {
      const float d0 = (float)(rowptr[e.x + 1] - rowptr[e.x]);
      const float d1 = (float)(e1 - b1);
      float* f = out + r * NIN;
      f[0] = log2f(1.f + d0);
      f[1] = log2f(1.f + d1);
      f[2] = log2f(1.f + (float)cand2);  // level 1's candidates (v2)
      f[3] = log2f(1.f + pairs);         // (v2, v3) candidate pairs below them
      f[4] = log2f(1.f + two_hop);
      f[5] = log2f(1.f + (float)maxnbrdeg[e.y]);
      f[6] = deg_rank ? deg_rank[e.y] : 0.f;
      for (int k = 0; k < 8; k++) f[7 + k] = d1 > 0.f ? (float)hist[k] / d1 : 0.f;
      f[15] = d1 > 0.f ? (float)match2 / d1 : 0.f;
    }
  }
}

__global__ void deg_rank_kernel(const uint64_t* rowptr, int64_t n, const unsigned int* cdf, int32_t maxd,
                                float* out) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int bucket = (int)floorf(log2f(1.f + (float)(rowptr[v + 1] - rowptr[v])) * 4.f);
    out[v] = (float)cdf[min(bucket, 255)] / (float)(n > 0 ? n : 1);
    (void)maxd;
  }
}

__global__ void deg_hist_kernel(const uint64_t* rowptr, int64_t n, unsigned int* hist) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
    const int bucket = (int)floorf(log2f(1.f + (float)(rowptr[v + 1] - rowptr[v])) * 4.f);
    atomicAdd(&hist[min(bucket, 255)], 1u);
  }
}

}  // namespace

// =====================================================================
// C-ABI
// =====================================================================

struct pm_mlp {
  int device = 0;
  float* w = nullptr;            // FP32 master weights
  __nv_bfloat16* wq = nullptr;   // BF16 copy used by forward/backward
  float* g = nullptr;
  float* m = nullptr;
  float* v = nullptr;
  float* loss = nullptr;
  int64_t step = 0;
  int nsm = 148;
};

extern "C" void pm_mlp_free(pm_mlp* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  cudaFree(m->w);
  cudaFree(m->wq);
  cudaFree(m->g);
  cudaFree(m->m);
  cudaFree(m->v);
  cudaFree(m->loss);
  delete m;
}

extern "C" pm_status pm_mlp_create(int device, uint64_t seed, pm_mlp** out) {
  if (!out) return fail(PM_ERR_INVALID, "pm_mlp_create: null argument");
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
    return fail(PM_ERR_NO_DEVICE, "no CUDA device available; libpumatch_b200 has no CPU path");
  CKL(cudaSetDevice(device));
  std::unique_ptr<pm_mlp, void (*)(pm_mlp*)> m(new pm_mlp, pm_mlp_free);
  m->device = device;
  CKL(cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, device));
  CKL(cudaMalloc(&m->w, sizeof(float) * NPARAM));
  CKL(cudaMalloc(&m->wq, sizeof(__nv_bfloat16) * NPARAM));
  CKL(cudaMalloc(&m->g, sizeof(float) * NPARAM));
  CKL(cudaMalloc(&m->m, sizeof(float) * NPARAM));
  CKL(cudaMalloc(&m->v, sizeof(float) * NPARAM));
  CKL(cudaMalloc(&m->loss, sizeof(float)));
  // He-uniform init from the seed (host side, deterministic)
  std::vector<float> h(NPARAM, 0.f);
  Rng r(seed, 77);
  auto fill = [&](int off, int fan_in, int count) {
    const float lim = std::sqrt(6.f / (float)fan_in);
    for (int i = 0; i < count; i++) h[off + i] = (float)((r.uniform() * 2.0 - 1.0) * lim);
  };
  fill(OFF_W1, NIN, NIN * NH);
  fill(OFF_W2, NH, NH * NH);
  fill(OFF_W3, NH, NH * NOUT);
  CKL(cudaMemcpy(m->w, h.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
  CKL(cudaMemset(m->m, 0, sizeof(float) * NPARAM));
  CKL(cudaMemset(m->v, 0, sizeof(float) * NPARAM));
  PM_CK_PENDING("pm_mlp_create");
  quantize_kernel<<<(NPARAM + 255) / 256, 256>>>(m->w, m->wq);
  CKL(cudaGetLastError());
  CKL(cudaDeviceSynchronize());
  *out = m.release();
  return PM_OK;
}

extern "C" pm_status pm_mlp_get_weights(pm_mlp* m, float* host_out) {
  if (!m || !host_out) return fail(PM_ERR_INVALID, "pm_mlp_get_weights: null argument");
  CKL(cudaSetDevice(m->device));
  CKL(cudaMemcpy(host_out, m->w, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
  return PM_OK;
}

extern "C" pm_status pm_mlp_set_weights(pm_mlp* m, const float* host_in) {
  if (!m || !host_in) return fail(PM_ERR_INVALID, "pm_mlp_set_weights: null argument");
  CKL(cudaSetDevice(m->device));
  CKL(cudaMemcpy(m->w, host_in, sizeof(float) * NPARAM, cudaMemcpyHostToDevice));
  PM_CK_PENDING("pm_mlp_set_weights");
  quantize_kernel<<<(NPARAM + 255) / 256, 256>>>(m->w, m->wq);
  CKL(cudaGetLastError());
  CKL(cudaDeviceSynchronize());
  m->step = 0;
  CKL(cudaMemset(m->m, 0, sizeof(float) * NPARAM));
  CKL(cudaMemset(m->v, 0, sizeof(float) * NPARAM));
  return PM_OK;
}

extern "C" pm_status pm_mlp_forward(pm_mlp* m, const float* d_x, int64_t n, float* d_y) {
  if (!m || (n > 0 && (!d_x || !d_y))) return fail(PM_ERR_INVALID, "pm_mlp_forward: bad arguments");
  CKL(cudaSetDevice(m->device));
  if (n == 0) return PM_OK;
  const int blocks = (int)std::min<int64_t>((n + 127) / 128, 8 * m->nsm);
  PM_CK_PENDING("MLP kernels");
  mlp_forward_kernel<<<blocks, 128>>>(m->wq, d_x, n, d_y);
  CKL(cudaGetLastError());
  CKL(cudaDeviceSynchronize());
  return PM_OK;
}

extern "C" pm_status pm_mlp_gradient(pm_mlp* m, const float* d_x, const float* d_t, int64_t n, float* host_grad,
                                     float* loss_out) {
  if (!m || n <= 0 || !d_x || !d_t) return fail(PM_ERR_INVALID, "pm_mlp_gradient: bad arguments");
  CKL(cudaSetDevice(m->device));
  CKL(cudaMemset(m->g, 0, sizeof(float) * NPARAM));
  CKL(cudaMemset(m->loss, 0, sizeof(float)));
  const int blocks = (int)std::min<int64_t>((n + TILE - 1) / TILE, 2 * m->nsm);
  CKL(cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sizeof(BackwardSmem)));
  PM_CK_PENDING("MLP kernels");
  mlp_backward_kernel<<<blocks, 256, sizeof(BackwardSmem)>>>(m->wq, d_x, d_t, n, m->g, m->loss);
  CKL(cudaGetLastError());
  if (host_grad) CKL(cudaMemcpy(host_grad, m->g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost));
  if (loss_out) CKL(cudaMemcpy(loss_out, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
  CKL(cudaDeviceSynchronize());
  return PM_OK;
}

extern "C" pm_status pm_mlp_train_step(pm_mlp* m, const float* d_x, const float* d_t, int64_t n, float lr,
                                       float* loss_out) {
  pm_status st = pm_mlp_gradient(m, d_x, d_t, n, nullptr, loss_out);
  if (st != PM_OK) return st;
  m->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
  PM_CK_PENDING("MLP kernels");
  adam_kernel<<<(NPARAM + 255) / 256, 256>>>(m->w, m->wq, m->g, m->m, m->v, lr, b1, b2, 1e-8f, c1, c2);
  CKL(cudaGetLastError());
  CKL(cudaDeviceSynchronize());
  return PM_OK;
}

namespace pm {
pm_status root_list_for(pm_ctx* c, const pm_graph* g, const pm_plan* p, const int2** roots, int64_t* n);
}

extern "C" pm_status pm_root_features(pm_ctx* c, const pm_graph* g, const pm_plan* p, float* d_features,
                                      int64_t cap, int64_t* n_roots) {
  if (!c || !g || !p || !n_roots) return fail(PM_ERR_INVALID, "pm_root_features: null argument");
  const int2* roots = nullptr;
  int64_t n = 0;
  pm_status st = root_list_for(c, g, p, &roots, &n);
  if (st != PM_OK) return st;
  *n_roots = n;
  if (!d_features || n == 0) return PM_OK;
  if (cap < n) return fail(PM_ERR_INVALID, "pm_root_features: feature buffer holds %lld roots, need %lld",
                           (long long)cap, (long long)n);
  // degree-quantile table
  unsigned int* hist = nullptr;
  float* rank = nullptr;
  PM_CK_PENDING("pm_root_features");
  CKL(cudaMalloc(&hist, 256 * sizeof(unsigned int)));
  CKL(cudaMalloc(&rank, sizeof(float) * std::max<int64_t>(g->n, 1)));
  CKL(cudaMemset(hist, 0, 256 * sizeof(unsigned int)));
  deg_hist_kernel<<<1024, 256>>>(g->d_rowptr, g->n, hist);
  std::vector<unsigned int> h(256);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(h.data(), hist, 256 * sizeof(unsigned int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    cudaFree(hist);
    cudaFree(rank);
    CKL(e);
  }
  unsigned int acc = 0;
  for (int i = 0; i < 256; i++) { acc += h[i]; h[i] = acc; }
  e = cudaMemcpy(hist, h.data(), 256 * sizeof(unsigned int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    deg_rank_kernel<<<1024, 256>>>(g->d_rowptr, g->n, hist, g->maxdeg, rank);
    e = cudaGetLastError();
  }
  const Plan* pl = plan_of(p);
  const int32_t* colidx = g->residency == PM_RESIDENT_HBM ? g->d_colidx : g->h_colidx_dev;
  FeatPlan fp;
  fp.lab2 = pl->nnodes > 2 ? pl->vertex_label[2] : -1;
  fp.lab3 = pl->nnodes > 3 ? pl->vertex_label[3] : -1;
  fp.bound_v0 = !pl->labeled && (pl->partial[pl->level_begin[1]] & 1u);
  fp.nl1 = g->d_lab_off ? g->nl1 : 0;
  fp.lab_off = g->d_lab_off;
  if (e == cudaSuccess) {
    features_kernel<<<4 * c->nsm, 256>>>(g->d_rowptr, colidx, g->d_labels, g->d_maxnbrdeg, rank, g->nlabels, fp,
                                         roots, n, d_features);
    e = cudaGetLastError();
  }
  cudaError_t s2 = cudaDeviceSynchronize();
  cudaFree(hist);
  cudaFree(rank);
  CKL(e);
  CKL(s2);
  return PM_OK;
}
