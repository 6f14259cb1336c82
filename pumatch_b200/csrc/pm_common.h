// pm_common.h -- internal declarations shared by the host (.cpp) and device
// (.cu) halves of libpumatch_b200.so.  Not part of the C-ABI.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "pumatch.h"

// Functions the host generators and their device counterpart share.
#ifdef __CUDACC__
#define PM_HD __host__ __device__
#else
#define PM_HD
#endif

namespace pm {

// ---------------------------------------------------------------- errors
// Sets the calling thread's last-error message and returns the status.
pm_status fail(pm_status s, const char* fmt, ...);

// ---------------------------------------------------------------- plans
// Host form of a compiled pattern (same content as pm_plan_desc).
struct Plan {
  int nnodes = 0;
  int nslots = 0;
  int multiplicity = 1;
  int labeled = 0;
  int level_begin[PM_MAX_PAT + 1] = {0};
  int degree[PM_MAX_PAT] = {0};
  int vertex_label[PM_MAX_PAT] = {0};
  uint32_t slot_labels[PM_MAX_SLOTS] = {0};
  uint32_t partial[PM_MAX_SLOTS] = {0};
  uint8_t set_ops[PM_MAX_SLOTS] = {0};
};

// Compiles .g text into a Plan; returns PM_OK or PM_ERR_FORMAT.
pm_status compile_plan(const std::string& text, bool labeled, Plan* out);

// Slot operation kinds, decoded from set_ops (reference src/pattern.h:348).
enum SlotKind : uint8_t { SLOT_FRESH = 0, SLOT_INTERSECT = 1, SLOT_COPY = 2 };
inline SlotKind slot_kind(uint8_t op) {
  return (op & 0x20) ? SLOT_FRESH : ((op & 0x40) ? SLOT_INTERSECT : SLOT_COPY);
}
inline int slot_parent(uint8_t op) { return op & 0x1F; }

// ---------------------------------------------------------------- RNG
// splitmix64 seeding xoshiro256** (the generators' only randomness source).
struct Rng {
  uint64_t s[4];
  PM_HD static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  PM_HD explicit Rng(uint64_t seed, uint64_t stream = 0) {
    uint64_t x = seed ^ (stream * 0xD1B54A32D192ED03ull);
    for (int i = 0; i < 4; i++) s[i] = splitmix(x);
  }
  PM_HD static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  PM_HD inline uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  PM_HD inline double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  PM_HD inline uint32_t below(uint32_t n) { return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32); }
};

// One R-MAT draw: per level one 16-bit slice of a 64-bit draw picks the
// quadrant (thresholds ta < tb < tc out of 65,536).  False for a rejected
// draw: an id >= n or a self-loop.  Shared by the host and device generators
// so that both produce the same edge sequence.
PM_HD inline bool rmat_draw(Rng& r, int scale, uint64_t n, uint32_t ta, uint32_t tb, uint32_t tc, uint32_t* u_out,
                            uint32_t* v_out) {
  uint64_t u = 0, v = 0, bits = 0;
  for (int l = 0; l < scale; l++) {
    if ((l & 3) == 0) bits = r.next();
    const uint32_t x = (uint32_t)(bits & 0xffff);
    bits >>= 16;
    const uint32_t bu = x >= tb, bv = (x >= ta && x < tb) || x >= tc;
    u = (u << 1) | bu;
    v = (v << 1) | bv;
  }
  *u_out = (uint32_t)u;
  *v_out = (uint32_t)v;
  return u < n && v < n && u != v;
}

// ---------------------------------------------------------------- CSR
// Builds a sorted CSR from unique undirected edge keys (lo << 32 | hi, lo < hi).
void csr_from_keys(int64_t n, const std::vector<uint64_t>& keys, uint64_t** rowptr,
                   int32_t** colidx, int64_t* n_adj, int32_t* max_degree);

}  // namespace pm
