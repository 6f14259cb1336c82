// pm_common.h -- internal declarations shared by the host (.cpp) and device
// (.cu) halves of libpumatch_b200.so.  Not part of the C-ABI.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "pumatch.h"

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
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  explicit Rng(uint64_t seed, uint64_t stream = 0) {
    uint64_t x = seed ^ (stream * 0xD1B54A32D192ED03ull);
    for (int i = 0; i < 4; i++) s[i] = splitmix(x);
  }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  inline uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  inline double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  inline uint32_t below(uint32_t n) { return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32); }
};

// ---------------------------------------------------------------- CSR
// Builds a sorted CSR from unique undirected edge keys (lo << 32 | hi, lo < hi).
void csr_from_keys(int64_t n, const std::vector<uint64_t>& keys, uint64_t** rowptr,
                   int32_t** colidx, int64_t* n_adj, int32_t* max_degree);

}  // namespace pm
