// Shared device/host definitions of the B200 sampler: the counter-based
// stream that replaces the reference's per-thread MMIX LCG
// (silvan/src/Rand_gen.cpp:15-25), the per-slot node record, error helpers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "silvan.h"

#define SILVAN_HD __host__ __device__ __forceinline__

namespace silvan {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  One draw of the stream
// (seed; sample, kind) at position `draw`:
//   counter = (draw, sample, kind, 0), key = (seed lo, seed hi)
//   value   = out[1] << 32 | out[0]
// kind 0 is the s-t sampler stream, kind 1 the Rademacher-sign stream of
// silvan/src/Probabilistic.cpp:487-497.  The reference's get_max(m) keeps the
// low 32 bits of the draw (Rand_gen.cpp:22-24), so callers use out[0] % m.
// ---------------------------------------------------------------------------
enum : uint32_t { kStreamSampler = 0, kStreamRademacher = 1 };

SILVAN_HD void philox_mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
#ifdef __CUDA_ARCH__
    lo = a * b;
    hi = __umulhi(a, b);
#else
    uint64_t p = (uint64_t)a * b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

SILVAN_HD uint32_t philox_lo32(uint64_t seed, uint32_t sample, uint32_t kind, uint32_t draw,
                               uint32_t *hi32 = nullptr) {
    uint32_t c0 = draw, c1 = sample, c2 = kind, c3 = 0u;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t hi0, lo0, hi1, lo1;
        philox_mulhilo(0xD2511F53u, c0, hi0, lo0);
        philox_mulhilo(0xCD9E8D57u, c2, hi1, lo1);
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    if (hi32) *hi32 = c1;
    return c0;
}

// 25 Rademacher signs of one committed sample as a bit mask (bit j set = +1):
// sigma_j = (get_max(10^8) >= 5*10^7) * 2 - 1 (Probabilistic.cpp:488-493).
constexpr int kTrials = 25;  // mctrials (silvan/include/Probabilistic.h:89)

SILVAN_HD uint32_t rademacher_mask(uint64_t seed, uint32_t sample) {
    uint32_t m = 0;
    for (int j = 0; j < kTrials; j++) {
        uint32_t r = philox_lo32(seed, sample, kStreamRademacher, (uint32_t)j) % 100000000u;
        if (r >= 50000000u) m |= 1u << j;
    }
    return m;
}

// ---------------------------------------------------------------------------
// Per-slot node record of a sample in flight: one 32-byte sector per node so
// that a visited-state probe brings every field of the node into L2 at once.
// All records of a slot are "neutral" between samples; a sample restores the
// records of its ball before it finishes.
// ---------------------------------------------------------------------------
struct __align__(32) NodeRec {
    uint32_t st;     // 0 = unvisited, else side << 30 | distance from its root
    uint32_t cnt;    // number of predecessors (hits from the previous level)
    uint64_t sigma;  // shortest-path count from the root, wrapping (n_paths)
    uint64_t first;  // min over hits of (item << 32 | pred): the joining hit
    uint64_t last;   // max over hits of (item << 32 | pred): the last pred
};
static_assert(sizeof(NodeRec) == 32, "NodeRec must be one sector");

constexpr uint32_t kSideU = 1u, kSideV = 2u;
constexpr uint32_t kDistMask = (1u << 30) - 1;
SILVAN_HD uint32_t st_make(uint32_t side, uint32_t dist) { return (side << 30) | dist; }
SILVAN_HD uint32_t st_side(uint32_t st) { return st >> 30; }
SILVAN_HD uint32_t st_dist(uint32_t st) { return st & kDistMask; }

// One committed-sample contribution: the path map entry (node, count) of the
// sample with round-local index `sample`.
struct PathRec {
    uint32_t node;
    uint32_t sample;
    uint32_t count;
};

}  // namespace silvan
