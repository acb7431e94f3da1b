/* Test infrastructure (oracle): counter-based RNG used by the CPU oracle and
 * by the Rand_gen replacement that is linked into the reference build under
 * oracle/_ref.  It is never linked into the product library.
 *
 * Philox4x32-10 as published in Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3" (SC'11): 10 rounds of two 32x32->64 multiplies
 * with the round constants and Weyl key increments given in that paper.
 *
 * Stream convention shared with the GPU sampler (the replacement for the
 * 64-bit MMIX LCG of silvan/src/Rand_gen.cpp:15-25):
 *   key     = (job_seed low 32 bits, job_seed high 32 bits)
 *   counter = (draw index within the sample, global sample index,
 *              stream kind (0 = s-t sampler, 1 = Rademacher signs), 0)
 *   get()       = out[1] << 32 | out[0]
 *   get_max(m)  = (uint32_t)get() % m          (silvan/src/Rand_gen.cpp:22-24:
 *                 the reference keeps the low 32 bits of the draw)
 */
#ifndef SILVAN_ORACLE_PHILOX_H
#define SILVAN_ORACLE_PHILOX_H
#include <stdint.h>

static inline void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2],
                                        uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* One 64-bit draw of the stream (seed, sample, kind) at position draw. */
static inline uint64_t oracle_draw(uint64_t seed, uint32_t sample, uint32_t kind, uint32_t draw) {
    uint32_t ctr[4] = {draw, sample, kind, 0u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    oracle_philox4x32_10(ctr, key, out);
    return ((uint64_t)out[1] << 32) | out[0];
}

#endif
