// Test infrastructure (oracle): a replacement implementation of the
// reference's Rand_gen class (interface silvan/include/Rand_gen.h:6-18) that
// is linked, instead of silvan/src/Rand_gen.cpp, into the reference build
// under oracle/_ref.  The reference's own sampler, graph and estimator sources
// are compiled unmodified around it, so the reference code itself becomes a
// replay oracle for the GPU sampler.
//
// The MMIX LCG of silvan/src/Rand_gen.cpp:15-19 is sequential per OpenMP
// thread; here each draw is Philox4x32-10 of (job seed; draw index, global
// sample index, stream kind).  The per-instance state lives in the single
// `seed` word the reference header declares:
//   bit 63      stream kind (1 = the Rademacher generator the reference
//               constructs with seed 2021 at silvan/src/Probabilistic.cpp:71,
//               0 = every Sp_sampler generator)
//   bits 32..62 (sample index + 1) of the sample the draw counter belongs to
//   bits 0..31  draw counter within that sample
// The global sample index is set by the harness before every random_path
// call (ref_harness.cpp wraps Sp_sampler::random_path at link time).
#include <cstdint>
#include "Rand_gen.h"
#include "oracle_philox.h"

extern "C" {
uint64_t ref_job_seed = 42;        // Philox key of the job
uint32_t ref_sample_index = 0;     // global index of the sample being drawn
int ref_rng_zero_modulus = 0;      // set when get_max(0) is requested
}

Rand_gen::Rand_gen(uint64_t seed) {
    this->seed = (seed == 2021 ? (1ull << 63) : 0ull);
}

Rand_gen::~Rand_gen() {}

uint64_t Rand_gen::get() {
    const uint64_t kind = seed >> 63;
    const uint32_t want_tag = (ref_sample_index + 1u) & 0x7FFFFFFFu;
    uint32_t tag = (uint32_t)((seed >> 32) & 0x7FFFFFFFu);
    uint32_t draw = (uint32_t)seed;
    if (tag != want_tag) {
        tag = want_tag;
        draw = 0;
    }
    seed = (kind << 63) | ((uint64_t)tag << 32) | (uint64_t)(draw + 1u);
    return oracle_draw(ref_job_seed, ref_sample_index, (uint32_t)kind, draw);
}

// silvan/src/Rand_gen.cpp:22-24: the draw is truncated to 32 bits, so the
// rejection loop there never repeats; the result is (uint32_t)get() % m.
// The reference divides by zero when m == 0 (a wrapped path count); the
// oracle records the event and returns 0 instead of trapping.
uint64_t Rand_gen::get_max(uint64_t m) {
    uint32_t r = (uint32_t)get();
    if (m == 0) {
        ref_rng_zero_modulus = 1;
        return 0;
    }
    return r % m;
}
