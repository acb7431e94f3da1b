// Device s-t shortest-path sampler: the balanced bidirectional BFS, meeting
// edge pick and random backtrack of silvan/src/Sp_sampler.cpp:41-265, one
// sample per CTA slot.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace silvan {

constexpr int kSamplerBlock = 512;   // threads per slot
constexpr uint32_t kMeetCap = 1u << 16;  // meeting edges per sample

struct SamplerArgs {
    // graph, CSR with 32-bit offsets; in_* alias out_* when undirected
    const uint32_t *out_off;
    const uint32_t *out_adj;
    const uint32_t *in_off;
    const uint32_t *in_adj;
    const uint32_t *cc;
    uint32_t n;
    int directed;
    // per-slot state, slot s owns [s*n, (s+1)*n) of each array
    NodeRec *rec;
    uint32_t *queue;
    uint32_t *hits;
    uint32_t *touched;
    uint2 *meet;        // slot s owns [s*kMeetCap, (s+1)*kMeetCap)
    uint64_t *meet_pre;
    // work: round-local samples [0, count) are global [first_sample, ...)
    uint64_t seed;
    uint32_t first_sample;
    uint32_t count;
    double alpha;
    uint32_t np_cap;
    uint32_t *work_counter;  // next round-local sample (device, zeroed per round)
    // per-sample outputs, round-local index
    int32_t *out_pl;
    int32_t *out_np;
    uint64_t *out_vis;
    int32_t *out_status;
    uint32_t *out_ball;   // nodes visited (both balls)
    uint32_t *out_pred;   // predecessor entries (hits on new-level nodes)
    // path-map records of the round
    PathRec *recs;
    unsigned long long *rec_cursor;
    uint64_t rec_cap;
};

// Neutral records for `slots` slots of n nodes.
cudaError_t sampler_init_slots(NodeRec *rec, uint32_t *hits, uint64_t total_nodes,
                               cudaStream_t stream);

// Runs the round with `grid` resident CTAs (persistent, work-stealing).
cudaError_t sampler_launch(const SamplerArgs &a, uint32_t grid, cudaStream_t stream);

// Function attributes for the occupancy-based slot choice.
int sampler_max_ctas_per_sm();

}  // namespace silvan
