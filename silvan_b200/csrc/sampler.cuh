// Device s-t shortest-path sampler: the balanced bidirectional BFS, meeting
// edge pick and random backtrack of silvan/src/Sp_sampler.cpp:41-265, one
// sample per CTA slot.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace silvan {

constexpr int kSamplerBlock = 512;   // default threads per slot
constexpr int kSamplerBlocks[4] = {128, 256, 512, 1024};  // compiled CTA sizes
constexpr uint32_t kMeetCap = 1u << 16;  // meeting edges per sample

// One job's share of a sampler launch: samples [first_sample, first_sample +
// count) of that job's graph, written to that job's round buffers.
struct SegDesc {
    const uint32_t *out_off;
    const uint32_t *out_adj;
    const uint32_t *in_off;   // alias out_* when undirected
    const uint32_t *in_adj;
    const uint32_t *cc;
    uint32_t n;
    int32_t directed;
    uint64_t seed;
    double alpha;
    uint32_t np_cap;
    uint32_t first_sample;  // global index of the segment's sample 0
    uint32_t count;
    uint32_t base;          // work index of the segment's sample 0 (prefix over segments)
    int32_t weighted;       // sigma-weighted backtrack (SILVAN_BACKTRACK_SIGMA_WEIGHTED)
    // per-sample outputs, segment-local index
    int32_t *out_pl;
    int32_t *out_np;
    uint64_t *out_vis;
    int32_t *out_status;
    uint32_t *out_ball;   // nodes visited (both balls)
    uint32_t *out_pred;   // predecessor entries (hits on new-level nodes)
    // path-map records of the segment, sample field = segment-local index
    PathRec *recs;
    unsigned long long *rec_cursor;
    uint64_t rec_cap;
};

// Launch-invariant description of a sampler round; the segments live in
// device memory so that the launch can be captured in a CUDA graph once and
// replayed with new segments.
struct RoundHeader {
    uint32_t nsegs;
    uint32_t total;   // samples over all segments
    uint32_t work;    // next work index (zeroed by round_begin)
    uint32_t pad;
    unsigned long long cycles;      // SM cycles spent in samples (zeroed by round_begin)
    unsigned long long max_cycles;  // cycles of the slowest sample (zeroed by round_begin)
};

struct SlotArrays {
    NodeRec *rec;
    uint32_t *queue;
    uint32_t *hits;
    uint32_t *touched;
    uint2 *meet;        // slot s owns [s*kMeetCap, (s+1)*kMeetCap)
    uint64_t *meet_pre;
    uint64_t stride;    // nodes per slot (largest graph served)
};

struct SamplerLaunch {
    SlotArrays slots;
    RoundHeader *hdr;
    const SegDesc *segs;
};

// Neutral records for `slots` slots of n nodes.
cudaError_t sampler_init_slots(NodeRec *rec, uint32_t *hits, uint64_t total_nodes,
                               cudaStream_t stream);

// Zeroes the work counter and every segment's record cursor.
cudaError_t sampler_round_begin(const SamplerLaunch &L, uint32_t max_segs, cudaStream_t stream);
// Runs the round with `grid` resident CTAs of `block` threads (one of
// kSamplerBlocks; persistent, work-stealing).
cudaError_t sampler_launch(const SamplerLaunch &L, uint32_t grid, cudaStream_t stream,
                           int block = kSamplerBlock);

// Resident CTAs per SM of the `block`-thread sampler (0 for other sizes).
int sampler_max_ctas_per_sm(int block = kSamplerBlock);

}  // namespace silvan
