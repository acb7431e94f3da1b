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
// SegDesc::assist_items value for the default threshold: levels of at least
// 32 tiles of the launch's CTA size while the round has samples left, 16
// tiles once it is drained
constexpr uint32_t kAssistItemsAuto = 0xffffffffu;

// One job's share of a sampler launch: samples [first_sample, first_sample +
// count) of that job's graph, written to that job's round buffers.
struct SegDesc {
    const uint32_t *out_off;
    const uint32_t *out_adj;
    const uint32_t *in_off;   // alias out_* when undirected
    const uint32_t *in_adj;
    const uint32_t *cc;
    const uint2 *out_rows;  // (start, end) of each row; alias when undirected
    const uint2 *in_rows;
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
    // BFS levels of at least this many adjacency entries are posted on the
    // launch's help board (0 = never, kAssistItemsAuto = the default threshold)
    uint32_t assist_items;
    uint32_t pad;
};

// Launch-invariant description of a sampler round; the segments live in
// device memory so that the launch can be captured in a CUDA graph once and
// replayed with new segments.
struct RoundHeader {
    uint32_t nsegs;
    uint32_t total;     // samples over all segments
    uint32_t work;      // next work index (zeroed by round_begin)
    uint32_t finished;  // samples completed (zeroed by round_begin)
    unsigned long long cycles;      // SM cycles spent in samples (zeroed by round_begin)
    unsigned long long max_cycles;  // cycles of the slowest sample (zeroed by round_begin)
    uint32_t open_mask;     // help-board entries with tiles left (zeroed by round_begin)
    uint32_t assisted;      // levels expanded with help (zeroed by round_begin)
    uint32_t helper_tiles;  // tiles of those levels done by helpers (zeroed by round_begin)
    // samples whose shared level gave up a wait (zeroed by round_begin); the
    // CTA of such a sample leaves the launch, because helpers may still write
    // to its slot, and the host re-initialises every slot after the launch
    uint32_t failed;
    uint32_t wait_polls;  // polls of each bounded help-board wait (set by the host)
    uint32_t pad;
};

// Polls of a bounded help-board wait unless the caller asks otherwise
// (silvan_params_t::wait_polls): at >= 64 ns per poll well above any real
// wait, which ends within microseconds.
constexpr uint32_t kDefaultWaitPolls = 1u << 20;

// Help board of a launch.  A CTA whose sample reaches a wide BFS level posts
// it on a free entry; CTAs between two samples, and CTAs left without samples
// at the end of the round, join the entry and take tiles of the level in
// order from its counter until every tile is taken.  Entries persist across
// launches; every use leaves its entry free again.
constexpr uint32_t kAssistEntries = 8;

// The level an entry describes (written by its owner before it opens).
struct AssistLevel {
    uint32_t ntiles, items, nodes, lo;
    uint32_t new_st, side, qbase, mbase;
    const uint2 *rows;    // (start, end) of the rows in the expansion direction
    const uint32_t *adj;
    NodeRec *rec;         // the owner's slot
    uint32_t *queue;
    uint2 *meet;
};

struct AssistEntry {
    uint32_t state;    // generation << 2 | phase (0 free, 1 set-up, 2 open, 3 closing)
    uint32_t inside;   // helpers between their entry and their exit
    uint32_t claim;    // next tile
    uint32_t done;     // finished tiles
    uint32_t ntiles;   // tiles of the open level
    uint32_t hits;     // new-level hits (predecessor entries), summed by the tiles
    uint32_t sum_new;  // degree sum of the joined nodes (wrapping), summed by the tiles
    uint32_t joins;    // joined nodes, summed by the tiles
    uint32_t meets;    // meeting edges (saturating), summed by the tiles
    uint32_t err;      // a tile gave up a wait
    AssistLevel lvl;
};

struct AssistBoard {
    AssistEntry *entries;  // kAssistEntries (nullptr: no board, nobody helps)
    uint32_t *pre;         // per entry node_cap + 1: item prefix of the frontier
    uint32_t *rs;          // per entry node_cap: row start of each frontier node
    uint4 *tiles;          // per entry tile_cap: first node, nodes, first item, end item
    uint32_t *hit_flag;    // per entry tile_cap: 1 tile's hits done, 2 those of all tiles <= it
    unsigned long long *cnt_flag;  // per entry tile_cap: look-back words of the append offsets
    uint32_t node_cap;
    uint32_t tile_cap;
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
    AssistBoard assist;  // zero: every level is expanded by its own CTA
};

// Neutral records for `slots` slots of n nodes.
cudaError_t sampler_init_slots(NodeRec *rec, uint32_t *hits, uint64_t total_nodes,
                               cudaStream_t stream);

// Device bytes of a help board for graphs of up to n nodes.
uint64_t assist_board_bytes(uint64_t n);
// Carves a board out of `mem` (assist_board_bytes(n) bytes) and frees its
// entries.
cudaError_t assist_board_init(AssistBoard *b, void *mem, uint64_t n, cudaStream_t stream);

// Zeroes the work counter and every segment's record cursor.
cudaError_t sampler_round_begin(const SamplerLaunch &L, uint32_t max_segs, cudaStream_t stream);
// Runs the round with `grid` resident CTAs of `block` threads (one of
// kSamplerBlocks; persistent, work-stealing).
cudaError_t sampler_launch(const SamplerLaunch &L, uint32_t grid, cudaStream_t stream,
                           int block = kSamplerBlock);

// Resident CTAs per SM of the `block`-thread sampler (0 for other sizes).
int sampler_max_ctas_per_sm(int block = kSamplerBlock);

}  // namespace silvan
