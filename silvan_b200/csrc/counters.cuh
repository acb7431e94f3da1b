// Device counters of a job and the kernels that commit a round of samples to
// them in the reference's sequential order (silvan/src/Probabilistic.cpp:
// 468-559), reduce them for the stopping rule (:251-414) and partition the
// nodes by empirical peeling (:853-871).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace silvan {

constexpr uint32_t kLargeBucket = 8192;  // samples per apply sub-round (bucket bound)
constexpr int kMaxPartitions = 128;

// Job-level scalars kept on the device.
struct JobScalars {
    unsigned long long sup_approx_bits;  // max approx (non-negative doubles as bits)
    unsigned long long sup_wimpy_bits;   // max emp_wimpy_vars
    unsigned long long vis_edges;
    unsigned long long void_samples;
    unsigned long long counted_samples;
    unsigned long long paths;            // sum of num_paths over counted samples
    unsigned long long ball_nodes;       // nodes visited by the samplers
    unsigned long long pred_entries;     // predecessor entries recorded
    int32_t error;                       // first SILVAN_E_* seen
    uint32_t n_cross;                    // crossings of the top-k "approx >= 3" mark
    uint32_t n_upd;                      // entries of upd_list
    uint32_t pad;
};

static_assert(sizeof(JobScalars) % 8 == 0, "JobScalars is copied in 8-byte words");

struct RoundBuffers {
    // per round-local sample
    int32_t *pl;
    int32_t *np;
    uint64_t *vis;
    int32_t *status;
    uint32_t *signs;
    uint32_t *ball;
    uint32_t *pred;
    double *inv_np;  // 1 / num_paths of each sample (set by the commit)
    uint32_t max_samples;
    // path-map records
    PathRec *recs;
    unsigned long long *rec_cursor;
    uint64_t rec_cap;
    // bucketing by node
    uint32_t *node_cnt;      // n, zero between rounds
    uint32_t *touched;       // distinct nodes of the round
    // control words of the commit rounds (zero when allocated; each round
    // leaves them as it found them): [0] touched nodes, [1] large buckets,
    // [2..3] grid barrier, [4] bucket-space cursor, [5] large-bucket claims,
    // [6] CTAs done; [7] touched nodes of the last round (read by undo_round)
    uint32_t *n_touched;
    uint32_t *bucket_off;    // start of each touched node's bucket
    uint32_t *bucket_len;    // its number of entries
    uint32_t *large;         // buckets of more than 32 entries (listed by bucket_alloc)
    uint32_t *n_large;       // = n_touched + 1 (both zeroed together)
    unsigned long long *entries;  // sample << 32 | count, grouped by node
    uint32_t *work_counter;  // sampler work counter
};

struct JobCounters {
    double *approx;
    double *wimpy;
    long long *mcrade;    // n x 25, node-major
    uint32_t *last_upd;   // 1 + global index of the last sample that updated the node
    uint8_t *cross_flag;  // approx_toadd of the reference (top-k pass 1)
    uint32_t *cross_sample;  // global sample index of each crossing
    uint64_t *sp_lengths;    // D + 1
    JobScalars *sc;
    int32_t *partition;   // dense partition id per node
    int32_t *peel_idx;    // raw peeling index per node
    uint32_t *upd_list;   // nodes updated since the counters were last reset
};

struct ApplyArgs {
    uint32_t n;
    uint32_t n_records;      // path-map records of the round
    uint64_t seed;
    uint32_t first_sample;   // global index of round-local sample 0
    uint32_t lo, hi;         // round-local sample range committed by this call
    int32_t pass;            // 1 or 2 (pass 2 updates mcrade)
    int32_t track_cross;     // pass 1 of top-k mode
    uint32_t D;
    int32_t journal;         // save what the round changes (RoundJournal) so it can be undone
};

// What a journaled commit round overwrites: the old counters of each node it
// folds (indexed by the node's position on the round's touched list), the
// job's scalars and the shortest-path length counts.  undo_round puts them
// back, which leaves the counters as they were before the round.  Sized for
// every node of the graph (a round touches each node at most once).
struct RoundJournal {
    long long *mcrade;     // n x 25 (pass 2 only)
    double *approx;        // n
    double *wimpy;         // n
    uint32_t *last_upd;    // n
    JobScalars *sc;        // 1
    uint64_t *sp_lengths;  // D + 1
};

// Everything a commit round reads, passed to its kernel by value.
struct ApplyState {
    RoundBuffers rb;
    JobCounters jc;
    RoundJournal jr;
    ApplyArgs a;
};

// Kernels apply_round launches: one cooperative kernel.
constexpr int kApplyRoundKernels = 1;

// Commits round-local samples [a.lo, a.hi) of the round buffers to the job
// counters: one cooperative kernel whose phases are separated by grid-wide
// barriers, with st as its argument.
cudaError_t apply_round(const ApplyState &st, cudaStream_t stream);
// Function attributes and resident grid of the commit kernel on the current
// device (call before capturing).
cudaError_t apply_init();
// Restores what the last commit round (journaled, and the last round on
// rb) changed: the nodes of rb's touched list, the scalars, the path-length
// counts.
cudaError_t undo_round(const RoundBuffers &rb, const JobCounters &jc, const RoundJournal &jr,
                       int pass, uint32_t D, cudaStream_t stream);

// Reduction for one stopping-rule evaluation: per partition and trial the
// maximum of mcrade (LLONG_MIN when no node of the partition was updated;
// the host takes the larger of it and -n_pairs), per partition the maximum
// of emp_wimpy_vars, and the global maxima of approx and emp_wimpy_vars.
// Only the nodes on upd_list are read: every other node still has
// approx = wimpy = mcrade = 0, which the host folds in per partition from
// touched[] (a partition with fewer touched nodes than members has zeros).
struct StopReduction {
    long long mc_max[kMaxPartitions * kTrials];
    double wimpy_max[kMaxPartitions];
    uint32_t touched[kMaxPartitions];
    double approx_max;
    double wimpy_all_max;
};
// out[v] = approx[v] / num_samples (the estimates the reference prints).
cudaError_t divide_estimates(const double *approx, double num_samples, double *out, uint32_t n,
                             cudaStream_t stream);

// Where a check's results land (host-mapped memory, read after the kernel):
// the reduction, the job's scalars, the D + 1 path-length counts (sp may be
// null).
struct StopReadback {
    StopReduction *red;
    JobScalars *sc;
    uint64_t *sp;
};
// The device accumulator of stop_reduce and its CTA ticket, made neutral once
// (stop_reduce leaves them neutral).
cudaError_t stop_reduce_init(StopReduction *acc, uint32_t *ticket, cudaStream_t stream);
// One kernel: the reduction over upd_list plus the scalars and path-length
// counts, written to `out`.
cudaError_t stop_reduce(const JobCounters &jc, int nparts, uint32_t D, StopReduction *acc,
                        uint32_t *ticket, const StopReadback &out, cudaStream_t stream);

cudaError_t peel_map(const JobCounters &jc, uint32_t n, const int32_t *lut, int32_t idx_min,
                     int32_t lut_size, uint32_t *hist, cudaStream_t stream);
cudaError_t peel_hist(const JobCounters &jc, uint32_t n, int32_t idx_min, int32_t nbins,
                      uint32_t *hist, cudaStream_t stream);
constexpr int32_t kPeelLocalBins = 8192;  // histograms up to this size are built in shared memory

// Where the end-of-pass-1 read lands (host-mapped memory).
struct Pass1Readback {
    JobScalars *sc;
    uint64_t *sp;      // D + 1 path-length counts
    uint32_t *hist;    // nbins peeling-index counts
    uint32_t *n_unc;   // uncertain indices listed
};
// One kernel: when nbins > 0, every node's peeling index
// (Probabilistic.cpp:855-862), the nodes whose index lies within rounding
// distance of a boundary (listed so that the host recomputes them with the C
// library's log) and the histogram of the indices (hist and n_uncertain are
// zeroed here); then the histogram, the uncertain count, the scalars and the
// path-length counts copied to `out`.  ticket is a zero word that the kernel
// leaves zero.
cudaError_t pass1_readback(const JobCounters &jc, uint32_t n, double num_samples, double a,
                           int32_t idx_min, int32_t nbins, uint32_t *hist, uint32_t *uncertain,
                           uint32_t *n_uncertain, uint32_t cap, uint32_t D, uint32_t *ticket,
                           const Pass1Readback &out, cudaStream_t stream);
// approx, wimpy and last_upd back to zero on the nodes of upd_list.
cudaError_t reset_updated(const JobCounters &jc, cudaStream_t stream);

// Ranking of the top-k mode (the reference's Ranking_list,
// silvan/src/Ranking_list.cpp:20-43, as Probabilistic.cpp:587-687 reads it):
// nodes ordered by (approx desc, last update desc, node desc) -- a node that
// reaches a value later is put before the nodes that reached it earlier, and
// within one sample the larger id is the later update -- with the
// never-updated nodes after all updated ones in ascending id.
//
// topk_select finds the K best updated nodes on the device: the 128-bit keys
// (approx bits, last update << 32 | node) of the updated nodes (upd_list) are
// radix-selected 16 bits at a time (a histogram per level; a level is refined
// only while its boundary group is too large), the candidates are compacted
// and sorted by one CTA in shared memory (or on the host when K is larger than
// that CTA's buffer), so only the K winners cross to the host.
struct TopkBuffers {
    uint32_t *hist = nullptr;            // 65536 bins
    uint32_t *state = nullptr;           // device selection state (8 words)
    unsigned long long *cand = nullptr;  // 2 x cap words: keys (hi, lo)
    uint32_t cap = 0;                    // candidate capacity
    uint32_t *h_state = nullptr;         // pinned copy of state
    unsigned long long *h_cand = nullptr;  // pinned, 2 x cap words
};
// Candidate capacity for a selection of K.
uint32_t topk_capacity(uint32_t K);
// The K best updated nodes (fewer when fewer were updated), best first, with
// their approx values.  n_upd is the number of entries of jc.upd_list.
int topk_select(const JobCounters &jc, uint32_t n_upd, uint32_t K, const TopkBuffers &tb,
                cudaStream_t stream, uint32_t *nodes, double *values, uint32_t *count);

}  // namespace silvan
