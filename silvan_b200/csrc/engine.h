// Host engine: device graph, sampler engine and the estimator state machine.
//
// An Engine owns sampler slots sized for the largest graph it serves and runs
// sampler rounds over any number of jobs at once (one persistent launch whose
// work is the concatenation of every job's request).  A Job owns its counters
// and round buffers and restates Probabilistic::run
// (silvan/src/Probabilistic.cpp:775-1139) as a state machine: it asks for the
// next range of samples, and after the engine has drawn them it commits them
// and evaluates the schedule events the reference evaluates at each point.
#pragma once
#include <array>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <deque>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "counters.cuh"
#include "graph_host.h"
#include "sampler.cuh"
#include "silvan.h"

namespace silvan {

void set_error(const std::string &msg);
const char *last_error_cstr();  // this thread's last message
int cuda_status(cudaError_t e, const char *what);
double now_seconds();

// Device memory from the library's caching allocator: freed blocks are kept
// per device and size class and handed out again.  Every device buffer that a
// DeviceGraph, Engine or Job frees must come from here.
int device_alloc(void **p, size_t bytes);
void device_free(void *p);

// Serialises CUDA-graph captures with whole-device synchronisations and
// allocations made by other threads.
std::mutex &capture_mutex();

struct DeviceGraph {
    // metadata (always set once uploaded)
    uint32_t n = 0;
    bool directed = false;
    uint64_t m = 0;     // out-edge entries (edges_num of the reference)
    uint64_t m_in = 0;  // in-edge entries (directed graphs)
    // host copy, kept when the graph was built on the host (file or pairs)
    bool has_host = false;
    HostGraph host;
    std::vector<uint32_t> cc;
    uint32_t ncomp = 0;
    uint32_t diameter = 0;
    double diameter_seconds = 0;
    // device CSR, 32-bit offsets; in_* alias out_* for undirected graphs
    uint32_t *d_out_off = nullptr, *d_out_adj = nullptr;
    uint32_t *d_in_off = nullptr, *d_in_adj = nullptr;
    uint32_t *d_cc = nullptr;
    // (start, end) of every row, for the sampler: in_rows aliases out_rows
    // for undirected graphs
    uint2 *d_out_rows = nullptr, *d_in_rows = nullptr;
    int device = 0;
    // Class of the graph for the sampler's schedule statistics: graphs with
    // the same direction, node count and mean degree (both to a power of 2)
    // share them, so a stream of fresh graphs of a few shapes is tuned once.
    uint64_t tune_class() const;

    int upload();  // from `host` and `cc`
    // from caller-owned host arrays (ideally pinned): copied straight to the
    // device, offsets narrowed and rows validated there
    int upload_raw(uint32_t n, bool directed, const uint64_t *out_off, const uint32_t *out_adj,
                   const uint64_t *in_off, const uint32_t *in_adj, const uint32_t *cc);
    uint64_t device_bytes() const;
    // d_out_rows / d_in_rows from the device offsets (every upload path ends
    // with it)
    int make_rows(cudaStream_t stream);
    // Components and diameter bound on the host copy, then the component
    // ids to the device (after a device ingest filled d_* and `host`).
    int finish_from_host_copy();
    ~DeviceGraph();
};

// Per-slot sampler state.
struct SlotPool {
    uint32_t slots = 0;
    uint64_t n = 0;
    NodeRec *rec = nullptr;
    uint32_t *queue = nullptr, *hits = nullptr, *touched = nullptr;
    uint2 *meet = nullptr;
    uint64_t *meet_pre = nullptr;
    int alloc(uint32_t slots, uint64_t n, cudaStream_t s);
    void free_all();
    static uint64_t bytes_per_slot(uint64_t n);
    ~SlotPool() { free_all(); }
};

struct JobRequest {
    uint32_t first_global = 0;  // global sample index of the range's first sample
    uint32_t count = 0;
    int pass = 1;
    bool track_cross = false;
    double alpha = 0;           // multi-path rate the range is drawn with
};

class Job;
class Engine;

// Process-wide pool of sampler engines per device: a job borrows one for its
// run, so repeated jobs do not re-allocate and re-initialise the slots.
Engine *engine_acquire(uint64_t n, uint32_t slots, int *rc);
void engine_release(Engine *e);

class Engine {
  public:
    ~Engine();
    // slots = 0 picks occupancy x SM count, capped by `mem_budget` bytes
    // (0 = half of the free device memory)
    int init(uint64_t n_max, uint32_t slots, uint64_t mem_budget);
    bool ready() const { return slots_.slots > 0; }
    uint64_t n_max() const { return slots_.n; }
    uint32_t slots() const { return slots_.slots; }
    cudaStream_t stream() const { return stream_; }
    // Draws every job's requested range in one persistent launch into the
    // jobs' round buffers; the jobs commit them.  Grows a job's record buffer
    // and redraws the round when the path maps did not fit.  `records`
    // receives the number of path-map records of each job.
    int round(const std::vector<Job *> &jobs, const std::vector<JobRequest> &reqs,
              std::vector<uint64_t> &records);
    // samples that one more launch could draw for free: a launch lasts at
    // least as long as its slowest sample, during which the other slots keep
    // drawing (0 until a launch has been measured)
    // measured on the last launch that drew samples of G's class of graphs
    uint32_t free_samples(const DeviceGraph *G, bool tail_only) const;
    // Samples (both passes) the last single-job run on G's class of graphs
    // used, when its second pass kept alpha (0: none recorded)
    uint64_t job_hint(const DeviceGraph *G) const;
    void note_job(const DeviceGraph *G, uint64_t used, bool alpha_kept);
    uint64_t launches() const { return launches_; }
    float sample_ms() const { return sample_ms_; }
    void reset_timers() {
        sample_ms_ = 0;
        launches_ = 0;
        sampler_launches_ = 0;
        assisted_levels_ = 0;
        helper_tiles_ = 0;
        block_samples_.fill(0);
    }
    uint32_t sampler_launches() const { return sampler_launches_; }
    uint32_t assisted_levels() const { return assisted_levels_; }
    uint64_t helper_tiles() const { return helper_tiles_; }
    // times every slot was re-initialised after a shared level gave up a wait
    uint32_t slot_resets() const { return slot_resets_; }
    // Shortens the requests of a multi-job round so that the round's
    // predicted CTA time fits `round_ms` on the resident slots: jobs that
    // need little get all of it, the rest share what is left evenly (every
    // job still draws at least one 11-sample block).  Without statistics for
    // every job's graph class the requests stay as they are.
    void fair_share(const std::vector<Job *> &jobs, std::vector<JobRequest> &reqs,
                    double round_ms) const;
    // CTA size that drew the most samples since reset_timers()
    uint32_t main_block() const;

  private:
    static constexpr int kNB = 4;  // compiled CTA sizes (kSamplerBlocks)
    // Measured cost of one graph's samples under each CTA size: CTA time
    // per sample (throughput) and the slowest sample of a round (its tail).
    struct BlockStats {
        double cta_ms = 0, tail_ms = 0;
        uint32_t rounds = 0;
    };
    struct Exec {
        int block;
        uint32_t grid;
        cudaGraphExec_t exec;
    };
    int ensure_segs(uint32_t nsegs);
    int choose_block(const std::vector<Job *> &jobs, const std::vector<JobRequest> &reqs,
                     const std::vector<uint32_t> &idx, uint32_t total) const;
    int sampler_exec(int block, uint32_t grid, cudaGraphExec_t *out);
    void drop_execs();
    SlotPool slots_;
    void *board_mem_ = nullptr;  // help board of the sampler launches
    AssistBoard board_{};
    cudaStream_t stream_ = nullptr;
    RoundHeader *d_hdr_ = nullptr, *h_hdr_ = nullptr;
    SegDesc *d_segs_ = nullptr, *h_segs_ = nullptr;
    unsigned long long *d_cursors_ = nullptr, *h_cursors_ = nullptr;
    uint32_t max_segs_ = 0;
    std::vector<Exec> execs_;          // captured round_begin + sampler per (block, grid)
    uint32_t max_grid_[kNB] = {};      // resident CTAs per CTA size (0 = unusable)
    std::unordered_map<uint64_t, std::array<BlockStats, kNB>> stats_;  // by tune_class()
    std::array<uint64_t, kNB> block_samples_{};
    uint32_t sampler_launches_ = 0;
    uint32_t assisted_levels_ = 0;  // BFS levels expanded with the help board
    uint64_t helper_tiles_ = 0;     // tiles of those levels done by helping CTAs
    uint32_t slot_resets_ = 0;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    float sample_ms_ = 0;
    uint64_t launches_ = 0;
    double clock_khz_ = 0;
    struct LastLaunch {
        double cta_ms = 0;     // CTA ms per sample
        double tail_ms = 0;    // the slowest sample
        double launch_ms = 0;
        uint32_t grid = 0;
        uint32_t samples = 0;  // drawn by the launch
    };
    std::unordered_map<uint64_t, LastLaunch> last_;  // by tune_class()
    // by tune_class(): the samples of the last kHintJobs jobs (see job_hint)
    std::unordered_map<uint64_t, std::deque<uint64_t>> job_total_;
    static constexpr size_t kHintJobs = 8, kHintMin = 4;
};

class Job {
  public:
    Job(DeviceGraph *g, const silvan_params_t &p) : g_(g), p_(p) {}
    ~Job();
    int init();  // counters and round buffers; no sampler slots
    uint64_t device_bytes() const;

    // single-job run on an engine of its own (created on first use)
    int run(silvan_result_t *res, FILE *sink);
    // at most `rounds` rounds of the job's schedule on its own engine
    int step(uint32_t rounds, silvan_status_t *st, FILE *sink);

    // ---- state machine used by Engine::round drivers -------------------------
    int begin(FILE *sink, cudaStream_t stream);
    bool done() const { return phase_ == kDone; }
    bool next_request(JobRequest &r);
    // after the engine drew the requested range: commits it schedule point by
    // schedule point and evaluates each point
    int on_drawn(const JobRequest &r, uint64_t n_records);
    // speculative draw sizes: within the slowest sample's time (first pass)
    // and within the last launch's time (second pass, capped by omega)
    void set_lookahead(uint32_t tail, uint32_t launch) {
        lookahead_tail_ = tail;
        lookahead_ = launch;
    }
    int finish(silvan_result_t *res);
    int error() const { return error_; }
    uint32_t nodes() const { return n_; }
    // forget the stream of an engine that is going away
    void detach() {
        if (stream_) cudaStreamSynchronize(stream_);
        stream_ = own_engine_ ? own_engine_->stream() : nullptr;
        sink_ = nullptr;
    }
    bool started() const { return phase_ != kInit; }

    // per-sample replay (parity hook): raw sampler output of [first, first+count)
    int replay(uint32_t first, uint32_t count, double alpha, std::vector<int32_t> &pl,
               std::vector<int32_t> &np, std::vector<uint64_t> &vis,
               std::vector<int32_t> &status, std::vector<PathRec> &recs);

    int read_estimates(double *out, uint32_t n);
    int read_counters(double *approx, double *wimpy, int64_t *mcrade, int32_t *part);
    int read_topk(uint32_t *nodes, double *values, uint32_t cap, uint32_t *count);

    // ---- used by Engine -------------------------------------------------------
    DeviceGraph *graph() const { return g_; }
    const silvan_params_t &params() const { return p_; }
    double alpha() const { return alpha_; }
    RoundBuffers &round_buffers() { return rb_; }
    int grow_records(uint64_t cap);
    uint64_t launches = 0;

  private:
    enum Phase { kInit, kPass1, kPass2, kDone };
    int alloc_round(uint32_t max_samples, uint64_t rec_cap);
    int apply_range(const JobRequest &r, uint32_t lo, uint32_t hi, uint64_t n_records,
                    bool journal = false);
    int evaluate();
    int speculate();
    int undo_speculation();
    int sync_scalars(JobScalars &sc);
    int read_sp_lengths(std::vector<uint64_t> &out);
    int peel(double a, bool enabled, std::vector<uint64_t> &sp);
    int finish_pass1();
    int stop_check(bool &stop);
    int stop_check_enqueue();
    int stop_check_finish(bool &stop);
    int scalars_error(const JobScalars &sc);
    int ranking(std::vector<uint32_t> &el, std::vector<double> &val);
    bool check_topk(std::string &out);
    void reset_pass2_counters();
    void flush();

    DeviceGraph *g_;
    silvan_params_t p_;
    Engine *own_engine_ = nullptr;  // borrowed from the pool while running
    int borrow_engine();
    void return_engine();
    cudaStream_t stream_ = nullptr;  // stream of the engine driving the job
    RoundBuffers rb_{};
    uint32_t n_ = 0;
    JobCounters jc_{};
    StopReduction *d_red_ = nullptr;  // the check kernel's accumulator (neutral between checks)
    uint32_t *d_ticket_ = nullptr;
    StopReadback readback_{};         // device view of h_red_, h_sc_, h_sp_
    StopReduction *h_red_ = nullptr;  // pinned
    JobScalars *h_sc_ = nullptr;      // pinned
    uint64_t *h_sp_ = nullptr;        // pinned, diameter + 1 shortest-path lengths
    uint32_t *d_unc_ = nullptr, *d_nunc_ = nullptr;
    int32_t *d_lut_ = nullptr;
    uint32_t *d_hist_ = nullptr;
    int32_t *h_lut_ = nullptr;    // pinned
    uint32_t *h_hist_ = nullptr;  // pinned, written by the end-of-pass-1 kernel
    uint32_t *h_nunc_ = nullptr;  // pinned, likewise
    uint32_t hist_cap_ = 0;
    TopkBuffers tk_{};  // top-k mode: device selection of the ranking
    // absolute mode, pass 2: the round after a check is committed (journaled)
    // while the host evaluates the check, and undone if the check stops the
    // run or moves the next schedule point
    RoundJournal jr_{};
    cudaEvent_t ev_chk_ = nullptr;  // the check's reads have landed
    struct Overlap {
        bool on = false;      // on_drawn is committing a drawn range
        JobRequest rc{};      // that range, as pass 2 commits it
        uint64_t g0 = 0, g1 = 0, n_records = 0;
        uint64_t spec_lo = 0, spec_hi = 0;  // pass samples of the journaled round (0, 0: none)
    } ov_;
    cudaEvent_t ev_run_[2] = {nullptr, nullptr};
    FILE *sink_ = nullptr;
    std::string out_;  // pending status lines

    // estimator state (members of Probabilistic, silvan/include/Probabilistic.h:59-110)
    Phase phase_ = kInit;
    int error_ = 0;
    bool absolute_ = true;
    bool peel_on_ = true;
    double peel_a_ = 2.0;
    uint32_t k_ = 0, union_sample_ = 0, tau_ = 0;
    uint64_t base_global_ = 0;   // global index of the pass's first sample
    uint32_t lookahead_ = 0;     // pass 2: samples drawn ahead of the next point
    uint32_t lookahead_tail_ = 0;  // pass 1 (absolute mode): samples drawn beyond it
    uint64_t hint_total_ = 0;      // samples the last job of this graph class used
    uint64_t predicted_stop_ = 0;  // pass 2 (absolute mode): sample size of the likely stop
    float commit_ms_ = 0;
    uint64_t drawn_ = 0;         // samples drawn over both passes
    cudaEvent_t ev_commit_[2] = {nullptr, nullptr};
    uint64_t pass_samples_ = 0;  // samples committed in the current pass
    uint64_t target_ = 0;        // sample count of the next schedule event
    uint64_t p1_chunk_ = 0;      // top-k pass 1: speculative chunk size
    bool p1_final_ = false;      // top-k pass 1: the stopping block is known
    double alpha_ = 2.3;
    int nparts_ = 1;
    std::vector<int> part_ids_;  // raw peeling index of each dense id
    std::vector<uint32_t> part_count_;
    std::vector<int32_t> part_host_;
    std::vector<double> eps_part_;
    double omega_ = 0, first_stop_ = 0, last_stop_ = 0, dfpb_ = 1.0;
    uint64_t next_stop_ = 0;
    int iteration_ = 0;
    double eps_final_topk_ = 1.0;
    uint32_t numresults_topk_ = 0;
    double eps_stop_ = -1;
    uint32_t checks_ = 0;
    uint32_t overlapped_checks_ = 0;
    double max_num_samples_ = 0;
    uint64_t p1_samples_ = 0;
    JobScalars sc1_{};
    int stop_reason_ = 0;
    double t_start_ = 0, t_first_ = 0, t2_start_ = 0;
    std::vector<uint32_t> final_rank_el_;
    std::vector<double> final_rank_val_;
    silvan_result_t result_{};
};

// Runs jobs to completion, one sampler launch per round for all unfinished
// jobs (multi-graph batching).
int run_batched(const std::vector<Job *> &jobs, uint64_t mem_budget, silvan_result_t *results,
                FILE *sink);

}  // namespace silvan
