// Host engine: device graph, job state and the estimator driver.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "counters.cuh"
#include "graph_host.h"
#include "sampler.cuh"
#include "silvan.h"

namespace silvan {

void set_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);

struct DeviceGraph {
    HostGraph host;
    std::vector<uint32_t> cc;
    uint32_t ncomp = 0;
    uint32_t diameter = 0;
    double diameter_seconds = 0;
    // device CSR, 32-bit offsets; in_* alias out_* for undirected graphs
    uint32_t *d_out_off = nullptr, *d_out_adj = nullptr;
    uint32_t *d_in_off = nullptr, *d_in_adj = nullptr;
    uint32_t *d_cc = nullptr;
    int device = 0;

    int upload();
    ~DeviceGraph();
};

// Per-slot sampler state plus per-round buffers.
struct SlotPool {
    uint32_t slots = 0, n = 0;
    NodeRec *rec = nullptr;
    uint32_t *queue = nullptr, *hits = nullptr, *touched = nullptr;
    uint2 *meet = nullptr;
    uint64_t *meet_pre = nullptr;
    int alloc(uint32_t slots, uint32_t n, cudaStream_t s);
    void free_all();
    ~SlotPool() { free_all(); }
};

struct RoundPool {
    RoundBuffers rb{};
    uint32_t n = 0;
    int alloc(uint32_t n, uint32_t max_samples, uint64_t rec_cap);
    int grow_records(uint64_t rec_cap);
    void free_all();
    ~RoundPool() { free_all(); }
};

class Job {
  public:
    Job(DeviceGraph *g, const silvan_params_t &p) : g_(g), p_(p) {}
    ~Job();
    int init();
    int run(silvan_result_t *res, FILE *sink);
    // step-wise: commit samples of the current pass up to `target`
    int run_to(uint64_t target, silvan_status_t *st);
    int read_estimates(double *out, uint32_t n);
    int read_counters(double *approx, double *wimpy, int64_t *mcrade, int32_t *part);
    int read_topk(uint32_t *nodes, double *values, uint32_t cap, uint32_t *count);

    // per-sample replay (parity hook): raw sampler output of [first, first+count)
    int replay(uint32_t first, uint32_t count, double alpha, std::vector<int32_t> &pl,
               std::vector<int32_t> &np, std::vector<uint64_t> &vis,
               std::vector<int32_t> &status, std::vector<PathRec> &recs);

  private:
    int sample_range(uint64_t lo, uint64_t hi, int pass, bool track_cross);
    int run_batch(uint32_t first_global, uint32_t count, int pass, bool track_cross);
    int sync_scalars(JobScalars &sc);
    int read_sp_lengths(std::vector<uint64_t> &out);
    int peel(double a, bool enabled);
    int stop_check(bool &stop, std::string &out);
    int ranking(std::vector<uint32_t> &el, std::vector<double> &val);
    bool check_topk(std::string &out);
    void reset_pass2_counters();

    DeviceGraph *g_;
    silvan_params_t p_;
    cudaStream_t stream_ = nullptr;
    SlotPool slots_;
    RoundPool round_;
    JobCounters jc_{};
    StopReduction *d_red_ = nullptr;
    StopReduction *h_red_ = nullptr;  // pinned
    JobScalars *h_sc_ = nullptr;      // pinned
    unsigned long long *h_cursor_ = nullptr;  // pinned
    uint32_t *d_unc_ = nullptr, *d_nunc_ = nullptr;
    int32_t *d_lut_ = nullptr;
    uint32_t *d_hist_ = nullptr;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_run_[2] = {nullptr, nullptr};
    uint64_t launches_ = 0;

    // estimator state (members of Probabilistic, silvan/include/Probabilistic.h:59-110)
    bool absolute_ = true;
    uint32_t k_ = 0, union_sample_ = 0, tau_ = 0;
    uint64_t global_next_ = 0;  // global index of the next sample
    uint64_t pass_samples_ = 0; // samples committed in the current pass
    int pass_ = 1;
    double alpha_ = 2.3;
    int nparts_ = 1;
    std::vector<int> part_ids_;        // raw peeling index of each dense id
    std::vector<uint32_t> part_count_;
    std::vector<double> eps_part_;
    double omega_ = 0, first_stop_ = 0, last_stop_ = 0, dfpb_ = 1.0;
    uint64_t next_stop_ = 0;
    int iteration_ = 0;
    double eps_final_topk_ = 1.0;
    uint32_t numresults_topk_ = 0;
    double eps_stop_ = -1;
    uint32_t checks_ = 0;
    double max_num_samples_ = 0;
    double sup_bcest_p1_ = 0, sup_wv_p1_ = 0;
    uint64_t void_p1_ = 0;
    float t_sample_ms_ = 0, t_apply_ms_ = 0;
    std::vector<uint32_t> final_rank_el_;
    std::vector<double> final_rank_val_;
    bool finished_ = false;
};

double now_seconds();

}  // namespace silvan
