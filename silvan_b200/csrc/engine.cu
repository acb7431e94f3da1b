// Host engine (see engine.h): device graph upload, slot and round pools, and
// the estimator driver that restates Probabilistic::run
// (silvan/src/Probabilistic.cpp:775-1139) in its one-thread semantics on top
// of device rounds.
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <map>
#include <mutex>
#include <sstream>

#include "bounds.h"

namespace silvan {

namespace {
thread_local std::string g_err;
constexpr uint32_t kRoundSamples = 65536;   // samples per sampler launch
constexpr uint64_t kInitialRecords = 1u << 22;
constexpr uint32_t kBlock = 11;             // samples per block (Probabilistic.cpp:829,1061)
constexpr uint32_t kUncertainCap = 1u << 16;

template <typename T>
int dmalloc(T **p, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)p, sizeof(T) * count);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        set_error(std::string("device allocation failed: ") + cudaGetErrorString(e));
        return SILVAN_E_OOM;
    }
    return SILVAN_OK;
}
template <typename T>
void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}
}  // namespace

void set_error(const std::string &msg) { g_err = msg; }
const char *last_error_cstr() { return g_err.c_str(); }

int cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return SILVAN_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? SILVAN_E_OOM : SILVAN_E_CUDA;
}

#define CK(expr)                                          \
    do {                                                  \
        int _rc = cuda_status((expr), #expr);             \
        if (_rc != SILVAN_OK) return _rc;                 \
    } while (0)
#define RK(expr)                  \
    do {                          \
        int _rc = (expr);         \
        if (_rc != SILVAN_OK) return _rc; \
    } while (0)

double now_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// ---------------------------------------------------------------------------
// DeviceGraph
// ---------------------------------------------------------------------------
int DeviceGraph::upload() {
    const HostGraph &h = host;
    if (h.n < 2) {
        set_error("graph needs at least two nodes");
        return SILVAN_E_BADARG;
    }
    if (h.num_edges() >= 0xffffffffull || (h.directed && h.in_adj.size() >= 0xffffffffull)) {
        set_error("graphs with 2^32 or more edge entries are not supported");
        return SILVAN_E_BADARG;
    }
    CK(cudaGetDevice(&device));
    const uint32_t n = h.n;
    std::vector<uint32_t> off32(n + 1);
    auto put = [&](uint32_t **doff, uint32_t **dadj, const std::vector<uint64_t> &off,
                   const std::vector<uint32_t> &adj) -> int {
        for (uint32_t i = 0; i <= n; i++) off32[i] = (uint32_t)off[i];
        RK(dmalloc(doff, n + 1));
        RK(dmalloc(dadj, adj.size()));
        CK(cudaMemcpy(*doff, off32.data(), sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice));
        if (!adj.empty())
            CK(cudaMemcpy(*dadj, adj.data(), sizeof(uint32_t) * adj.size(),
                          cudaMemcpyHostToDevice));
        return SILVAN_OK;
    };
    RK(put(&d_out_off, &d_out_adj, h.out_off, h.out_adj));
    if (h.directed) {
        RK(put(&d_in_off, &d_in_adj, h.in_off, h.in_adj));
    } else {
        d_in_off = d_out_off;
        d_in_adj = d_out_adj;
    }
    RK(dmalloc(&d_cc, n));
    CK(cudaMemcpy(d_cc, cc.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    return SILVAN_OK;
}

DeviceGraph::~DeviceGraph() {
    if (d_in_off != d_out_off) dfree(d_in_off);
    if (d_in_adj != d_out_adj) dfree(d_in_adj);
    d_in_off = d_in_adj = nullptr;
    dfree(d_out_off);
    dfree(d_out_adj);
    dfree(d_cc);
}

// ---------------------------------------------------------------------------
// pools
// ---------------------------------------------------------------------------
int SlotPool::alloc(uint32_t s, uint32_t nn, cudaStream_t st) {
    free_all();
    slots = s;
    n = nn;
    const uint64_t tot = (uint64_t)s * nn;
    RK(dmalloc(&rec, tot));
    RK(dmalloc(&queue, tot));
    RK(dmalloc(&hits, tot));
    RK(dmalloc(&touched, tot));
    RK(dmalloc(&meet, (uint64_t)s * kMeetCap));
    RK(dmalloc(&meet_pre, (uint64_t)s * kMeetCap));
    CK(sampler_init_slots(rec, hits, tot, st));
    return SILVAN_OK;
}

void SlotPool::free_all() {
    dfree(rec);
    dfree(queue);
    dfree(hits);
    dfree(touched);
    dfree(meet);
    dfree(meet_pre);
}

int RoundPool::alloc(uint32_t nn, uint32_t max_samples, uint64_t rec_cap) {
    free_all();
    n = nn;
    RoundBuffers &r = rb;
    r.max_samples = max_samples;
    RK(dmalloc(&r.pl, max_samples));
    RK(dmalloc(&r.np, max_samples));
    RK(dmalloc(&r.vis, max_samples));
    RK(dmalloc(&r.status, max_samples));
    RK(dmalloc(&r.signs, max_samples));
    RK(dmalloc(&r.ball, max_samples));
    RK(dmalloc(&r.pred, max_samples));
    RK(dmalloc(&r.rec_cursor, 1));
    RK(dmalloc(&r.node_cnt, nn));
    RK(dmalloc(&r.n_touched, 1));
    RK(dmalloc(&r.block_sums, 1024));
    RK(dmalloc(&r.work_counter, 1));
    CK(cudaMemset(r.node_cnt, 0, sizeof(uint32_t) * nn));
    return grow_records(rec_cap);
}

int RoundPool::grow_records(uint64_t cap) {
    RoundBuffers &r = rb;
    dfree(r.recs);
    dfree(r.touched);
    dfree(r.bucket_off);
    dfree(r.entries);
    r.rec_cap = cap;
    const uint64_t tcap = std::min<uint64_t>(cap, n) + 1;
    RK(dmalloc(&r.recs, cap));
    RK(dmalloc(&r.touched, tcap));
    RK(dmalloc(&r.bucket_off, tcap + 1));
    RK(dmalloc(&r.entries, cap));
    return SILVAN_OK;
}

void RoundPool::free_all() {
    RoundBuffers &r = rb;
    dfree(r.pl);
    dfree(r.np);
    dfree(r.vis);
    dfree(r.status);
    dfree(r.signs);
    dfree(r.ball);
    dfree(r.pred);
    dfree(r.recs);
    dfree(r.rec_cursor);
    dfree(r.node_cnt);
    dfree(r.touched);
    dfree(r.n_touched);
    dfree(r.bucket_off);
    dfree(r.entries);
    dfree(r.block_sums);
    dfree(r.work_counter);
}

// ---------------------------------------------------------------------------
// Job
// ---------------------------------------------------------------------------
Job::~Job() {
    if (stream_) cudaStreamSynchronize(stream_);
    dfree(jc_.approx);
    dfree(jc_.wimpy);
    dfree(jc_.mcrade);
    dfree(jc_.last_upd);
    dfree(jc_.cross_flag);
    dfree(jc_.cross_sample);
    dfree(jc_.sp_lengths);
    dfree(jc_.sc);
    dfree(jc_.partition);
    dfree(jc_.peel_idx);
    dfree(d_red_);
    dfree(d_unc_);
    dfree(d_nunc_);
    dfree(d_lut_);
    dfree(d_hist_);
    if (h_red_) cudaFreeHost(h_red_);
    if (h_sc_) cudaFreeHost(h_sc_);
    if (h_cursor_) cudaFreeHost(h_cursor_);
    for (auto &e : ev_)
        if (e) cudaEventDestroy(e);
    for (auto &e : ev_run_)
        if (e) cudaEventDestroy(e);
    slots_.free_all();
    round_.free_all();
    if (stream_) cudaStreamDestroy(stream_);
}

int Job::init() {
    const uint32_t n = g_->host.n;
    if (!(p_.eps > 0 && p_.eps < 1) || !(p_.delta > 0 && p_.delta < 1)) {
        set_error("eps and delta must lie in (0, 1)");
        return SILVAN_E_BADARG;
    }
    if (p_.np_cap == 0) p_.np_cap = 1u << 24;
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    for (auto &e : ev_) CK(cudaEventCreate(&e));
    for (auto &e : ev_run_) CK(cudaEventCreate(&e));
    uint32_t slots = p_.slots;
    if (slots == 0) {
        int dev = 0, sms = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        int per = std::max(1, sampler_max_ctas_per_sm());
        slots = (uint32_t)(sms * per);
        // keep the slot state within half of the free memory
        size_t fr = 0, tot = 0;
        CK(cudaMemGetInfo(&fr, &tot));
        const uint64_t per_slot = (uint64_t)n * (sizeof(NodeRec) + 12) + (uint64_t)kMeetCap * 16;
        const uint64_t fit = (fr / 2) / std::max<uint64_t>(per_slot, 1);
        if (fit < slots) slots = (uint32_t)std::max<uint64_t>(fit, 1);
    }
    RK(slots_.alloc(slots, n, stream_));
    RK(round_.alloc(n, kRoundSamples, kInitialRecords));
    RK(dmalloc(&jc_.approx, n));
    RK(dmalloc(&jc_.wimpy, n));
    RK(dmalloc(&jc_.mcrade, (uint64_t)n * kTrials));
    RK(dmalloc(&jc_.last_upd, n));
    RK(dmalloc(&jc_.cross_flag, n));
    RK(dmalloc(&jc_.cross_sample, n));
    RK(dmalloc(&jc_.sp_lengths, (uint64_t)g_->diameter + 1));
    RK(dmalloc(&jc_.sc, 1));
    RK(dmalloc(&jc_.partition, n));
    RK(dmalloc(&jc_.peel_idx, n));
    RK(dmalloc(&d_red_, 1));
    RK(dmalloc(&d_unc_, kUncertainCap));
    RK(dmalloc(&d_nunc_, 1));
    CK(cudaMallocHost((void **)&h_red_, sizeof(StopReduction)));
    CK(cudaMallocHost((void **)&h_sc_, sizeof(JobScalars)));
    CK(cudaMallocHost((void **)&h_cursor_, sizeof(unsigned long long)));
    CK(cudaMemsetAsync(jc_.approx, 0, sizeof(double) * n, stream_));
    CK(cudaMemsetAsync(jc_.wimpy, 0, sizeof(double) * n, stream_));
    CK(cudaMemsetAsync(jc_.mcrade, 0, sizeof(long long) * (uint64_t)n * kTrials, stream_));
    CK(cudaMemsetAsync(jc_.last_upd, 0, sizeof(uint32_t) * n, stream_));
    CK(cudaMemsetAsync(jc_.cross_flag, 0, n, stream_));
    CK(cudaMemsetAsync(jc_.sp_lengths, 0, sizeof(uint64_t) * (g_->diameter + 1), stream_));
    CK(cudaMemsetAsync(jc_.sc, 0, sizeof(JobScalars), stream_));
    CK(cudaMemsetAsync(jc_.partition, 0, sizeof(int32_t) * n, stream_));
    CK(cudaStreamSynchronize(stream_));
    return SILVAN_OK;
}

// Draws global samples [first_global, first_global + count) and commits them.
int Job::run_batch(uint32_t first_global, uint32_t count, int pass, bool track_cross) {
    const DeviceGraph &G = *g_;
    RoundBuffers &rb = round_.rb;
    SamplerArgs A{};
    A.out_off = G.d_out_off;
    A.out_adj = G.d_out_adj;
    A.in_off = G.d_in_off;
    A.in_adj = G.d_in_adj;
    A.cc = G.d_cc;
    A.n = G.host.n;
    A.directed = G.host.directed ? 1 : 0;
    A.rec = slots_.rec;
    A.queue = slots_.queue;
    A.hits = slots_.hits;
    A.touched = slots_.touched;
    A.meet = slots_.meet;
    A.meet_pre = slots_.meet_pre;
    A.seed = p_.seed;
    A.alpha = alpha_;
    A.np_cap = p_.np_cap;
    A.work_counter = rb.work_counter;
    A.out_pl = rb.pl;
    A.out_np = rb.np;
    A.out_vis = rb.vis;
    A.out_status = rb.status;
    A.out_ball = rb.ball;
    A.out_pred = rb.pred;
    const bool plain = p_.form == SILVAN_FORM_PLAIN;
    for (uint32_t done = 0; done < count;) {
        const uint32_t c = std::min<uint32_t>(count - done, kRoundSamples);
        A.first_sample = first_global + done;
        A.count = c;
        for (;;) {
            A.recs = rb.recs;
            A.rec_cursor = rb.rec_cursor;
            A.rec_cap = rb.rec_cap;
            CK(cudaMemsetAsync(rb.work_counter, 0, sizeof(uint32_t), stream_));
            CK(cudaMemsetAsync(rb.rec_cursor, 0, sizeof(unsigned long long), stream_));
            const uint32_t grid = std::min<uint32_t>(slots_.slots, c);
            if (!plain) CK(cudaEventRecord(ev_[0], stream_));
            CK(sampler_launch(A, grid, stream_));
            launches_ += 1;
            if (plain) break;
            CK(cudaEventRecord(ev_[1], stream_));
            CK(cudaMemcpyAsync(h_cursor_, rb.rec_cursor, sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
            t_sample_ms_ += ms;
            if (*h_cursor_ <= rb.rec_cap) break;
            // the round's path maps did not fit: grow and redraw (deterministic)
            uint64_t cap = rb.rec_cap;
            while (cap < *h_cursor_) cap *= 2;
            RK(round_.grow_records(cap));
        }
        ApplyArgs ap{};
        ap.n = G.host.n;
        ap.seed = p_.seed;
        ap.first_sample = A.first_sample;
        ap.pass = pass;
        ap.track_cross = track_cross ? 1 : 0;
        ap.D = G.diameter;
        if (!plain) CK(cudaEventRecord(ev_[2], stream_));
        for (uint32_t lo = 0; lo < c; lo += kLargeBucket) {
            ap.lo = lo;
            ap.hi = std::min<uint32_t>(c, lo + kLargeBucket);
            CK(apply_round(rb, jc_, ap, stream_));
            launches_ += kApplyRoundKernels - (pass == 2 ? 0 : 1);
        }
        if (!plain) {
            CK(cudaEventRecord(ev_[3], stream_));
            CK(cudaEventSynchronize(ev_[3]));
            float ms = 0;
            cudaEventElapsedTime(&ms, ev_[2], ev_[3]);
            t_apply_ms_ += ms;
        }
        done += c;
    }
    return SILVAN_OK;
}

// Commits samples of the current pass until pass_samples_ == target.
int Job::sample_range(uint64_t lo, uint64_t hi, int pass, bool track_cross) {
    (void)lo;
    if (hi <= pass_samples_) return SILVAN_OK;
    const uint64_t cnt = hi - pass_samples_;
    if (global_next_ + cnt >= 0xffffffffull) {
        set_error("more than 2^32 samples");
        return SILVAN_E_BADARG;
    }
    if (p_.form == SILVAN_FORM_PLAIN) {
        for (uint64_t done = 0; done < cnt; done += kBlock) {
            const uint32_t c = (uint32_t)std::min<uint64_t>(kBlock, cnt - done);
            RK(run_batch((uint32_t)(global_next_ + done), c, pass, track_cross));
        }
    } else {
        RK(run_batch((uint32_t)global_next_, (uint32_t)cnt, pass, track_cross));
    }
    global_next_ += cnt;
    pass_samples_ = hi;
    return SILVAN_OK;
}

int Job::sync_scalars(JobScalars &sc) {
    CK(cudaMemcpyAsync(h_sc_, jc_.sc, sizeof(JobScalars), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    sc = *h_sc_;
    if (sc.error != 0) {
        const char *what = sc.error == SILVAN_E_OVERFLOW
                               ? "a sample's 64-bit path count wrapped to 0 (the reference "
                                 "divides by zero here)"
                           : sc.error == SILVAN_E_NP_CAP
                               ? "a sample asked for more shortest paths than the job's cap"
                           : sc.error == SILVAN_E_CAPACITY ? "a per-sample buffer overflowed"
                                                           : "device sampler error";
        set_error(what);
        return sc.error;
    }
    return SILVAN_OK;
}

int Job::read_sp_lengths(std::vector<uint64_t> &out) {
    out.assign((size_t)g_->diameter + 1, 0);
    CK(cudaMemcpyAsync(out.data(), jc_.sp_lengths, sizeof(uint64_t) * out.size(),
                       cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    return SILVAN_OK;
}

// Empirical peeling (silvan/src/Probabilistic.cpp:853-871).
int Job::peel(double a, bool enabled) {
    const uint32_t n = g_->host.n;
    const double ms = (double)pass_samples_;
    part_ids_.clear();
    part_count_.clear();
    if (!enabled) {
        CK(cudaMemsetAsync(jc_.partition, 0, sizeof(int32_t) * n, stream_));
        part_ids_.push_back(0);
        part_count_.push_back(n);
        nparts_ = 1;
        return SILVAN_OK;
    }
    CK(peel_index(jc_, n, ms, a, d_unc_, d_nunc_, kUncertainCap, stream_));
    launches_ += 3;
    uint32_t nunc = 0;
    CK(cudaMemcpyAsync(&nunc, d_nunc_, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    auto host_idx = [&](double w) {
        double emp_w = w / ms;
        double min_inv = fmin(1. / emp_w, ms);
        return (int)(log(min_inv) / log(a) + 1);
    };
    if (nunc > kUncertainCap) {
        std::vector<double> w(n);
        std::vector<int32_t> idx(n);
        CK(cudaMemcpy(w.data(), jc_.wimpy, sizeof(double) * n, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; i++) idx[i] = host_idx(w[i]);
        CK(cudaMemcpy(jc_.peel_idx, idx.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    } else if (nunc > 0) {
        std::vector<uint32_t> unc(nunc);
        CK(cudaMemcpy(unc.data(), d_unc_, sizeof(uint32_t) * nunc, cudaMemcpyDeviceToHost));
        for (uint32_t v : unc) {
            double w;
            CK(cudaMemcpy(&w, jc_.wimpy + v, sizeof(double), cudaMemcpyDeviceToHost));
            int32_t idx = host_idx(w);
            CK(cudaMemcpy(jc_.peel_idx + v, &idx, sizeof(int32_t), cudaMemcpyHostToDevice));
        }
    }
    // histogram of the indices: they lie in [1, log(m)/log(a) + 1]
    const int32_t idx_min = std::min(0, host_idx(ms)) ;
    const int32_t idx_max = std::max(host_idx(0.0), host_idx(ms)) + 2;
    const int32_t nbins = idx_max - idx_min + 1;
    if (nbins > (1 << 22)) {
        set_error("empirical peeling parameter too close to 1");
        return SILVAN_E_BADARG;
    }
    dfree(d_hist_);
    RK(dmalloc(&d_hist_, nbins));
    CK(peel_hist(jc_, n, idx_min, nbins, d_hist_, stream_));
    std::vector<uint32_t> hist(nbins);
    CK(cudaMemcpyAsync(hist.data(), d_hist_, sizeof(uint32_t) * nbins, cudaMemcpyDeviceToHost,
                       stream_));
    CK(cudaStreamSynchronize(stream_));
    std::vector<int32_t> lut(nbins, 0);
    int dense = 0;
    for (int32_t b = 0; b < nbins; b++) {
        if (hist[b]) {
            lut[b] = dense++;
            part_ids_.push_back(b + idx_min);
            part_count_.push_back(hist[b]);
        }
    }
    nparts_ = dense;
    if (nparts_ > kMaxPartitions) {
        set_error("more than 128 non-empty peeling partitions");
        return SILVAN_E_BADARG;
    }
    dfree(d_lut_);
    RK(dmalloc(&d_lut_, nbins));
    CK(cudaMemcpy(d_lut_, lut.data(), sizeof(int32_t) * nbins, cudaMemcpyHostToDevice));
    CK(peel_map(jc_, n, d_lut_, idx_min, nbins, nullptr, stream_));
    return SILVAN_OK;
}

// Current ranking list (silvan/src/Ranking_list.cpp): the union_sample nodes
// of largest (approx, last update), never-updated nodes after the updated
// ones in ascending id.
int Job::ranking(std::vector<uint32_t> &el, std::vector<double> &val) {
    const uint32_t n = g_->host.n;
    std::vector<double> ap(n);
    std::vector<uint32_t> lu(n);
    CK(cudaMemcpyAsync(ap.data(), jc_.approx, sizeof(double) * n, cudaMemcpyDeviceToHost,
                       stream_));
    CK(cudaMemcpyAsync(lu.data(), jc_.last_upd, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost,
                       stream_));
    CK(cudaStreamSynchronize(stream_));
    const uint32_t K = union_sample_;
    std::vector<uint32_t> idx;
    idx.reserve(n);
    for (uint32_t i = 0; i < n; i++)
        if (lu[i] != 0) idx.push_back(i);
    auto better = [&](uint32_t x, uint32_t y) {
        if (ap[x] != ap[y]) return ap[x] > ap[y];
        if (lu[x] != lu[y]) return lu[x] > lu[y];
        return x > y;  // same sample: ascending node order, later node is newer
    };
    const size_t take = std::min<size_t>(K, idx.size());
    std::partial_sort(idx.begin(), idx.begin() + take, idx.end(), better);
    idx.resize(take);
    // never-updated nodes of the initial list (ids < K) fill the tail
    for (uint32_t i = 0; i < K && idx.size() < K; i++)
        if (lu[i] == 0) idx.push_back(i);
    el = idx;
    val.resize(el.size());
    for (size_t i = 0; i < el.size(); i++) val[i] = ap[el[i]];
    return SILVAN_OK;
}

namespace {
// Fixed-length descending list (silvan/src/Ranking_list.cpp:20-43), used for
// the per-check bound lists of the top-k test.
struct SmallRanking {
    std::vector<uint32_t> el;
    std::vector<double> val;
    explicit SmallRanking(uint32_t k) : el(k), val(k, 0.0) {
        for (uint32_t i = 0; i < k; i++) el[i] = i;
    }
    void put(uint32_t e, double nv) {
        uint32_t k = (uint32_t)el.size(), i;
        for (i = k; i-- > 0;)
            if (val[i] > nv) break;
        i++;
        uint32_t ce = e;
        double cv = nv;
        while (i < k) {
            std::swap(ce, el[i]);
            std::swap(cv, val[i]);
            if (ce == e) break;
            i++;
        }
    }
};
}  // namespace

// check_topk_guarantees (silvan/src/Probabilistic.cpp:587-687).
bool Job::check_topk(std::string &outs) {
    std::ostringstream out;
    const double ms = (double)pass_samples_;
    out << "EVALUATING STOPPING CONDITION FOR TOP-K RELATIVE APPROX" << "\n";
    const double dpb = p_.delta / pow(2., iteration_);
    eps_final_topk_ = 1.0;
    double lb_topk = 0.0, ub_topk = 1.0;
    std::vector<uint32_t> el;
    std::vector<double> val;
    if (ranking(el, val) != SILVAN_OK) {
        outs += out.str();
        return false;
    }
    std::vector<uint64_t> sp;
    read_sp_lengths(sp);
    std::vector<int32_t> part_of(el.size());
    for (size_t i = 0; i < el.size(); i++)
        cudaMemcpy(&part_of[i], jc_.partition + el[i], sizeof(int32_t), cudaMemcpyDeviceToHost);
    SmallRanking sub(k_), slb(k_);
    uint32_t ins = 0;
    bool rel = true;
    const uint32_t n = g_->host.n;
    for (uint64_t i = 0; i < union_sample_ && rel; i++) {
        const uint32_t node = el[i];
        const double an = val[i] / ms;
        const double ec = eps_part_[part_of[i]];
        double lbb = an - ec, ubb = an + ec;
        const double adu =
            upper_bound_avg_diameter(sp, (int)g_->diameter, dpb, pass_samples_).ub;
        const double lbr = relative_bound(an, dpb, adu, ms, false, n);
        const double ubr = relative_bound(an, dpb, adu, ms, true, n);
        lbb = fmax(lbb, lbr);
        ubb = fmin(ubb, ubr);
        sub.put(node, ubb);
        slb.put(node, lbb);
        ins++;
        if (ins >= k_) {
            ub_topk = fmin(ub_topk, sub.val[k_ - 1]);
            lb_topk = fmax(lb_topk, slb.val[k_ - 1]);
        }
        if (ubb > lb_topk) {
            eps_final_topk_ = fmin(eps_final_topk_, ec);
            const bool lc = lbb >= an / (1. + p_.eps);
            const bool uc = ubb <= an / (1. - p_.eps);
            const bool lcr = lbr >= an / (1. + p_.eps);
            const bool ucr = ubr <= an / (1. - p_.eps);
            if (!lc) {
                out << "do not stop as current node has to improve lowerbound " << "\n";
                out << "   lowerbound_bc_ " << lbb << "\n";
                out << "   lowerbound_bc_rel " << lbr << "\n";
                out << "   rel condition " << lcr << "\n";
                out << "   approx_node/(1.+err) " << an / (1. + p_.eps) << "\n";
            }
            if (!uc) {
                out << "do not stop as current node has to improve upperbound " << "\n";
                out << "   upperbound_bc_ " << ubb << "\n";
                out << "   upperbound_bc_rel " << ubr << "\n";
                out << "   rel condition " << ucr << "\n";
                out << "   approx_node/(1.-err) " << an / (1. - p_.eps) << "\n";
            }
            if (!lc || !uc) {
                out << "   approx_node " << an << "\n";
                out << "   node_partition_index " << part_ids_[part_of[i]] << "\n";
            }
            rel = rel && lc && uc;
        } else {
            eps_final_topk_ = fmin(eps_final_topk_, lb_topk - an);
        }
    }
    out << "*** ub_topk_bc " << ub_topk << "\n";
    out << "*** lb_topk_bc " << lb_topk << "\n";
    if (rel) {
        out << "RELATIVE APPROX FOR TOP-K OBTAINED" << "\n";
        uint32_t cnt = 0;
        for (uint32_t i = 0; i < ins; i++) {
            const double an = val[i] / ms;
            const double ec = eps_part_[part_of[i]];
            if (an + ec > lb_topk) {
                out << i + 1 << ") (" << el[i] << ") " << an - ec << " " << an << " " << an + ec
                    << " " << "\n";
                cnt++;
            }
        }
        numresults_topk_ = cnt;
    }
    outs += out.str();
    return rel;
}

// compute_finished_mcrade (silvan/src/Probabilistic.cpp:251-414).
int Job::stop_check(bool &stop, std::string &outs) {
    std::ostringstream out;
    checks_++;
    const double ms = (double)pass_samples_;
    double dpb = 1.0;
    if (absolute_ && p_.m_hat) dpb = dfpb_;
    else dpb = p_.delta / pow(2., iteration_);
    out << "\n";
    out << "EVALUATING STOPPING CONDITION at iteration " << iteration_ << " (m=" << pass_samples_
        << ", d=" << dpb << ")" << "\n";
    const long long init = -(long long)pass_samples_;
    CK(stop_reduce(jc_, g_->host.n, nparts_, init, d_red_, stream_));
    launches_ += 2;
    CK(cudaMemcpyAsync(h_red_, d_red_, sizeof(StopReduction), cudaMemcpyDeviceToHost, stream_));
    JobScalars sc;
    RK(sync_scalars(sc));
    const StopReduction &R = *h_red_;
    if (absolute_) {
        std::vector<uint64_t> sp;
        RK(read_sp_lengths(sp));
        const double adu = upper_bound_avg_diameter(sp, (int)g_->diameter, dpb, pass_samples_).ub;
        const double t1 = R.approx_max / ms;
        const double t1u = upper_bound_top1(t1, dpb, pass_samples_);
        const double wvu = upper_bound_top1(R.wimpy_all_max / ms, dpb, pass_samples_);
        if (p_.m_hat) {
            const uint64_t mns = (uint64_t)upper_bound_samples(t1u, wvu, adu, p_.eps, dpb);
            if (last_stop_ > (double)mns) {
                last_stop_ = (double)mns;
                omega_ = last_stop_;
                out << "******NEW STOPPING CONDITION UPDATE!!! last_stopping_samples: "
                    << last_stop_ << "\n";
                const double mni = log((double)mns / (double)first_stop_) / log(1.2) + 1;
                dfpb_ = p_.delta / (floor(mni));
            }
            if (mns <= pass_samples_) out << "******NEW STOPPING CONDITION TRUE!!! " << "\n";
        }
    }
    eps_part_.assign(nparts_, 1.0);
    for (int i = 0; i < nparts_; i++) {
        double avg = 0.0;
        for (int j = 0; j < kTrials; j++) avg += R.mc_max[i * kTrials + j] / (double)kTrials;
        avg = avg / ms;
        const double sw = R.wimpy_max[i] / ms;
        const double dp = dpb / nparts_;
        eps_part_[i] = epsilon_mcrade(sw, avg, dp, ms, (double)part_count_[i], kTrials);
    }
    if (absolute_) {
        double sup = 0;
        for (int i = 0; i < nparts_; i++) sup = fmax(sup, eps_part_[i]);
        stop = sup <= p_.eps;
        if (stop) {
            eps_stop_ = sup;
            out << "MCRADE STOPS WITH eps " << sup << "\n";
            out << "MCRADE STOPS at iteration " << iteration_ << "\n";
            out << "MCRADE STOPS at sample size " << pass_samples_ << "\n";
        } else {
            out << "   mcrade eps " << sup << "\n";
        }
        outs += out.str();
        return SILVAN_OK;
    }
    std::string tk;
    stop = check_topk(tk);
    out << tk;
    if (stop) {
        out << "MCRADE REL STOPS " << "\n";
        out << "MCRADE STOPS at iteration " << iteration_ << "\n";
        out << "MCRADE STOPS at sample size " << pass_samples_ << "\n";
    } else {
        out << "MCRADE REL DOES NOT STOP " << "\n";
    }
    outs += out.str();
    return SILVAN_OK;
}

void Job::reset_pass2_counters() {
    const uint32_t n = g_->host.n;
    cudaMemsetAsync(jc_.approx, 0, sizeof(double) * n, stream_);
    cudaMemsetAsync(jc_.wimpy, 0, sizeof(double) * n, stream_);
    cudaMemsetAsync(jc_.mcrade, 0, sizeof(long long) * (uint64_t)n * kTrials, stream_);
    cudaMemsetAsync(jc_.last_upd, 0, sizeof(uint32_t) * n, stream_);
}

// Probabilistic::run (silvan/src/Probabilistic.cpp:775-1139).
int Job::run(silvan_result_t *res, FILE *sink) {
    std::ostringstream out;
    auto flush = [&]() {
        if (sink) {
            std::string s = out.str();
            fwrite(s.data(), 1, s.size(), sink);
            fflush(sink);
        }
        out.str("");
        out.clear();
    };
    const uint32_t n = g_->host.n;
    const uint64_t m = g_->host.num_edges();
    const int D = (int)g_->diameter;
    const double eps = p_.eps, delta = p_.delta;
    absolute_ = p_.k == 0;
    out << "estimated diameter of the graph: " << D << "\n";
    out << "time for estimating diameter " << g_->diameter_seconds << "\n";
    uint32_t tau = (uint32_t)fmax(1. / eps * (log(1. / delta)), 1000.);
    tau = (uint32_t)fmax((double)tau, 2 * D * (log(1. / delta)));
    tau_ = tau;
    out << "Starting first pass. Tentative number of samples: " << tau << "\n";
    const bool peel_on = p_.a > 1;
    const double a = peel_on ? p_.a : 100. * tau;
    const uint32_t threads = p_.threads ? p_.threads : 1;
    union_sample_ = std::min(n, (uint32_t)fmax(2 * sqrt((double)m) / threads, p_.k + 20.));
    k_ = std::min(p_.k, n);
    flush();
    CK(cudaMemsetAsync(jc_.sp_lengths, 0, sizeof(uint64_t) * (D + 1), stream_));
    launches_ = 0;
    const double start_time = now_seconds();
    CK(cudaEventRecord(ev_run_[0], stream_));

    // ---- pass 1 (:819-846) --------------------------------------------------
    pass_ = 1;
    alpha_ = p_.alpha;
    global_next_ = 0;
    pass_samples_ = 0;
    if (absolute_) {
        const uint64_t P1 = (uint64_t)kBlock * ((tau + kBlock - 1) / kBlock);
        RK(sample_range(0, P1, 1, false));
    } else {
        // stop after the first block with n_pairs >= tau and at least 1.5 k
        // nodes whose approx reached 3 (crossings are recorded per sample)
        uint64_t target = (uint64_t)kBlock * ((tau + kBlock - 1) / kBlock);
        uint64_t chunk = target;
        std::vector<uint32_t> cross;
        for (;;) {
            RK(sample_range(0, target, 1, true));
            JobScalars sc;
            RK(sync_scalars(sc));
            cross.resize(sc.n_cross);
            if (sc.n_cross)
                CK(cudaMemcpy(cross.data(), jc_.cross_sample, sizeof(uint32_t) * sc.n_cross,
                              cudaMemcpyDeviceToHost));
            std::sort(cross.begin(), cross.end());
            // first block end b*11 >= tau with #crossings before it >= 1.5 k
            uint64_t stop_at = 0;
            const double need = 1.5 * p_.k;
            uint64_t first_b = (tau + kBlock - 1) / kBlock;
            for (uint64_t b = first_b; b * kBlock <= target; b++) {
                const uint64_t end = b * kBlock;
                const uint64_t c =
                    std::lower_bound(cross.begin(), cross.end(), (uint32_t)end) - cross.begin();
                if ((double)c >= need) {
                    stop_at = end;
                    break;
                }
            }
            if (stop_at == 0) {
                chunk *= 2;
                target += chunk;
                continue;
            }
            if (stop_at < target) {
                // roll back: recompute pass 1 up to stop_at
                CK(cudaMemsetAsync(jc_.approx, 0, sizeof(double) * n, stream_));
                CK(cudaMemsetAsync(jc_.wimpy, 0, sizeof(double) * n, stream_));
                CK(cudaMemsetAsync(jc_.last_upd, 0, sizeof(uint32_t) * n, stream_));
                CK(cudaMemsetAsync(jc_.cross_flag, 0, n, stream_));
                CK(cudaMemsetAsync(jc_.sp_lengths, 0, sizeof(uint64_t) * (D + 1), stream_));
                CK(cudaMemsetAsync(jc_.sc, 0, sizeof(JobScalars), stream_));
                global_next_ = 0;
                pass_samples_ = 0;
                RK(sample_range(0, stop_at, 1, true));
            }
            break;
        }
    }
    const uint64_t P1 = pass_samples_;
    JobScalars sc1;
    RK(sync_scalars(sc1));
    double sup_bcest;
    double sup_wv;
    std::memcpy(&sup_bcest, &sc1.sup_approx_bits, sizeof(double));
    std::memcpy(&sup_wv, &sc1.sup_wimpy_bits, sizeof(double));
    out << "First pass finished after " << P1 << " iteration" << "\n";

    // ---- empirical peeling (:853-889) ---------------------------------------
    RK(peel(a, peel_on));
    out << "number_of_non_empty_partitions  " << nparts_ << "\n";
    for (int i = 0; i < nparts_; i++)
        out << "  part. w. index  " << part_ids_[i] << " has " << part_count_[i]
            << " elements, map to " << i << "\n";
    out << "time for first pass " << now_seconds() - start_time << "\n";
    out << "void_samples first pass " << sc1.void_samples << "\n";
    const double t_first = now_seconds() - start_time;
    flush();

    // ---- bounds and alpha switch (:906-942) ---------------------------------
    double mns = 0.;
    alpha_ = p_.alpha;
    if (absolute_) {
        std::vector<uint64_t> sp;
        RK(read_sp_lengths(sp));
        AvgDiamBound adb = upper_bound_avg_diameter(sp, D, delta / 8., P1);
        out << "avg_diam_: " << adb.avg << "\n";
        out << "avg_diam_upperbound_b: " << adb.ub_b << "\n";
        out << "avg_diam_upperbound_eb: " << adb.ub_eb << "\n";
        out << "var_estimate_avg_diam: " << adb.var << "\n";
        CK(cudaMemsetAsync(jc_.sp_lengths, 0, sizeof(uint64_t) * (D + 1), stream_));
        const double t1u = upper_bound_top1(sup_bcest / (double)P1, delta / 8., P1);
        const double wvu = upper_bound_top1(sup_wv / (double)P1, delta / 8., P1);
        if (!p_.alpha_given && wvu > 0.9 * t1u) alpha_ = -1.;
        if (p_.m_hat) mns = upper_bound_samples(t1u, wvu, adb.ub, eps, delta / 2.);
        const double vc = 0.5 / eps / eps * (log2(D - 1) + 1 + log(2. / delta));
        out << "sup_bcest: " << sup_bcest / (double)P1 << "\n";
        out << "sup_emp_wimpy_var: " << sup_wv / (double)P1 << "\n";
        out << "top1bc_upperbound: " << t1u << "\n";
        out << "wimpy_var_upperbound: " << wvu << "\n";
        out << "max_num_samples: " << mns << "\n";
        out << "VC_bound: " << vc << "\n";
        out << "alpha_sp_sampling: " << alpha_ << "\n";
    }
    max_num_samples_ = mns;
    iteration_ = 1;
    double est_kth = 1.0;
    if (!absolute_) {
        std::vector<uint32_t> el;
        std::vector<double> val;
        RK(ranking(el, val));
        const double vk = p_.k < val.size() ? val[p_.k] : 0.0;
        est_kth = vk / (double)P1 + 1.0 / (double)P1;
        out << "est_kth_bc: " << est_kth << "\n";
    }
    reset_pass2_counters();
    CK(cudaMemsetAsync(jc_.sc, 0, sizeof(JobScalars), stream_));
    omega_ = pow(10., 15);
    if (mns > 0.) omega_ = mns;

    // ---- first sample size by bisection (:973-1025) --------------------------
    uint64_t num_samples = P1;
    double lo = 1. / eps * log(2. / delta), hi = omega_;
    const double svn = sup_wv / (double)P1 + 1 / (double)P1;
    while (hi - lo > 10) {
        num_samples = (uint64_t)((hi + lo) / 2.);
        double eg;
        if (absolute_)
            eg = sqrt(2 * svn * log(2. / delta) / (double)num_samples) +
                 log(2. / delta) / (double)num_samples / 3.;
        else
            eg = sqrt(2 * est_kth * log(2. / delta / est_kth) / (double)num_samples) +
                 log(2. / delta / est_kth) / (double)num_samples / 3.;
        if (absolute_) {
            if (eg > eps) lo = (double)num_samples;
            else hi = (double)num_samples;
        } else {
            const bool v1 = est_kth + eg > est_kth / (1. - eps);
            const bool v2 = est_kth - eg < est_kth / (1. + eps);
            const bool v3 = eg >= est_kth * eps * pow((1 - eps) / (1 + eps), 2.);
            if (v1 || v2 || v3) lo = (double)num_samples;
            else hi = (double)num_samples;
        }
    }
    first_stop_ = (double)num_samples;
    if (p_.m_hat) {
        const double mni = log((double)mns / (double)first_stop_) / log(1.2) + 1;
        dfpb_ = delta / (floor(mni));
    }
    out << "first_stopping_samples: " << first_stop_ << "\n";
    last_stop_ = omega_;
    out << "last_stopping_samples: " << last_stop_ << "\n";
    if (first_stop_ >= last_stop_ / 4) {
        first_stop_ = last_stop_ / 4;
        out << "first_stopping_samples dropped to " << first_stop_ << "\n";
    }
    next_stop_ = (uint64_t)first_stop_;
    out << "Starting second phase... " << "\n";
    flush();

    // ---- pass 2 (:1054-1102) -------------------------------------------------
    const double t2_start = now_seconds();
    pass_ = 2;
    pass_samples_ = 0;
    int reason = 0;
    for (;;) {
        // the next block end at which the reference acts
        uint64_t target = UINT64_MAX;
        if (p_.m_hat) target = std::min<uint64_t>(target, kBlock * (uint64_t)ceil(omega_ / kBlock));
        {
            uint64_t b = (next_stop_ + kBlock - 1) / kBlock;
            if (b * kBlock <= pass_samples_) b = pass_samples_ / kBlock + 1;
            const uint64_t t = b * kBlock;
            if ((double)t < last_stop_) target = std::min(target, t);
        }
        if (target == UINT64_MAX) {
            set_error("stopping schedule has no next evaluation point");
            return SILVAN_E_STATE;
        }
        if (target <= pass_samples_) target = pass_samples_ + kBlock;
        RK(sample_range(pass_samples_, target, 2, false));
        if (p_.m_hat && (double)pass_samples_ >= omega_) {
            reason = 2;
            break;
        }
        if ((double)pass_samples_ < last_stop_ && pass_samples_ >= next_stop_) {
            bool stop = false;
            std::string s;
            RK(stop_check(stop, s));
            out << s;
            if (stop) {
                out << "MCRADE STOPS after seconds " << now_seconds() - start_time << "\n";
                out << "/* stop_mcrade is true */" << "\n";
                reason = 1;
                flush();
                break;
            }
            next_stop_ = (uint64_t)(next_stop_ * 1.2);
            iteration_ += 1;
            flush();
        }
    }
    CK(cudaEventRecord(ev_run_[1], stream_));
    JobScalars sc2;
    RK(sync_scalars(sc2));
    const double t_end = now_seconds();
    float run_ms = 0;
    cudaEventElapsedTime(&run_ms, ev_run_[0], ev_run_[1]);
    double sup_b2, sup_w2;
    std::memcpy(&sup_b2, &sc2.sup_approx_bits, sizeof(double));
    std::memcpy(&sup_w2, &sc2.sup_wimpy_bits, sizeof(double));
    const uint64_t N2 = pass_samples_;
    out << "out of second pass " << "\n";
    out << "time for second pass " << t_end - t2_start << "\n";
    out << "void_samples second pass " << sc2.void_samples << " ("
        << (double)sc2.void_samples / (double)N2 << ")" << "\n";
    const uint64_t vis_total = sc1.vis_edges + sc2.vis_edges;
    if (p_.verbose > 0) {
        if (!absolute_) out << "eps_final_topk " << eps_final_topk_ << "\n";
        out << std::setprecision(6) << "\n" << "Finished after " << N2 << " iterations." << "\n";
        out << "Edges visited: " << vis_total << "\n";
        out << "Average edges visited: " << (N2 ? vis_total / N2 : 0) << "\n";
        out << "Total time: " << t_end - start_time << "\n";
        out << "Time bfs: " << t_sample_ms_ / 1000.0 << "\n";
        out << "Time critical: " << t_apply_ms_ / 1000.0 << "\n";
        out << "Time compute finished: " << 0 << "\n";
        out << "Time mcera: " << 0 << "\n";
        out << "(Printing thread: " << 0 << ")" << "\n";
        out << "Avg time bfs: " << t_sample_ms_ / 1000.0 << "\n";
        out << "Avg time critical: " << t_apply_ms_ / 1000.0 << "\n";
        out << "Avg time critical (round): " << 0 << "\n";
        out << "Avg time compute finished: " << 0 << "\n";
        out << "Avg time mcera: " << 0 << "\n";
        out << "sup bc est: " << sup_b2 / (double)N2 << "\n";
        out << "sup_emp_wimpy_var: " << sup_w2 / (double)N2 << "\n";
        out << "void_samples: " << sc2.void_samples << "\n";
        out << "num_samples: " << N2 << "\n";
    }
    flush();
    if (!absolute_) {
        std::vector<uint32_t> el;
        std::vector<double> val;
        RK(ranking(el, val));
        final_rank_el_ = el;
        final_rank_val_ = val;
    }
    finished_ = true;
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->first_pass_samples = P1;
        res->num_samples = N2;
        res->vis_edges = vis_total;
        res->void_samples = sc2.void_samples;
        res->backtracked_paths = sc2.paths;
        res->tau = tau;
        res->diameter = (uint32_t)D;
        res->iteration_index = iteration_;
        res->num_partitions = nparts_;
        res->stop_reason = reason;
        res->union_sample = union_sample_;
        res->numresults_topk = numresults_topk_;
        res->checks = checks_;
        res->omega = omega_;
        res->first_stopping_samples = first_stop_;
        res->last_stopping_samples = last_stop_;
        res->alpha_sp_sampling = alpha_;
        res->eps_stop = eps_stop_;
        res->eps_final_topk = eps_final_topk_;
        res->sup_bcest = sup_b2 / (double)N2;
        res->sup_emp_wimpy_var = sup_w2 / (double)N2;
        res->max_num_samples = mns;
        res->time_total_s = t_end - start_time;
        res->time_first_pass_s = t_first;
        res->time_sampling_s = t_sample_ms_ / 1000.0;
        res->time_apply_s = t_apply_ms_ / 1000.0;
        res->time_device_s = run_ms / 1000.0;
        res->ball_nodes = sc1.ball_nodes + sc2.ball_nodes;
        res->pred_entries = sc1.pred_entries + sc2.pred_entries;
        res->kernel_launches = launches_;
    }
    return SILVAN_OK;
}

int Job::run_to(uint64_t target, silvan_status_t *st) {
    RK(sample_range(pass_samples_, target, pass_, false));
    JobScalars sc;
    int rc = sync_scalars(sc);
    if (st) {
        st->samples = pass_samples_;
        st->void_samples = sc.void_samples;
        st->vis_edges = sc.vis_edges;
        st->backtracked_paths = sc.paths;
        st->pass = pass_;
        st->error = sc.error;
    }
    return rc;
}

int Job::read_estimates(double *out, uint32_t n) {
    if (n != g_->host.n) {
        set_error("estimate buffer size does not match the graph");
        return SILVAN_E_BADARG;
    }
    CK(cudaMemcpy(out, jc_.approx, sizeof(double) * n, cudaMemcpyDeviceToHost));
    const double ms = (double)pass_samples_;
    for (uint32_t i = 0; i < n; i++) out[i] = out[i] / ms;
    return SILVAN_OK;
}

int Job::read_counters(double *approx, double *wimpy, int64_t *mcrade, int32_t *part) {
    const uint32_t n = g_->host.n;
    if (approx) CK(cudaMemcpy(approx, jc_.approx, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (wimpy) CK(cudaMemcpy(wimpy, jc_.wimpy, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (mcrade)
        CK(cudaMemcpy(mcrade, jc_.mcrade, sizeof(long long) * (uint64_t)n * kTrials,
                      cudaMemcpyDeviceToHost));
    if (part) {
        std::vector<int32_t> dense(n);
        CK(cudaMemcpy(dense.data(), jc_.partition, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; i++)
            part[i] = dense[i] < (int)part_ids_.size() ? part_ids_[dense[i]] : 0;
    }
    return SILVAN_OK;
}

int Job::read_topk(uint32_t *nodes, double *values, uint32_t cap, uint32_t *count) {
    if (!finished_ || absolute_) {
        set_error("no top-k result");
        return SILVAN_E_STATE;
    }
    const uint32_t c = std::min<uint32_t>(numresults_topk_, (uint32_t)final_rank_el_.size());
    if (count) *count = c;
    for (uint32_t i = 0; i < c && i < cap; i++) {
        nodes[i] = final_rank_el_[i];
        values[i] = final_rank_val_[i] / (double)pass_samples_;
    }
    return SILVAN_OK;
}

int Job::replay(uint32_t first, uint32_t count, double alpha, std::vector<int32_t> &pl,
                std::vector<int32_t> &np, std::vector<uint64_t> &vis,
                std::vector<int32_t> &status, std::vector<PathRec> &recs) {
    pl.assign(count, 0);
    np.assign(count, 0);
    vis.assign(count, 0);
    status.assign(count, 0);
    recs.clear();
    const double save_alpha = alpha_;
    const int save_form = p_.form;
    alpha_ = alpha;
    p_.form = SILVAN_FORM_BATCHED;
    RoundBuffers &rb = round_.rb;
    for (uint32_t done = 0; done < count;) {
        const uint32_t c = std::min<uint32_t>(count - done, kRoundSamples);
        // sample only: run the sampler part of run_batch without committing
        SamplerArgs A{};
        const DeviceGraph &G = *g_;
        A.out_off = G.d_out_off;
        A.out_adj = G.d_out_adj;
        A.in_off = G.d_in_off;
        A.in_adj = G.d_in_adj;
        A.cc = G.d_cc;
        A.n = G.host.n;
        A.directed = G.host.directed ? 1 : 0;
        A.rec = slots_.rec;
        A.queue = slots_.queue;
        A.hits = slots_.hits;
        A.touched = slots_.touched;
        A.meet = slots_.meet;
        A.meet_pre = slots_.meet_pre;
        A.seed = p_.seed;
        A.alpha = alpha_;
        A.np_cap = p_.np_cap;
        A.work_counter = rb.work_counter;
        A.out_pl = rb.pl;
        A.out_np = rb.np;
        A.out_vis = rb.vis;
        A.out_status = rb.status;
        A.out_ball = rb.ball;
        A.out_pred = rb.pred;
        A.first_sample = first + done;
        A.count = c;
        for (;;) {
            A.recs = rb.recs;
            A.rec_cursor = rb.rec_cursor;
            A.rec_cap = rb.rec_cap;
            CK(cudaMemsetAsync(rb.work_counter, 0, sizeof(uint32_t), stream_));
            CK(cudaMemsetAsync(rb.rec_cursor, 0, sizeof(unsigned long long), stream_));
            CK(sampler_launch(A, std::min<uint32_t>(slots_.slots, c), stream_));
            CK(cudaMemcpyAsync(h_cursor_, rb.rec_cursor, sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, stream_));
            CK(cudaStreamSynchronize(stream_));
            if (*h_cursor_ <= rb.rec_cap) break;
            uint64_t cap = rb.rec_cap;
            while (cap < *h_cursor_) cap *= 2;
            RK(round_.grow_records(cap));
        }
        CK(cudaMemcpy(pl.data() + done, rb.pl, sizeof(int32_t) * c, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(np.data() + done, rb.np, sizeof(int32_t) * c, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(vis.data() + done, rb.vis, sizeof(uint64_t) * c, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(status.data() + done, rb.status, sizeof(int32_t) * c,
                      cudaMemcpyDeviceToHost));
        const size_t r0 = recs.size();
        recs.resize(r0 + *h_cursor_);
        if (*h_cursor_)
            CK(cudaMemcpy(recs.data() + r0, rb.recs, sizeof(PathRec) * (*h_cursor_),
                          cudaMemcpyDeviceToHost));
        for (size_t i = r0; i < recs.size(); i++) recs[i].sample += done;
        done += c;
    }
    alpha_ = save_alpha;
    p_.form = save_form;
    return SILVAN_OK;
}

}  // namespace silvan
