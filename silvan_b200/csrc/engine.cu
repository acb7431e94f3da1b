// Host engine (see engine.h).
#include "engine.h"
#include "components.h"
#include "graph_dev.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <map>
#include <mutex>
#include <sstream>
#include <unordered_map>

#include "bounds.h"
#include "graph_dev.cuh"

namespace silvan {

// Held while a stream is being captured into a CUDA graph and around every
// call that synchronises the whole device or maps and unmaps memory: such a
// call from another thread would invalidate a capture in progress (the
// server's uploader thread allocates while its round thread captures).
std::mutex &capture_mutex() {
    static std::mutex *m = new std::mutex();
    return *m;
}

namespace {
thread_local std::string g_err;
constexpr uint32_t kRoundSamples = 65536;  // samples per job per round
constexpr uint64_t kInitialRecords = 1u << 20;
constexpr uint32_t kBlock = 11;  // samples per block (Probabilistic.cpp:829,1061)
constexpr uint32_t kUncertainCap = 1u << 16;

// Caching allocator for device and pinned host memory.  Requests start and
// finish all the time in a serving process, and cudaMalloc / cudaFree (and
// even more so cudaMallocHost / cudaFreeHost) cost milliseconds each, so
// freed blocks are kept per device and size class and handed out again.  A
// freed block is reusable only after a device synchronisation (the one
// cudaFree would have done), taken when a request finds no ready block but
// freed ones are waiting.  On allocation failure the cached blocks of the
// device are released and the allocation is tried once more.
class BlockCache {
  public:
    void *alloc(size_t bytes, bool host, cudaError_t *err) {
        int dev = 0;
        cudaGetDevice(&dev);
        const size_t cls = size_class(bytes);
        const Key key{host ? -1 - dev : dev, cls};
        {
            std::lock_guard<std::mutex> lk(mu_);
            void *p = take(key);
            if (!p && !pending_[key].empty()) {
                std::lock_guard<std::mutex> cl(capture_mutex());
                cudaDeviceSynchronize();
                for (auto &kv : pending_) {
                    auto &f = ready_[kv.first];
                    f.insert(f.end(), kv.second.begin(), kv.second.end());
                    kv.second.clear();
                }
                p = take(key);
            }
            if (p) {
                live_[p] = key;
                *err = cudaSuccess;
                return p;
            }
        }
        void *p = nullptr;
        {
            std::lock_guard<std::mutex> cl(capture_mutex());
            *err = host ? cudaMallocHost(&p, cls) : cudaMalloc(&p, cls);
        }
        if (*err != cudaSuccess) {
            cudaGetLastError();
            release(dev);
            std::lock_guard<std::mutex> cl(capture_mutex());
            *err = host ? cudaMallocHost(&p, cls) : cudaMalloc(&p, cls);
            if (*err != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
        }
        std::lock_guard<std::mutex> lk(mu_);
        live_[p] = key;
        return p;
    }
    void free(void *p) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu_);
        auto it = live_.find(p);
        if (it == live_.end()) return;
        pending_[it->second].push_back(p);
        live_.erase(it);
    }

    // Device bytes held by freed blocks of device dev kept for reuse.
    uint64_t idle_bytes(int dev) {
        std::lock_guard<std::mutex> lk(mu_);
        uint64_t b = 0;
        for (auto *m : {&ready_, &pending_})
            for (auto &kv : *m)
                if (kv.first.first == dev) b += (uint64_t)kv.first.second * kv.second.size();
        return b;
    }

  private:
    typedef std::pair<int, size_t> Key;  // device (host blocks: -1 - device), class
    static size_t size_class(size_t b) {
        if (b <= 256) return 256;
        if (b <= (2u << 20)) {
            size_t c = 256;
            while (c < b) c <<= 1;
            return c;
        }
        return (b + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1);
    }
    void *take(const Key &k) {
        auto it = ready_.find(k);
        if (it == ready_.end() || it->second.empty()) return nullptr;
        void *p = it->second.back();
        it->second.pop_back();
        return p;
    }
    void release(int dev) {
        std::lock_guard<std::mutex> lk(mu_);
        std::lock_guard<std::mutex> cl(capture_mutex());
        cudaDeviceSynchronize();
        for (auto *m : {&ready_, &pending_})
            for (auto &kv : *m) {
                if (kv.first.first != dev && kv.first.first != -1 - dev) continue;
                for (void *p : kv.second) {
                    if (kv.first.first < 0) cudaFreeHost(p);
                    else cudaFree(p);
                }
                kv.second.clear();
            }
    }
    std::mutex mu_;
    std::map<Key, std::vector<void *>> ready_, pending_;
    std::unordered_map<void *, Key> live_;
};

BlockCache &block_cache() {
    static BlockCache *c = new BlockCache();  // outlives every static destructor
    return *c;
}

template <typename T>
int dmalloc(T **p, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e;
    *p = (T *)block_cache().alloc(sizeof(T) * count, false, &e);
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error(std::string("device allocation failed: ") + cudaGetErrorString(e));
        return SILVAN_E_OOM;
    }
    return SILVAN_OK;
}
template <typename T>
void dfree(T *&p) {
    block_cache().free((void *)p);
    p = nullptr;
}
template <typename T>
int hmalloc(T **p, size_t count) {
    const size_t bytes = sizeof(T) * std::max<size_t>(count, 1);
    cudaError_t e;
    *p = (T *)block_cache().alloc(bytes, true, &e);
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error("pinned host allocation failed");
        return SILVAN_E_OOM;
    }
    std::memset((void *)*p, 0, bytes);
    return SILVAN_OK;
}
template <typename T>
void hfree(T *&p) {
    block_cache().free((void *)p);
    p = nullptr;
}
}  // namespace

int device_alloc(void **p, size_t bytes) {
    cudaError_t e;
    *p = block_cache().alloc(bytes ? bytes : 1, false, &e);
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error(std::string("device allocation failed: ") + cudaGetErrorString(e));
        return SILVAN_E_OOM;
    }
    return SILVAN_OK;
}

void device_free(void *p) { block_cache().free(p); }

void set_error(const std::string &msg) { g_err = msg; }
const char *last_error_cstr() { return g_err.c_str(); }

int cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return SILVAN_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? SILVAN_E_OOM : SILVAN_E_CUDA;
}

#define CK(expr)                              \
    do {                                      \
        int _rc = cuda_status((expr), #expr); \
        if (_rc != SILVAN_OK) return _rc;     \
    } while (0)
#define RK(expr)                          \
    do {                                  \
        int _rc = (expr);                 \
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
    has_host = true;
    n = h.n;
    directed = h.directed;
    m = h.num_edges();
    m_in = h.directed ? h.in_adj.size() : m;
    if (h.n < 2) {
        set_error("graph needs at least two nodes");
        return SILVAN_E_BADARG;
    }
    if (h.num_edges() >= 0xffffffffull || (h.directed && h.in_adj.size() >= 0xffffffffull)) {
        set_error("graphs with 2^32 or more edge entries are not supported");
        return SILVAN_E_BADARG;
    }
    CK(cudaGetDevice(&device));
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
    return make_rows(cudaStreamLegacy);
}

int DeviceGraph::make_rows(cudaStream_t stream) {
    RK(dmalloc(&d_out_rows, n));
    CK(silvan::make_rows(d_out_off, d_out_rows, n, stream));
    if (d_in_off != d_out_off) {
        RK(dmalloc(&d_in_rows, n));
        CK(silvan::make_rows(d_in_off, d_in_rows, n, stream));
    } else {
        d_in_rows = d_out_rows;
    }
    CK(cudaStreamSynchronize(stream));
    return SILVAN_OK;
}

int DeviceGraph::finish_from_host_copy() {
    // The component numbers are the completion order of the reference's
    // sequential depth-first search (the host copy of the out-rows); the
    // diameter bound over them runs on the device.
    const double t0 = now_seconds();
    ncomp = compute_scc(host, cc);
    RK(dmalloc(&d_cc, n));
    CK(cudaMemcpy(d_cc, cc.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    RK(device_directed_bound(*this, cudaStreamLegacy));
    diameter_seconds = now_seconds() - t0;
    return SILVAN_OK;
}

int DeviceGraph::upload_raw(uint32_t nn, bool dir, const uint64_t *out_off,
                            const uint32_t *out_adj, const uint64_t *in_off,
                            const uint32_t *in_adj, const uint32_t *cc_in) {
    has_host = false;
    n = nn;
    directed = dir;
    m = out_off[nn];
    m_in = dir ? in_off[nn] : m;
    if (nn < 2) {
        set_error("graph needs at least two nodes");
        return SILVAN_E_BADARG;
    }
    if (m >= 0xffffffffull || m_in >= 0xffffffffull) {
        set_error("graphs with 2^32 or more edge entries are not supported");
        return SILVAN_E_BADARG;
    }
    CK(cudaGetDevice(&device));
    // Every copy goes up in order on one stream: one copy engine runs at the
    // link's full rate (55 GB/s from pinned memory on a B200 host), where
    // two streams of copies shared it at 49 GB/s.  The offsets and the
    // components go first, the adjacency after them; the offsets' narrowing
    // and the row table run on a second stream as soon as the offsets have
    // landed, and each direction's row check as soon as its adjacency has.
    cudaStream_t cs = nullptr, ks = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t *tmp[2] = {nullptr, nullptr};
    uint32_t *bad = nullptr;
    struct Cleanup {
        cudaStream_t *cs, *ks;
        cudaEvent_t *ev;
        uint64_t **tmp;
        uint32_t **bad;
        ~Cleanup() {
            for (cudaStream_t *s : {cs, ks})
                if (*s) {
                    cudaStreamSynchronize(*s);
                    cudaStreamDestroy(*s);
                }
            for (int i = 0; i < 4; i++)
                if (ev[i]) cudaEventDestroy(ev[i]);
            dfree(tmp[0]);
            dfree(tmp[1]);
            dfree(*bad);
        }
    } cleanup{&cs, &ks, ev, tmp, &bad};
    CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&ks, cudaStreamNonBlocking));
    for (int i = 0; i < 4; i++) CK(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
    RK(dmalloc(&tmp[0], (size_t)nn + 1));
    RK(dmalloc(&bad, 1));
    RK(dmalloc(&d_cc, nn));
    RK(dmalloc(&d_out_off, (size_t)nn + 1));
    RK(dmalloc(&d_out_adj, m));
    if (dir) {
        RK(dmalloc(&tmp[1], (size_t)nn + 1));
        RK(dmalloc(&d_in_off, (size_t)nn + 1));
        RK(dmalloc(&d_in_adj, m_in));
    }
    CK(cudaMemsetAsync(bad, 0, sizeof(uint32_t), ks));
    CK(cudaMemcpyAsync(tmp[0], out_off, sizeof(uint64_t) * (nn + 1), cudaMemcpyHostToDevice, cs));
    CK(cudaEventRecord(ev[0], cs));
    if (dir) {
        CK(cudaMemcpyAsync(tmp[1], in_off, sizeof(uint64_t) * (nn + 1), cudaMemcpyHostToDevice,
                           cs));
        CK(cudaEventRecord(ev[1], cs));
    }
    CK(cudaMemcpyAsync(d_cc, cc_in, sizeof(uint32_t) * nn, cudaMemcpyHostToDevice, cs));
    if (m) CK(cudaMemcpyAsync(d_out_adj, out_adj, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, cs));
    CK(cudaEventRecord(ev[2], cs));
    if (dir) {
        if (m_in)
            CK(cudaMemcpyAsync(d_in_adj, in_adj, sizeof(uint32_t) * m_in, cudaMemcpyHostToDevice,
                               cs));
        CK(cudaEventRecord(ev[3], cs));
    } else {
        d_in_off = d_out_off;
        d_in_adj = d_out_adj;
    }
    CK(cudaStreamWaitEvent(ks, ev[0], 0));
    CK(narrow_offsets(tmp[0], d_out_off, nn + 1, m, bad, ks));
    if (dir) {
        CK(cudaStreamWaitEvent(ks, ev[1], 0));
        CK(narrow_offsets(tmp[1], d_in_off, nn + 1, m_in, bad, ks));
    }
    RK(make_rows(ks));  // waits for the offsets only; the adjacency is still going up
    CK(cudaStreamWaitEvent(ks, ev[2], 0));
    CK(validate_rows(d_out_off, d_out_adj, nn, bad, ks));
    if (dir) {
        CK(cudaStreamWaitEvent(ks, ev[3], 0));
        CK(validate_rows(d_in_off, d_in_adj, nn, bad, ks));
    }
    uint32_t hbad = 0;
    CK(cudaMemcpyAsync(&hbad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, ks));
    CK(cudaStreamSynchronize(ks));
    CK(cudaStreamSynchronize(cs));
    if (hbad) {
        set_error("CSR rows must hold ascending unique ids < n");
        return SILVAN_E_BADARG;
    }
    return SILVAN_OK;
}

uint64_t DeviceGraph::device_bytes() const {
    uint64_t b = 4ull * (n + 1) + 4ull * m + 4ull * n + 8ull * n;
    if (directed) b += 4ull * (n + 1) + 4ull * m_in + 8ull * n;
    return b;
}

DeviceGraph::~DeviceGraph() {
    if (d_in_rows != d_out_rows) dfree(d_in_rows);
    d_in_rows = nullptr;
    dfree(d_out_rows);
    if (d_in_off != d_out_off) dfree(d_in_off);
    if (d_in_adj != d_out_adj) dfree(d_in_adj);
    d_in_off = d_in_adj = nullptr;
    dfree(d_out_off);
    dfree(d_out_adj);
    dfree(d_cc);
}

// ---------------------------------------------------------------------------
// SlotPool
// ---------------------------------------------------------------------------
uint64_t SlotPool::bytes_per_slot(uint64_t n) {
    return n * (sizeof(NodeRec) + 12) + (uint64_t)kMeetCap * 16;
}

int SlotPool::alloc(uint32_t s, uint64_t nn, cudaStream_t st) {
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
    CK(cudaStreamSynchronize(st));
    return SILVAN_OK;
}

void SlotPool::free_all() {
    dfree(rec);
    dfree(queue);
    dfree(hits);
    dfree(touched);
    dfree(meet);
    dfree(meet_pre);
    slots = 0;
}

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
Engine::~Engine() {
    if (stream_) cudaStreamSynchronize(stream_);
    drop_execs();
    dfree(d_hdr_);
    dfree(d_segs_);
    dfree(d_cursors_);
    hfree(h_hdr_);
    hfree(h_segs_);
    hfree(h_cursors_);
    for (auto &e : ev_)
        if (e) cudaEventDestroy(e);
    slots_.free_all();
    device_free(board_mem_);
    if (stream_) cudaStreamDestroy(stream_);
}

int Engine::init(uint64_t n_max, uint32_t slots, uint64_t mem_budget) {
    CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    {
        int dev = 0, khz = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev));
        clock_khz_ = khz;
    }
    for (auto &e : ev_) CK(cudaEventCreate(&e));
    int sms = 0;
    {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    uint32_t resident[kNB];
    uint32_t most = 0;
    for (int b = 0; b < kNB; b++) {
        resident[b] = (uint32_t)sms * (uint32_t)std::max(0, sampler_max_ctas_per_sm(kSamplerBlocks[b]));
        most = std::max(most, resident[b]);
    }
    if (slots == 0) slots = std::max<uint32_t>(most, 1);
    if (mem_budget == 0) {
        // half of the free memory, counting the blocks this process freed
        // and keeps for reuse (an engine created after another one would
        // otherwise see half of the previous budget, and so on)
        size_t fr = 0, tot = 0;
        int dev = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaMemGetInfo(&fr, &tot));
        mem_budget = (fr + block_cache().idle_bytes(dev)) / 2;
    }
    const uint64_t fit = mem_budget / std::max<uint64_t>(SlotPool::bytes_per_slot(n_max), 1);
    if (fit < slots) slots = (uint32_t)std::max<uint64_t>(fit, 1);
    RK(slots_.alloc(slots, n_max, stream_));
    RK(device_alloc(&board_mem_, assist_board_bytes(n_max)));
    CK(assist_board_init(&board_, board_mem_, n_max, stream_));
    for (int b = 0; b < kNB; b++) max_grid_[b] = std::min(resident[b], slots);
    RK(dmalloc(&d_hdr_, 1));
    RK(hmalloc(&h_hdr_, 1));
    return ensure_segs(64);
}

int Engine::ensure_segs(uint32_t nsegs) {
    if (nsegs <= max_segs_) return SILVAN_OK;
    uint32_t cap = std::max<uint32_t>(64, max_segs_);
    while (cap < nsegs) cap *= 2;
    dfree(d_segs_);
    dfree(d_cursors_);
    hfree(h_segs_);
    hfree(h_cursors_);
    RK(dmalloc(&d_segs_, cap));
    RK(dmalloc(&d_cursors_, cap));
    RK(hmalloc(&h_segs_, cap));
    RK(hmalloc(&h_cursors_, cap));
    max_segs_ = cap;
    drop_execs();
    return SILVAN_OK;
}

void Engine::drop_execs() {
    for (Exec &x : execs_) cudaGraphExecDestroy(x.exec);
    execs_.clear();
}

// The round's two kernels (round_begin + sampler) captured once per (CTA
// size, grid) and replayed with new segments.
int Engine::sampler_exec(int block, uint32_t grid, cudaGraphExec_t *out) {
    for (const Exec &x : execs_)
        if (x.block == block && x.grid == grid) {
            *out = x.exec;
            return SILVAN_OK;
        }
    SamplerLaunch L{};
    L.slots = SlotArrays{slots_.rec,  slots_.queue,    slots_.hits, slots_.touched,
                         slots_.meet, slots_.meet_pre, slots_.n};
    L.hdr = d_hdr_;
    L.segs = d_segs_;
    L.assist = board_;
    cudaGraph_t g = nullptr;
    std::lock_guard<std::mutex> cl(capture_mutex());
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    cudaError_t e1 = sampler_round_begin(L, max_segs_, stream_);
    cudaError_t e2 = sampler_launch(L, grid, stream_, block);
    cudaError_t e3 = cudaStreamEndCapture(stream_, &g);
    CK(e1);
    CK(e2);
    CK(e3);
    cudaGraphExec_t x = nullptr;
    cudaError_t e4 = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    CK(e4);
    if (execs_.size() >= 16) drop_execs();
    execs_.push_back(Exec{block, grid, x});
    *out = x;
    return SILVAN_OK;
}

// Autotuned CTA size of a round.  Every CTA size is tried once on each class
// of graphs (the samples are the same whichever size draws them); after that the round
// takes the size with the least predicted time: the slowest sample of the
// round, or the CTA time of all its samples spread over the resident CTAs,
// whichever is longer.
int Engine::choose_block(const std::vector<Job *> &jobs, const std::vector<JobRequest> &reqs,
                         const std::vector<uint32_t> &idx, uint32_t total) const {
    const silvan_params_t &p0 = jobs[idx[0]]->params();
    if (p0.block) return (int)p0.block;
    if (p0.form == SILVAN_FORM_PLAIN) return kSamplerBlock;
    static const int order[kNB] = {2, 1, 0, 3};  // 512, 256, 128, 1024
    for (int oi = 0; oi < kNB; oi++) {
        const int b = order[oi];
        if (!max_grid_[b]) continue;
        for (uint32_t i : idx) {
            auto it = stats_.find(jobs[i]->graph()->tune_class());
            if (it == stats_.end() || it->second[b].rounds == 0) return kSamplerBlocks[b];
        }
    }
    int best = kSamplerBlock;
    double best_t = 1e300;
    for (int b = 0; b < kNB; b++) {
        if (!max_grid_[b]) continue;
        double tail = 0, work = 0;
        for (uint32_t i : idx) {
            const BlockStats &st = stats_.at(jobs[i]->graph()->tune_class())[b];
            tail = std::max(tail, st.tail_ms);
            work += reqs[i].count * st.cta_ms;
        }
        const double t = std::max(tail, work / std::min(max_grid_[b], total));
        if (t < best_t) {
            best_t = t;
            best = kSamplerBlocks[b];
        }
    }
    return best;
}

void Engine::fair_share(const std::vector<Job *> &jobs, std::vector<JobRequest> &reqs,
                        double round_ms) const {
    const size_t n = jobs.size();
    if (n < 2) return;
    std::vector<double> cost(n, 0.0);
    uint32_t grid = 0;
    for (int b = 0; b < kNB; b++) grid = std::max(grid, max_grid_[b]);
    for (size_t i = 0; i < n; i++) {
        auto it = stats_.find(jobs[i]->graph()->tune_class());
        if (it == stats_.end()) return;
        double best = 0;
        for (int b = 0; b < kNB; b++) {
            const BlockStats &st = it->second[b];
            if (st.rounds && max_grid_[b] && (best == 0 || st.cta_ms / max_grid_[b] < best))
                best = st.cta_ms / max_grid_[b];
        }
        if (best <= 0) return;
        cost[i] = best * grid;  // CTA ms per sample at the best CTA size
    }
    std::vector<size_t> order(n);
    for (size_t i = 0; i < n; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        return reqs[a].count * cost[a] < reqs[b].count * cost[b];
    });
    double left = round_ms * grid;
    for (size_t k = 0; k < n; k++) {
        const size_t i = order[k];
        const double share = left / (double)(n - k);
        const double need = reqs[i].count * cost[i];
        if (need > share) {
            const uint32_t c = (uint32_t)std::max<double>(kBlock, std::floor(share / cost[i]));
            reqs[i].count = std::min(reqs[i].count, c);
        }
        left = std::max(0.0, left - reqs[i].count * cost[i]);
    }
}

uint32_t Engine::main_block() const {
    int b = 2;
    for (int i = 0; i < kNB; i++)
        if (block_samples_[i] > block_samples_[b]) b = i;
    return (uint32_t)kSamplerBlocks[b];
}

uint64_t DeviceGraph::tune_class() const {
    auto lg = [](uint64_t x) {
        uint64_t r = 0;
        while (x > 1) {
            x >>= 1;
            r++;
        }
        return r;
    };
    return (directed ? 1ull : 0ull) | lg(n) << 1 | lg(n ? m / n : 0) << 8;
}

int Engine::round(const std::vector<Job *> &jobs, const std::vector<JobRequest> &reqs,
                  std::vector<uint64_t> &records) {
    std::vector<uint32_t> idx;
    for (uint32_t i = 0; i < jobs.size(); i++)
        if (reqs[i].count > 0) idx.push_back(i);
    records.assign(jobs.size(), 0);
    if (idx.empty()) return SILVAN_OK;
    RK(ensure_segs((uint32_t)idx.size()));
    auto fill = [&](uint32_t s, uint32_t j, uint32_t base) {
        Job *job = jobs[j];
        const JobRequest &r = reqs[j];
        const DeviceGraph &G = *job->graph();
        RoundBuffers &rb = job->round_buffers();
        SegDesc &S = h_segs_[s];
        S.out_off = G.d_out_off;
        S.out_rows = G.d_out_rows;
        S.in_rows = G.d_in_rows;
        S.out_adj = G.d_out_adj;
        S.in_off = G.d_in_off;
        S.in_adj = G.d_in_adj;
        S.cc = G.d_cc;
        S.n = G.n;
        S.directed = G.directed ? 1 : 0;
        S.seed = job->params().seed;
        S.alpha = r.alpha;
        S.np_cap = job->params().np_cap;
        S.weighted = job->params().backtrack == SILVAN_BACKTRACK_SIGMA_WEIGHTED ? 1 : 0;
        {
            const uint32_t ai = job->params().assist_items;
            S.assist_items = ai == 0u ? kAssistItemsAuto : (ai == 0xffffffffu ? 0u : ai);
        }
        S.first_sample = r.first_global;
        S.count = r.count;
        S.base = base;
        S.out_pl = rb.pl;
        S.out_np = rb.np;
        S.out_vis = rb.vis;
        S.out_status = rb.status;
        S.out_ball = rb.ball;
        S.out_pred = rb.pred;
        S.recs = rb.recs;
        S.rec_cursor = d_cursors_ + s;
        S.rec_cap = rb.rec_cap;
    };
    uint32_t total = 0;
    for (uint32_t s = 0; s < idx.size(); s++) {
        const JobRequest &r = reqs[idx[s]];
        if (r.count > kRoundSamples || jobs[idx[s]]->graph()->n > slots_.n) {
            set_error("request larger than the round buffers or graph larger than the slots");
            return SILVAN_E_BADARG;
        }
        fill(s, idx[s], total);
        total += r.count;
    }
    // the round's wait limit: the smallest any of its jobs asks for
    uint32_t polls = kDefaultWaitPolls;
    for (uint32_t i : idx) {
        const uint32_t w = jobs[i]->params().wait_polls;
        polls = std::min(polls, w == 0u ? kDefaultWaitPolls : (w == 0xffffffffu ? 0u : w));
    }
    h_hdr_->nsegs = (uint32_t)idx.size();
    h_hdr_->total = total;
    h_hdr_->work = 0;
    h_hdr_->cycles = 0;
    h_hdr_->max_cycles = 0;
    h_hdr_->wait_polls = polls;
    const int block = choose_block(jobs, reqs, idx, total);
    int bi = -1;
    for (int b = 0; b < kNB; b++)
        if (kSamplerBlocks[b] == block && max_grid_[b]) bi = b;
    if (bi < 0) {
        set_error("sampler CTA size must be 128, 256, 512 or 1024 threads");
        return SILVAN_E_BADARG;
    }
    const uint32_t grid = std::min<uint32_t>(max_grid_[bi], total);
    cudaGraphExec_t exec = nullptr;
    RK(sampler_exec(block, grid, &exec));
    for (;;) {
        CK(cudaMemcpyAsync(d_segs_, h_segs_, sizeof(SegDesc) * idx.size(),
                           cudaMemcpyHostToDevice, stream_));
        CK(cudaMemcpyAsync(d_hdr_, h_hdr_, sizeof(RoundHeader), cudaMemcpyHostToDevice, stream_));
        CK(cudaEventRecord(ev_[0], stream_));
        CK(cudaGraphLaunch(exec, stream_));
        CK(cudaEventRecord(ev_[1], stream_));
        launches_ += 2;
        sampler_launches_++;
        CK(cudaMemcpyAsync(h_cursors_, d_cursors_, sizeof(unsigned long long) * idx.size(),
                           cudaMemcpyDeviceToHost, stream_));
        CK(cudaMemcpyAsync(h_hdr_, d_hdr_, sizeof(RoundHeader), cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
        if (h_hdr_->failed > 0 || h_hdr_->finished < total) {
            // A shared level gave up a wait: its records may be left
            // non-neutral and the CTAs that owned them left the launch.  Every
            // slot is re-initialised (the launch has ended, so nothing writes
            // to them any more) before any later round uses it.  The samples
            // concerned carry SILVAN_E_TIMEOUT into their jobs' commits; if
            // samples were left undrawn, the whole round fails.
            CK(sampler_init_slots(slots_.rec, slots_.hits, (uint64_t)slots_.slots * slots_.n,
                                  stream_));
            CK(cudaStreamSynchronize(stream_));
            slot_resets_++;
            if (h_hdr_->finished < total) {
                set_error("sampler round ended with samples undrawn (waits between CTAs "
                          "that share a level gave up)");
                return SILVAN_E_TIMEOUT;
            }
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, ev_[0], ev_[1]);
        sample_ms_ += ms;
        block_samples_[bi] += total;
        assisted_levels_ += h_hdr_->assisted;
        helper_tiles_ += h_hdr_->helper_tiles;
        // cost model of the CTA-size choice and of speculative draws: a launch
        // lasts about as long as its slowest sample, so the samples that fit
        // into that time on the other slots cost (almost) nothing extra
        if (h_hdr_->total > 0 && clock_khz_ > 0) {
            const double cta_ms = (double)h_hdr_->cycles / clock_khz_ / h_hdr_->total;
            const double tail_ms = (double)h_hdr_->max_cycles / clock_khz_;
            for (uint32_t i : idx)
                last_[jobs[i]->graph()->tune_class()] = LastLaunch{cta_ms, tail_ms, ms, grid, total};
            for (uint32_t i : idx) {
                // the slowest sample of a launch grows with the launch's size
                // and is rare: the estimate follows a longer tail at once and
                // a shorter one slowly
                BlockStats &st = stats_[jobs[i]->graph()->tune_class()][bi];
                st.cta_ms = st.rounds ? 0.5 * (st.cta_ms + cta_ms) : cta_ms;
                st.tail_ms = (!st.rounds || tail_ms > st.tail_ms) ? tail_ms
                                                                  : 0.75 * st.tail_ms + 0.25 * tail_ms;
                st.rounds++;
            }
        }
        bool redo = false;
        uint32_t base = 0;
        for (uint32_t s = 0; s < idx.size(); s++) {
            Job *job = jobs[idx[s]];
            if (h_cursors_[s] > job->round_buffers().rec_cap) {
                uint64_t cap = job->round_buffers().rec_cap;
                while (cap < h_cursors_[s]) cap *= 2;
                RK(job->grow_records(cap));
                redo = true;
            }
            fill(s, idx[s], base);
            base += reqs[idx[s]].count;
        }
        if (!redo) break;
        // the path maps did not fit: redraw the round (deterministic)
        h_hdr_->nsegs = (uint32_t)idx.size();
        h_hdr_->total = total;
        h_hdr_->work = 0;
        h_hdr_->cycles = 0;
        h_hdr_->max_cycles = 0;
        h_hdr_->wait_polls = polls;
    }
    for (uint32_t s = 0; s < idx.size(); s++) records[idx[s]] = h_cursors_[s];
    return SILVAN_OK;
}

// Samples the first launch of the next job of this class draws.  Seeds stop
// at different schedule points (on R-MAT scale 20 the totals of 60 seeds
// spread over +-13 % of their mean), so one earlier total is a noisy guess:
// with fewer than kHintMin totals recorded, 25 % above the last one; with
// more, 3 % above the largest of the last kHintJobs, which about one job in
// kHintJobs + 1 exceeds (it then draws its rest in a second launch).
uint64_t Engine::job_hint(const DeviceGraph *G) const {
    auto it = job_total_.find(G->tune_class());
    if (it == job_total_.end() || it->second.empty()) return 0;
    const std::deque<uint64_t> &h = it->second;
    if (h.size() < kHintMin) return h.back() + h.back() / 4;
    const uint64_t mx = *std::max_element(h.begin(), h.end());
    return mx + mx / 32;
}

void Engine::note_job(const DeviceGraph *G, uint64_t used, bool alpha_kept) {
    // only a job whose second pass kept the first pass's alpha can use
    // samples drawn ahead in its first launch
    if (!alpha_kept) {
        job_total_.erase(G->tune_class());
        return;
    }
    std::deque<uint64_t> &h = job_total_[G->tune_class()];
    h.push_back(used);
    while (h.size() > kHintJobs) h.pop_front();
}

uint32_t Engine::free_samples(const DeviceGraph *G, bool tail_only) const {
    // the samples the other slots draw while the slowest sample runs, or
    // while the whole last launch ran (a throughput-bound launch feeds its own
    // length back, so that estimate needs a cap from the caller)
    auto it = last_.find(G->tune_class());
    if (it == last_.end()) return 0;
    const LastLaunch &l = it->second;
    const double t = tail_only ? l.tail_ms : l.launch_ms;
    if (l.cta_ms <= 0 || t <= 0) return 0;
    double f = t * l.grid / l.cta_ms;
    // a launch longer than its work (a long tail) predicts many free samples;
    // the next launch may not have that tail, so the estimate grows by at
    // most a factor of two per launch
    if (!tail_only) f = std::min(f, 2.0 * l.samples);
    return (uint32_t)std::min<double>(f, (double)kRoundSamples);
}

// ---------------------------------------------------------------------------
// Engine pool
// ---------------------------------------------------------------------------
namespace {
struct PooledEngine {
    int device;
    uint32_t requested_slots;
    Engine *eng;
};
std::mutex g_pool_mu;
std::vector<PooledEngine> g_pool_free;
std::vector<PooledEngine> g_pool_busy;
}  // namespace

Engine *engine_acquire(uint64_t n, uint32_t slots, int *rc) {
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        for (size_t i = 0; i < g_pool_free.size(); i++) {
            PooledEngine &p = g_pool_free[i];
            if (p.device == dev && p.eng->n_max() >= n && p.requested_slots == slots) {
                PooledEngine q = p;
                g_pool_free.erase(g_pool_free.begin() + i);
                g_pool_busy.push_back(q);
                *rc = SILVAN_OK;
                return q.eng;
            }
        }
    }
    Engine *e = new Engine();
    *rc = e->init(n, slots, 0);
    if (*rc != SILVAN_OK) {
        // release idle engines of this device and try once more
        std::vector<Engine *> drop;
        {
            std::lock_guard<std::mutex> lk(g_pool_mu);
            for (size_t i = 0; i < g_pool_free.size();)
                if (g_pool_free[i].device == dev) {
                    drop.push_back(g_pool_free[i].eng);
                    g_pool_free.erase(g_pool_free.begin() + i);
                } else {
                    i++;
                }
        }
        for (Engine *d : drop) delete d;
        delete e;
        e = new Engine();
        *rc = e->init(n, slots, 0);
        if (*rc != SILVAN_OK) {
            delete e;
            return nullptr;
        }
    }
    std::lock_guard<std::mutex> lk(g_pool_mu);
    g_pool_busy.push_back(PooledEngine{dev, slots, e});
    return e;
}

void engine_release(Engine *e) {
    if (!e) return;
    cudaStreamSynchronize(e->stream());
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (size_t i = 0; i < g_pool_busy.size(); i++)
        if (g_pool_busy[i].eng == e) {
            g_pool_free.push_back(g_pool_busy[i]);
            g_pool_busy.erase(g_pool_busy.begin() + i);
            return;
        }
}

int Job::borrow_engine() {
    if (own_engine_) return SILVAN_OK;
    int rc = SILVAN_OK;
    own_engine_ = engine_acquire(n_, p_.slots, &rc);
    return rc;
}

void Job::return_engine() {
    if (!own_engine_) return;
    engine_release(own_engine_);
    own_engine_ = nullptr;
}

// ---------------------------------------------------------------------------
// Job: allocation and commit
// ---------------------------------------------------------------------------
Job::~Job() {
    if (own_engine_) cudaStreamSynchronize(own_engine_->stream());
    return_engine();
    stream_ = nullptr;
    RoundBuffers &r = rb_;
    dfree(r.pl);
    dfree(r.np);
    dfree(r.vis);
    dfree(r.status);
    dfree(r.signs);
    dfree(r.ball);
    dfree(r.pred);
    dfree(r.inv_np);
    dfree(r.recs);
    dfree(r.node_cnt);
    dfree(r.touched);
    dfree(r.large);
    dfree(r.n_touched);
    dfree(r.bucket_off);
    dfree(r.bucket_len);
    dfree(r.entries);
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
    dfree(jc_.upd_list);
    dfree(d_red_);
    dfree(d_ticket_);
    dfree(d_unc_);
    dfree(d_nunc_);
    dfree(d_lut_);
    dfree(d_hist_);
    hfree(h_lut_);
    hfree(h_hist_);
    hfree(h_nunc_);
    dfree(jr_.mcrade);
    dfree(jr_.approx);
    dfree(jr_.wimpy);
    dfree(jr_.last_upd);
    dfree(jr_.sc);
    dfree(jr_.sp_lengths);
    if (ev_chk_) cudaEventDestroy(ev_chk_);
    dfree(tk_.hist);
    dfree(tk_.state);
    dfree(tk_.cand);
    hfree(tk_.h_state);
    hfree(tk_.h_cand);
    hfree(h_red_);
    hfree(h_sc_);
    hfree(h_sp_);
    for (auto &e : ev_run_)
        if (e) cudaEventDestroy(e);
    for (auto &e : ev_commit_)
        if (e) cudaEventDestroy(e);
}

int Job::alloc_round(uint32_t max_samples, uint64_t rec_cap) {
    RoundBuffers &r = rb_;
    r.max_samples = max_samples;
    RK(dmalloc(&r.pl, max_samples));
    RK(dmalloc(&r.np, max_samples));
    RK(dmalloc(&r.vis, max_samples));
    RK(dmalloc(&r.status, max_samples));
    RK(dmalloc(&r.signs, max_samples));
    RK(dmalloc(&r.ball, max_samples));
    RK(dmalloc(&r.pred, max_samples));
    RK(dmalloc(&r.node_cnt, n_));
    RK(dmalloc(&r.n_touched, 8));
    CK(cudaMemset(r.n_touched, 0, 8 * sizeof(uint32_t)));
    RK(dmalloc(&r.inv_np, max_samples));
    r.n_large = r.n_touched + 1;
    r.rec_cursor = nullptr;
    r.work_counter = nullptr;
    CK(cudaMemset(r.node_cnt, 0, sizeof(uint32_t) * n_));
    return grow_records(rec_cap);
}

int Job::grow_records(uint64_t cap) {
    RoundBuffers &r = rb_;
    if (stream_) cudaStreamSynchronize(stream_);
    dfree(r.recs);
    dfree(r.touched);
    dfree(r.large);
    dfree(r.bucket_off);
    dfree(r.bucket_len);
    dfree(r.entries);
    r.rec_cap = cap;
    const uint64_t tcap = std::min<uint64_t>(cap, n_) + 1;
    RK(dmalloc(&r.recs, cap));
    RK(dmalloc(&r.touched, tcap));
    RK(dmalloc(&r.large, tcap));
    RK(dmalloc(&r.bucket_off, tcap + 1));
    RK(dmalloc(&r.bucket_len, tcap));
    RK(dmalloc(&r.entries, cap));
    return SILVAN_OK;
}

uint64_t Job::device_bytes() const {
    const uint64_t n = n_;
    uint64_t b = n * (8 + 8 + 8 * kTrials + 4 + 1 + 4 + 4 + 4 + 4);
    if (p_.k == 0) b += n * (8 * kTrials + 8 + 8 + 4);  // the round journal
    b += (uint64_t)kRoundSamples * 36 + rb_.rec_cap * (12 + 8) +
         std::min<uint64_t>(rb_.rec_cap, n) * 8;
    return b;
}

int Job::init() {
    n_ = g_->n;
    if (!(p_.eps > 0 && p_.eps < 1) || !(p_.delta > 0 && p_.delta < 1)) {
        set_error("eps and delta must lie in (0, 1)");
        return SILVAN_E_BADARG;
    }
    if (p_.block != 0 && p_.block != 128 && p_.block != 256 && p_.block != 512 &&
        p_.block != 1024) {
        set_error("block must be 0 (autotuned), 128, 256, 512 or 1024");
        return SILVAN_E_BADARG;
    }
    if (p_.backtrack != SILVAN_BACKTRACK_REFERENCE &&
        p_.backtrack != SILVAN_BACKTRACK_SIGMA_WEIGHTED) {
        set_error("backtrack must be SILVAN_BACKTRACK_REFERENCE or SILVAN_BACKTRACK_SIGMA_WEIGHTED");
        return SILVAN_E_BADARG;
    }
    if (p_.np_cap == 0) p_.np_cap = 1u << 24;
    for (auto &e : ev_run_) CK(cudaEventCreate(&e));
    for (auto &e : ev_commit_) CK(cudaEventCreate(&e));
    RK(alloc_round(kRoundSamples, kInitialRecords));
    const uint32_t n = n_;
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
    RK(dmalloc(&jc_.upd_list, n));
    if (p_.k == 0) {
        RK(dmalloc(&jr_.mcrade, (uint64_t)n * kTrials));
        RK(dmalloc(&jr_.approx, n));
        RK(dmalloc(&jr_.wimpy, n));
        RK(dmalloc(&jr_.last_upd, n));
        RK(dmalloc(&jr_.sc, 1));
        RK(dmalloc(&jr_.sp_lengths, (uint64_t)g_->diameter + 1));
        CK(cudaEventCreateWithFlags(&ev_chk_, cudaEventDisableTiming));
    }
    RK(dmalloc(&d_red_, 1));
    RK(dmalloc(&d_ticket_, 1));
    RK(dmalloc(&d_unc_, kUncertainCap));
    RK(dmalloc(&d_nunc_, 1));
    RK(hmalloc(&h_red_, 1));
    RK(hmalloc(&h_sc_, 1));
    RK(hmalloc(&h_sp_, (size_t)g_->diameter + 1));
    RK(hmalloc(&h_nunc_, 1));
    // the check kernel writes its results straight into these pinned buffers
    CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&readback_.red), h_red_, 0));
    CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&readback_.sc), h_sc_, 0));
    CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&readback_.sp), h_sp_, 0));
    CK(stop_reduce_init(d_red_, d_ticket_, cudaStreamLegacy));
    CK(cudaMemset(jc_.approx, 0, sizeof(double) * n));
    CK(cudaMemset(jc_.wimpy, 0, sizeof(double) * n));
    CK(cudaMemset(jc_.mcrade, 0, sizeof(long long) * (uint64_t)n * kTrials));
    CK(cudaMemset(jc_.last_upd, 0, sizeof(uint32_t) * n));
    CK(cudaMemset(jc_.cross_flag, 0, n));
    CK(cudaMemset(jc_.sp_lengths, 0, sizeof(uint64_t) * (g_->diameter + 1)));
    CK(cudaMemset(jc_.sc, 0, sizeof(JobScalars)));
    CK(cudaMemset(jc_.partition, 0, sizeof(int32_t) * n));
    CK(apply_init());
    // the set-up above ran on the legacy stream (a whole-device synchronisation
    // here could meet another thread's graph capture)
    CK(cudaStreamSynchronize(cudaStreamLegacy));
    return SILVAN_OK;
}

// Commits samples [lo, hi) (indices into the drawn range r) whose raw outputs
// the engine left in rb_, in apply sub-rounds of at most kLargeBucket samples.
int Job::apply_range(const JobRequest &r, uint32_t lo, uint32_t hi, uint64_t n_records,
                     bool journal) {
    if (journal && (hi - lo > kLargeBucket || !jr_.approx)) {
        set_error("a journaled commit round must be a single sub-round");
        return SILVAN_E_STATE;
    }
    for (uint32_t a0 = lo; a0 < hi; a0 += kLargeBucket) {
        ApplyState st{};
        st.rb = rb_;
        st.jc = jc_;
        st.jr = jr_;
        ApplyArgs &a = st.a;
        a.journal = journal ? 1 : 0;
        a.n = n_;
        a.n_records = (uint32_t)n_records;
        a.seed = p_.seed;
        a.first_sample = r.first_global;
        a.lo = a0;
        a.hi = std::min<uint32_t>(hi, a0 + kLargeBucket);
        a.pass = r.pass;
        a.track_cross = r.track_cross ? 1 : 0;
        a.D = g_->diameter;
        CK(apply_round(st, stream_));
        launches += kApplyRoundKernels;
    }
    return SILVAN_OK;
}

// ---------------------------------------------------------------------------
// Job: device reads
// ---------------------------------------------------------------------------
int Job::sync_scalars(JobScalars &sc) {
    CK(cudaMemcpyAsync(h_sc_, jc_.sc, sizeof(JobScalars), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    sc = *h_sc_;
    return scalars_error(sc);
}

int Job::scalars_error(const JobScalars &sc) {
    if (sc.error != 0) {
        const char *what = sc.error == SILVAN_E_OVERFLOW
                               ? "a sample's 64-bit path count wrapped to 0 (the reference "
                                 "divides by zero here)"
                           : sc.error == SILVAN_E_NP_CAP
                               ? "a sample asked for more shortest paths than the job's cap"
                           : sc.error == SILVAN_E_CAPACITY ? "a per-sample buffer overflowed"
                           : sc.error == SILVAN_E_TIMEOUT
                               ? "a bounded wait between GPU thread blocks gave up (a BFS level "
                                 "shared between CTAs, or a grid barrier of the commit)"
                               : "device sampler inconsistency";
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

void Job::flush() {
    if (sink_ && !out_.empty()) {
        fwrite(out_.data(), 1, out_.size(), sink_);
        fflush(sink_);
    }
    out_.clear();
}

// Empirical peeling (silvan/src/Probabilistic.cpp:853-871).
// The end of pass 1 in one round trip: one kernel computes every node's
// peeling index and their histogram (Probabilistic.cpp:853-889) and writes
// the histogram, the scalars (sc1_) and the path-length counts (sp) to
// host-mapped memory.  Nodes whose index the device's log could have moved
// are recomputed with the C library's log, and the histogram again, before
// the partitions are numbered.
int Job::peel(double a, bool enabled, std::vector<uint64_t> &sp) {
    const uint32_t n = n_;
    const uint32_t D = g_->diameter;
    const double ms = (double)pass_samples_;
    part_ids_.clear();
    part_count_.clear();
    auto host_idx = [&](double w) {
        double emp_w = w / ms;
        double min_inv = fmin(1. / emp_w, ms);
        return (int)(log(min_inv) / log(a) + 1);
    };
    int32_t idx_min = 0, nbins = 0;
    if (enabled) {
        // the indices lie in [1, log(m)/log(a) + 1]
        idx_min = std::min(0, host_idx(ms));
        const int32_t idx_max = std::max(host_idx(0.0), host_idx(ms)) + 2;
        nbins = idx_max - idx_min + 1;
        if (nbins > (1 << 22)) {
            set_error("empirical peeling parameter too close to 1");
            return SILVAN_E_BADARG;
        }
        if ((uint32_t)nbins > hist_cap_) {
            dfree(d_hist_);
            hfree(h_hist_);
            dfree(d_lut_);
            hfree(h_lut_);
            RK(dmalloc(&d_hist_, nbins));
            RK(hmalloc(&h_hist_, nbins));
            RK(dmalloc(&d_lut_, nbins));
            RK(hmalloc(&h_lut_, nbins));
            hist_cap_ = (uint32_t)nbins;
        }
    }
    Pass1Readback out{readback_.sc, readback_.sp, nullptr, nullptr};
    CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&out.n_unc), h_nunc_, 0));
    if (enabled) CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&out.hist), h_hist_, 0));
    CK(pass1_readback(jc_, n, ms, a, idx_min, nbins, d_hist_, d_unc_, d_nunc_, kUncertainCap, D,
                      d_ticket_, out, stream_));
    launches += 1;
    CK(cudaStreamSynchronize(stream_));
    sc1_ = *h_sc_;
    RK(scalars_error(sc1_));
    sp.assign(h_sp_, h_sp_ + D + 1);
    if (!enabled) {
        CK(cudaMemsetAsync(jc_.partition, 0, sizeof(int32_t) * n, stream_));
        part_ids_.push_back(0);
        part_count_.push_back(n);
        nparts_ = 1;
        part_host_.assign(n, 0);
        return SILVAN_OK;
    }
    const uint32_t nunc = *h_nunc_;
    std::vector<uint32_t> hist(h_hist_, h_hist_ + nbins);
    if (nunc > 0) {
        if (nunc > kUncertainCap) {
            std::vector<double> w(n);
            std::vector<int32_t> idx(n);
            CK(cudaMemcpy(w.data(), jc_.wimpy, sizeof(double) * n, cudaMemcpyDeviceToHost));
            for (uint32_t i = 0; i < n; i++) idx[i] = host_idx(w[i]);
            CK(cudaMemcpy(jc_.peel_idx, idx.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice));
        } else {
            std::vector<uint32_t> unc(nunc);
            CK(cudaMemcpy(unc.data(), d_unc_, sizeof(uint32_t) * nunc, cudaMemcpyDeviceToHost));
            for (uint32_t v : unc) {
                double w;
                CK(cudaMemcpy(&w, jc_.wimpy + v, sizeof(double), cudaMemcpyDeviceToHost));
                int32_t idx = host_idx(w);
                CK(cudaMemcpy(jc_.peel_idx + v, &idx, sizeof(int32_t), cudaMemcpyHostToDevice));
            }
        }
        CK(peel_hist(jc_, n, idx_min, nbins, d_hist_, stream_));
        launches += 1;
        CK(cudaMemcpyAsync(hist.data(), d_hist_, sizeof(uint32_t) * nbins, cudaMemcpyDeviceToHost,
                           stream_));
        CK(cudaStreamSynchronize(stream_));
    }
    int dense = 0;
    for (int32_t b = 0; b < nbins; b++) {
        h_lut_[b] = 0;
        if (hist[b]) {
            h_lut_[b] = dense++;
            part_ids_.push_back(b + idx_min);
            part_count_.push_back(hist[b]);
        }
    }
    nparts_ = dense;
    if (nparts_ > kMaxPartitions) {
        set_error("more than 128 non-empty peeling partitions");
        return SILVAN_E_BADARG;
    }
    CK(cudaMemcpyAsync(d_lut_, h_lut_, sizeof(int32_t) * nbins, cudaMemcpyHostToDevice, stream_));
    CK(peel_map(jc_, n, d_lut_, idx_min, nbins, nullptr, stream_));
    launches += 1;
    if (!absolute_) {  // the top-k test looks partitions up per ranked node
        part_host_.resize(n);
        CK(cudaMemcpyAsync(part_host_.data(), jc_.partition, sizeof(int32_t) * n,
                           cudaMemcpyDeviceToHost, stream_));
        CK(cudaStreamSynchronize(stream_));
    }
    return SILVAN_OK;
}

// Current ranking list (silvan/src/Ranking_list.cpp): the union_sample nodes
// of largest (approx, last update, id), selected on the device; the
// never-updated nodes of the initial list (ids < union_sample, ascending)
// after the updated ones.
int Job::ranking(std::vector<uint32_t> &el, std::vector<double> &val) {
    const uint32_t K = union_sample_;
    if (!tk_.hist) {
        tk_.cap = topk_capacity(K);
        RK(dmalloc(&tk_.hist, 65536));
        RK(dmalloc(&tk_.state, 8));
        RK(dmalloc(&tk_.cand, 2 * (uint64_t)tk_.cap));
        RK(hmalloc(&tk_.h_state, 8));
        RK(hmalloc(&tk_.h_cand, 2 * (uint64_t)tk_.cap));
    }
    JobScalars sc;
    CK(cudaMemcpyAsync(h_sc_, jc_.sc, sizeof(JobScalars), cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    sc = *h_sc_;
    el.resize(K);
    val.resize(K);
    uint32_t cnt = 0;
    RK(topk_select(jc_, sc.n_upd, K, tk_, stream_, el.data(), val.data(), &cnt));
    el.resize(cnt);
    val.resize(cnt);
    if (cnt < K) {
        // never-updated nodes of the initial list (ids < K) fill the tail
        const uint32_t m = std::min(K, n_);
        std::vector<uint32_t> lu(m);
        CK(cudaMemcpyAsync(lu.data(), jc_.last_upd, sizeof(uint32_t) * m, cudaMemcpyDeviceToHost,
                           stream_));
        CK(cudaStreamSynchronize(stream_));
        for (uint32_t i = 0; i < m && el.size() < K; i++)
            if (lu[i] == 0) {
                el.push_back(i);
                val.push_back(0.0);
            }
    }
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
    const double adu = upper_bound_avg_diameter(sp, (int)g_->diameter, dpb, pass_samples_).ub;
    SmallRanking sub(k_), slb(k_);
    uint32_t ins = 0;
    bool rel = true;
    const uint32_t n = n_;
    for (uint64_t i = 0; i < union_sample_ && i < el.size() && rel; i++) {
        const uint32_t node = el[i];
        const double an = val[i] / ms;
        const double ec = eps_part_[part_host_[node]];
        double lbb = an - ec, ubb = an + ec;
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
                out << "   node_partition_index " << part_ids_[part_host_[node]] << "\n";
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
            const double ec = eps_part_[part_host_[el[i]]];
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
// The device part of a check: one kernel writes the reduction, the
// shortest-path lengths and the scalars to host-mapped memory; ev_chk_ marks
// its end.
int Job::stop_check_enqueue() {
    StopReadback out = readback_;
    if (!absolute_) out.sp = nullptr;
    CK(stop_reduce(jc_, nparts_, g_->diameter, d_red_, d_ticket_, out, stream_));
    launches += 1;
    if (ev_chk_) CK(cudaEventRecord(ev_chk_, stream_));
    return SILVAN_OK;
}

int Job::stop_check(bool &stop) {
    RK(stop_check_enqueue());
    return stop_check_finish(stop);
}

// The host part: waits for the reads of stop_check_enqueue only (work queued
// after them keeps running).
int Job::stop_check_finish(bool &stop) {
    if (ev_chk_) CK(cudaEventSynchronize(ev_chk_));
    else CK(cudaStreamSynchronize(stream_));
    RK(scalars_error(*h_sc_));
    std::ostringstream out;
    checks_++;
    const double ms = (double)pass_samples_;
    double dpb = 1.0;
    if (absolute_ && p_.m_hat) dpb = dfpb_;
    else dpb = p_.delta / pow(2., iteration_);
    out << "\n";
    out << "EVALUATING STOPPING CONDITION at iteration " << iteration_ << " (m=" << pass_samples_
        << ", d=" << dpb << ")" << "\n";
    const StopReduction &R = *h_red_;
    if (absolute_) {
        const std::vector<uint64_t> sp(h_sp_, h_sp_ + g_->diameter + 1);
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
        // nodes never updated in this pass hold mcrade = 0 in every trial
        const bool zeros = R.touched[i] < part_count_[i];
        double avg = 0.0;
        for (int j = 0; j < kTrials; j++) {
            // the reduction starts each maximum at -n_pairs
        const long long mr = std::max(R.mc_max[i * kTrials + j], -(long long)pass_samples_);
        const long long mj = zeros ? std::max(mr, 0ll) : mr;
            avg += mj / (double)kTrials;
        }
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
            // the bound shrinks about as 1 / sqrt(samples): the sample size
            // at which it reaches eps sizes the draws ahead of the stop
            const double r = sup / p_.eps;
            if (r > 1 && r < 1e3) predicted_stop_ = (uint64_t)((double)pass_samples_ * r * r * 1.02);
        }
        out_ += out.str();
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
    out_ += out.str();
    return SILVAN_OK;
}

// Pass 2 starts from zero counters.  Pass 1 changes approx, wimpy and
// last_upd of the nodes on upd_list only, and no mcrade, so only those are
// written (before the scalars, which hold the list's length, are zeroed).
void Job::reset_pass2_counters() {
    reset_updated(jc_, stream_);
    launches += 1;
}

// ---------------------------------------------------------------------------
// Job: the estimator as a state machine (Probabilistic::run,
// silvan/src/Probabilistic.cpp:775-1139)
// ---------------------------------------------------------------------------
int Job::begin(FILE *sink, cudaStream_t stream) {
    if (phase_ != kInit) {
        set_error("a job runs once");
        return SILVAN_E_STATE;
    }
    sink_ = sink;
    stream_ = stream;
    const uint64_t m = g_->m;
    const int D = (int)g_->diameter;
    const double eps = p_.eps, delta = p_.delta;
    absolute_ = p_.k == 0;
    std::ostringstream out;
    out << "estimated diameter of the graph: " << D << "\n";
    out << "time for estimating diameter " << g_->diameter_seconds << "\n";
    uint32_t tau = (uint32_t)fmax(1. / eps * (log(1. / delta)), 1000.);
    tau = (uint32_t)fmax((double)tau, 2 * D * (log(1. / delta)));
    tau_ = tau;
    out << "Starting first pass. Tentative number of samples: " << tau << "\n";
    peel_on_ = p_.a > 1;
    peel_a_ = peel_on_ ? p_.a : 100. * tau;
    const uint32_t threads = p_.threads ? p_.threads : 1;
    union_sample_ = std::min(n_, (uint32_t)fmax(2 * sqrt((double)m) / threads, p_.k + 20.));
    k_ = std::min(p_.k, n_);
    out_ += out.str();
    flush();
    CK(cudaMemsetAsync(jc_.sp_lengths, 0, sizeof(uint64_t) * (D + 1), stream_));
    t_start_ = now_seconds();
    CK(cudaEventRecord(ev_run_[0], stream_));
    phase_ = kPass1;
    alpha_ = p_.alpha;
    base_global_ = 0;
    pass_samples_ = 0;
    // pass 1 stops after the first 11-sample block with n_pairs >= tau
    // (:828-845); top-k mode also needs 1.5 k nodes with approx >= 3
    target_ = (uint64_t)kBlock * ((tau + kBlock - 1) / kBlock);
    p1_chunk_ = target_;
    return SILVAN_OK;
}

bool Job::next_request(JobRequest &r) {
    if (phase_ == kDone || phase_ == kInit || error_) return false;
    uint64_t cnt = target_ - pass_samples_;
    if (p_.form == SILVAN_FORM_PLAIN) {
        cnt = std::min<uint64_t>(cnt, kBlock);
    } else if (phase_ == kPass2 || absolute_) {
        // draw ahead of the next schedule point: samples are deterministic in
        // their index, so drawing early changes nothing but the launch count;
        // the ones beyond the final stop are discarded.  In absolute mode the
        // first pass has a fixed length, and the samples drawn beyond it are
        // the second pass's first ones when the second pass keeps alpha.
        // in the first pass, at most four times its length: a long tail
        // would otherwise ask for a launch whose size favours long tails
        uint64_t ahead = phase_ == kPass2 ? lookahead_
                                          : std::min<uint64_t>(lookahead_tail_, 4 * target_);
        if (phase_ == kPass1 && hint_total_ > target_ && hint_total_ > pass_samples_) {
            // the earlier jobs of this class of graphs suggest drawing
            // hint_total_ samples (Engine::job_hint) with pass 2 on the same
            // stream: draw that far at once, so that one launch usually
            // covers the whole estimation (a second launch costs more than
            // a few extra samples)
            ahead = std::max<uint64_t>(ahead, hint_total_ - pass_samples_);
        }
        if (phase_ == kPass2 && predicted_stop_ > pass_samples_) {
            // absolute mode after a failed check: up to the schedule point at
            // or after the predicted stop (at most 4x the samples so far)
            uint64_t ns = std::max<uint64_t>(next_stop_, 1);
            const uint64_t want = std::min<uint64_t>(predicted_stop_, 5 * pass_samples_);
            while (ns < want && (double)ns < last_stop_)
                ns = std::max<uint64_t>(ns + 1, (uint64_t)(ns * 1.2));
            const uint64_t b = (uint64_t)kBlock * ((ns + kBlock - 1) / kBlock);
            ahead = std::max<uint64_t>(lookahead_tail_, b > pass_samples_ ? b - pass_samples_ : 0);
        }
        cnt = std::max<uint64_t>(cnt, ahead);
        if (phase_ == kPass2 && p_.m_hat) {
            // the omega cap only decreases, so the run never goes beyond it
            const uint64_t cap = (uint64_t)kBlock * (uint64_t)ceil(omega_ / kBlock);
            if (cap > pass_samples_) cnt = std::min<uint64_t>(cnt, cap - pass_samples_);
        }
    }
    cnt = std::min<uint64_t>(cnt, kRoundSamples);
    r.first_global = (uint32_t)(base_global_ + pass_samples_);
    r.count = (uint32_t)cnt;
    r.pass = phase_ == kPass1 ? 1 : 2;
    r.track_cross = phase_ == kPass1 && !absolute_;
    r.alpha = alpha_;
    if (base_global_ + pass_samples_ + cnt >= 0xffffffffull) return false;
    return cnt > 0;
}

namespace {
// The next block end at which pass 2 of the reference acts
// (Probabilistic.cpp:1060-1087): the omega stop or a schedule check.
uint64_t pass2_target(uint64_t done, bool m_hat, double omega, uint64_t next_stop,
                      double last_stop) {
    uint64_t target = UINT64_MAX;
    if (m_hat) target = std::min<uint64_t>(target, kBlock * (uint64_t)ceil(omega / kBlock));
    uint64_t b = (next_stop + kBlock - 1) / kBlock;
    if (b * kBlock <= done) b = done / kBlock + 1;
    const uint64_t t = b * kBlock;
    if ((double)t < last_stop) target = std::min(target, t);
    if (target == UINT64_MAX || target <= done) target = done + kBlock;
    return target;
}
}  // namespace

int Job::finish_pass1() {
    const int D = (int)g_->diameter;
    const double eps = p_.eps, delta = p_.delta;
    const uint64_t P1 = pass_samples_;
    p1_samples_ = P1;
    // empirical peeling (:853-889), with the scalars and path-length counts
    std::vector<uint64_t> sp;
    RK(peel(peel_a_, peel_on_, sp));
    double sup_bcest, sup_wv;
    std::memcpy(&sup_bcest, &sc1_.sup_approx_bits, sizeof(double));
    std::memcpy(&sup_wv, &sc1_.sup_wimpy_bits, sizeof(double));
    std::ostringstream out;
    out << "First pass finished after " << P1 << " iteration" << "\n";
    out << "number_of_non_empty_partitions  " << nparts_ << "\n";
    for (int i = 0; i < nparts_; i++)
        out << "  part. w. index  " << part_ids_[i] << " has " << part_count_[i]
            << " elements, map to " << i << "\n";
    out << "time for first pass " << now_seconds() - t_start_ << "\n";
    out << "void_samples first pass " << sc1_.void_samples << "\n";
    t_first_ = now_seconds() - t_start_;
    // bounds and the alpha switch (:906-942)
    double mns = 0.;
    if (absolute_) {
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
    // first sample size by bisection (:973-1025)
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
    out_ += out.str();
    flush();
    t2_start_ = now_seconds();
    phase_ = kPass2;
    base_global_ = P1;
    pass_samples_ = 0;
    target_ = pass2_target(0, p_.m_hat != 0, omega_, next_stop_, last_stop_);
    return SILVAN_OK;
}

int Job::on_drawn(const JobRequest &r, uint64_t n_records) {
    // the drawn range is [g0, g1) in global sample indices; commit it up to
    // each schedule point in turn and evaluate the point (:828-845,
    // :1060-1087), across the end of pass 1 when the draw reaches into pass 2
    const uint64_t g0 = r.first_global, g1 = g0 + r.count;
    drawn_ += r.count;
    if (g0 != base_global_ + pass_samples_) {
        set_error("drawn range does not continue the committed samples");
        return SILVAN_E_STATE;
    }
    const uint64_t save_apply = launches;
    CK(cudaEventRecord(ev_commit_[0], stream_));
    for (;;) {
        JobRequest rc = r;
        rc.pass = phase_ == kPass1 ? 1 : 2;
        rc.track_cross = phase_ == kPass1 && !absolute_;
        const uint64_t cur = base_global_ + pass_samples_;
        const uint64_t c_hi = std::min(base_global_ + target_, g1);
        if (c_hi > cur) {
            RK(apply_range(rc, (uint32_t)(cur - g0), (uint32_t)(c_hi - g0), n_records));
            pass_samples_ += c_hi - cur;
        }
        if (pass_samples_ < target_) break;  // the next point lies beyond the drawn range
        const Phase ph = phase_;
        ov_.on = true;
        ov_.rc = rc;
        ov_.g0 = g0;
        ov_.g1 = g1;
        ov_.n_records = n_records;
        const int ev = evaluate();
        ov_.on = false;
        RK(ev);
        if (done()) break;
        if (phase_ != ph) {
            // pass 1 ended: the rest of the draw is pass 2's if drawn with its alpha
            if (alpha_ != r.alpha) break;
            continue;
        }
        // pass 1 redrawn from the start (the next round of a check that let
        // the run go on may already be committed: pass_samples_ moved on)
        if (base_global_ + pass_samples_ < c_hi) break;
    }
    CK(cudaEventRecord(ev_commit_[1], stream_));
    CK(cudaEventSynchronize(ev_commit_[1]));
    if (launches != save_apply) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev_commit_[0], ev_commit_[1]);
        commit_ms_ += ms;
        if (done()) result_.time_apply_s = commit_ms_ / 1000.0;  // the run ended in this call
    }
    return SILVAN_OK;
}

// Pass 2 of absolute mode, between the device part of a check and its host
// part: commits the round up to the schedule point that follows the check
// when the check lets the run go on and leaves omega and the last stopping
// size where they are, with a journal (ov_ records the round).  The host
// evaluates the check meanwhile; evaluate() keeps the round if the point
// comes out the same and undoes it otherwise.  The samples must be in the
// drawn range and fit one commit sub-round.
int Job::speculate() {
    ov_.spec_lo = ov_.spec_hi = 0;
    if (!ov_.on || !absolute_ || !jr_.approx || p_.serial_checks || phase_ != kPass2 ||
        ov_.rc.pass != 2 || ov_.rc.alpha != alpha_)
        return SILVAN_OK;
    const uint64_t ns = (uint64_t)(next_stop_ * 1.2);
    const uint64_t t = pass2_target(pass_samples_, p_.m_hat != 0, omega_, ns, last_stop_);
    if (t <= pass_samples_ || t - pass_samples_ > kLargeBucket) return SILVAN_OK;
    const uint64_t cur = base_global_ + pass_samples_, hi = base_global_ + t;
    if (cur < ov_.g0 || hi > ov_.g1) return SILVAN_OK;
    RK(apply_range(ov_.rc, (uint32_t)(cur - ov_.g0), (uint32_t)(hi - ov_.g0), ov_.n_records, true));
    ov_.spec_lo = pass_samples_;
    ov_.spec_hi = t;
    return SILVAN_OK;
}

int Job::undo_speculation() {
    CK(undo_round(rb_, jc_, jr_, 2, g_->diameter, stream_));
    launches += 1;
    ov_.spec_lo = ov_.spec_hi = 0;
    return SILVAN_OK;
}

// The reference's action at the end of the block where pass_samples_ reached
// target_.
int Job::evaluate() {
    if (phase_ == kPass1) {
        if (!absolute_ && !p1_final_) {
            // first block end with n_pairs >= tau and at least 1.5 k nodes
            // whose approx reached 3
            JobScalars sc;
            RK(sync_scalars(sc));
            std::vector<uint32_t> cross(sc.n_cross);
            if (sc.n_cross)
                CK(cudaMemcpy(cross.data(), jc_.cross_sample, sizeof(uint32_t) * sc.n_cross,
                              cudaMemcpyDeviceToHost));
            std::sort(cross.begin(), cross.end());
            uint64_t stop_at = 0;
            const double need = 1.5 * p_.k;
            for (uint64_t b = (tau_ + kBlock - 1) / kBlock; b * kBlock <= target_; b++) {
                const uint64_t c = std::lower_bound(cross.begin(), cross.end(),
                                                    (uint32_t)(b * kBlock)) -
                                   cross.begin();
                if ((double)c >= need) {
                    stop_at = b * kBlock;
                    break;
                }
            }
            if (stop_at == 0) {
                p1_chunk_ *= 2;
                target_ += p1_chunk_;
                return SILVAN_OK;
            }
            p1_final_ = true;
            if (stop_at < target_) {
                // redraw pass 1 up to the stopping block (deterministic)
                const uint32_t n = n_;
                const int D = (int)g_->diameter;
                CK(cudaMemsetAsync(jc_.approx, 0, sizeof(double) * n, stream_));
                CK(cudaMemsetAsync(jc_.wimpy, 0, sizeof(double) * n, stream_));
                CK(cudaMemsetAsync(jc_.last_upd, 0, sizeof(uint32_t) * n, stream_));
                CK(cudaMemsetAsync(jc_.cross_flag, 0, n, stream_));
                CK(cudaMemsetAsync(jc_.sp_lengths, 0, sizeof(uint64_t) * (D + 1), stream_));
                CK(cudaMemsetAsync(jc_.sc, 0, sizeof(JobScalars), stream_));
                pass_samples_ = 0;
                target_ = stop_at;
                return SILVAN_OK;
            }
        }
        return finish_pass1();
    }
    // pass 2 (:1060-1087)
    bool stop = false;
    if (p_.m_hat && (double)pass_samples_ >= omega_) {
        stop = true;
        stop_reason_ = 2;
    } else if ((double)pass_samples_ < last_stop_ && pass_samples_ >= next_stop_) {
        RK(stop_check_enqueue());
        RK(speculate());
        RK(stop_check_finish(stop));
        if (stop) {
            std::ostringstream o;
            o << "MCRADE STOPS after seconds " << now_seconds() - t_start_ << "\n";
            o << "/* stop_mcrade is true */" << "\n";
            out_ += o.str();
            stop_reason_ = 1;
        } else {
            next_stop_ = (uint64_t)(next_stop_ * 1.2);
            iteration_ += 1;
        }
        flush();
    }
    if (!stop) {
        target_ = pass2_target(pass_samples_, p_.m_hat != 0, omega_, next_stop_, last_stop_);
        if (ov_.spec_hi) {
            // the journaled round ends at the point the check left: it stands
            if (target_ == ov_.spec_hi && pass_samples_ == ov_.spec_lo) {
                pass_samples_ = ov_.spec_hi;
                overlapped_checks_++;
                ov_.spec_lo = ov_.spec_hi = 0;
            } else {
                RK(undo_speculation());
            }
        }
        return SILVAN_OK;
    }
    if (ov_.spec_hi) RK(undo_speculation());
    // ---- end of the run (:1103-1138) ---------------------------------------
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
    std::ostringstream out;
    out << "out of second pass " << "\n";
    out << "time for second pass " << t_end - t2_start_ << "\n";
    out << "void_samples second pass " << sc2.void_samples << " ("
        << (double)sc2.void_samples / (double)N2 << ")" << "\n";
    const uint64_t vis_total = sc1_.vis_edges + sc2.vis_edges;
    const double t_bfs = own_engine_ ? own_engine_->sample_ms() / 1000.0 : 0.0;
    const double t_crit = commit_ms_ / 1000.0;
    if (p_.verbose > 0) {
        if (!absolute_) out << "eps_final_topk " << eps_final_topk_ << "\n";
        out << std::setprecision(6) << "\n" << "Finished after " << N2 << " iterations." << "\n";
        out << "Edges visited: " << vis_total << "\n";
        out << "Average edges visited: " << (N2 ? vis_total / N2 : 0) << "\n";
        out << "Total time: " << t_end - t_start_ << "\n";
        out << "Time bfs: " << t_bfs << "\n";
        out << "Time critical: " << t_crit << "\n";
        out << "Time compute finished: " << 0 << "\n";
        out << "Time mcera: " << 0 << "\n";
        out << "(Printing thread: " << 0 << ")" << "\n";
        out << "Avg time bfs: " << t_bfs << "\n";
        out << "Avg time critical: " << t_crit << "\n";
        out << "Avg time critical (round): " << 0 << "\n";
        out << "Avg time compute finished: " << 0 << "\n";
        out << "Avg time mcera: " << 0 << "\n";
        out << "sup bc est: " << sup_b2 / (double)N2 << "\n";
        out << "sup_emp_wimpy_var: " << sup_w2 / (double)N2 << "\n";
        out << "void_samples: " << sc2.void_samples << "\n";
        out << "num_samples: " << N2 << "\n";
    }
    out_ += out.str();
    flush();
    if (!absolute_) RK(ranking(final_rank_el_, final_rank_val_));
    silvan_result_t &res = result_;
    std::memset(&res, 0, sizeof(res));
    res.first_pass_samples = p1_samples_;
    res.num_samples = N2;
    res.vis_edges = vis_total;
    res.void_samples = sc2.void_samples;
    res.backtracked_paths = sc2.paths;
    res.tau = tau_;
    res.diameter = g_->diameter;
    res.iteration_index = iteration_;
    res.num_partitions = nparts_;
    res.stop_reason = stop_reason_;
    res.union_sample = union_sample_;
    res.numresults_topk = numresults_topk_;
    res.checks = checks_;
    res.omega = omega_;
    res.first_stopping_samples = first_stop_;
    res.last_stopping_samples = last_stop_;
    res.alpha_sp_sampling = alpha_;
    res.eps_stop = eps_stop_;
    res.eps_final_topk = eps_final_topk_;
    res.sup_bcest = sup_b2 / (double)N2;
    res.sup_emp_wimpy_var = sup_w2 / (double)N2;
    res.max_num_samples = max_num_samples_;
    res.time_total_s = t_end - t_start_;
    res.time_first_pass_s = t_first_;
    res.time_sampling_s = t_bfs;
    res.time_apply_s = t_crit;
    res.time_device_s = run_ms / 1000.0;
    res.ball_nodes = sc1_.ball_nodes + sc2.ball_nodes;
    res.pred_entries = sc1_.pred_entries + sc2.pred_entries;
    res.kernel_launches = launches + (own_engine_ ? own_engine_->launches() : 0);
    res.sampler_launches = own_engine_ ? own_engine_->sampler_launches() : 0;
    res.sampler_block = own_engine_ ? own_engine_->main_block() : 0;
    res.samples_drawn = drawn_;
    res.assisted_levels = own_engine_ ? own_engine_->assisted_levels() : 0;
    res.helper_tiles = own_engine_ ? own_engine_->helper_tiles() : 0;
    res.overlapped_checks = overlapped_checks_;
    phase_ = kDone;
    return SILVAN_OK;
}

int Job::finish(silvan_result_t *res) {
    if (phase_ != kDone) {
        set_error("job has not finished");
        return SILVAN_E_STATE;
    }
    if (res) *res = result_;
    return SILVAN_OK;
}

int Job::run(silvan_result_t *res, FILE *sink) {
    RK(borrow_engine());
    struct Return {
        Job *j;
        ~Return() { j->return_engine(); }
    } ret{this};
    own_engine_->reset_timers();
    launches = 0;
    RK(begin(sink, own_engine_->stream()));
    std::vector<Job *> jobs{this};
    std::vector<JobRequest> reqs(1);
    std::vector<uint64_t> nrec;
    set_lookahead(own_engine_->free_samples(g_, true), own_engine_->free_samples(g_, false));
    hint_total_ = own_engine_->job_hint(g_);
    while (!done()) {
        if (!next_request(reqs[0])) {
            set_error("sample index space exhausted");
            return SILVAN_E_STATE;
        }
        int rc = own_engine_->round(jobs, reqs, nrec);
        if (rc == SILVAN_OK) rc = on_drawn(reqs[0], nrec[0]);
        if (rc != SILVAN_OK) {
            error_ = rc;
            return rc;
        }
        set_lookahead(own_engine_->free_samples(g_, true), own_engine_->free_samples(g_, false));
    }
    RK(finish(res));
    // the next job of this class of graphs draws about as far in its first
    // launch (when the second pass kept alpha, so those draws are used)
    own_engine_->note_job(g_, result_.first_pass_samples + result_.num_samples,
                          alpha_ == p_.alpha);
    return SILVAN_OK;
}

int Job::step(uint32_t rounds, silvan_status_t *st, FILE *sink) {
    if (phase_ == kDone) {
        if (st) {
            st->samples = result_.num_samples;
            st->void_samples = result_.void_samples;
            st->vis_edges = result_.vis_edges;
            st->backtracked_paths = result_.backtracked_paths;
            st->pass = 2;
            st->done = 1;
        }
        return SILVAN_OK;
    }
    RK(borrow_engine());
    if (phase_ == kInit) {
        own_engine_->reset_timers();
        launches = 0;
        RK(begin(sink, own_engine_->stream()));
        set_lookahead(own_engine_->free_samples(g_, true), own_engine_->free_samples(g_, false));
    }
    std::vector<Job *> jobs{this};
    std::vector<JobRequest> reqs(1);
    std::vector<uint64_t> nrec;
    for (uint32_t i = 0; i < rounds && !done(); i++) {
        if (!next_request(reqs[0])) {
            set_error("sample index space exhausted");
            return SILVAN_E_STATE;
        }
        int rc = own_engine_->round(jobs, reqs, nrec);
        if (rc == SILVAN_OK) rc = on_drawn(reqs[0], nrec[0]);
        if (rc != SILVAN_OK) {
            error_ = rc;
            return rc;
        }
        set_lookahead(own_engine_->free_samples(g_, true), own_engine_->free_samples(g_, false));
    }
    if (st) {
        JobScalars sc{};
        if (!done()) RK(sync_scalars(sc));
        st->samples = done() ? result_.num_samples : pass_samples_;
        st->void_samples = done() ? result_.void_samples : sc.void_samples;
        st->vis_edges = done() ? result_.vis_edges : sc.vis_edges;
        st->backtracked_paths = done() ? result_.backtracked_paths : sc.paths;
        st->pass = phase_ == kPass1 ? 1 : 2;
        st->done = done() ? 1 : 0;
    }
    if (done()) return_engine();
    return SILVAN_OK;
}

int run_batched(const std::vector<Job *> &jobs, uint64_t mem_budget, silvan_result_t *results,
                FILE *sink) {
    if (jobs.empty()) return SILVAN_OK;
    uint64_t n_max = 0;
    for (Job *j : jobs) {
        if (j->started()) {
            set_error("a job runs once");
            return SILVAN_E_STATE;
        }
        n_max = std::max<uint64_t>(n_max, j->nodes());
    }
    uint32_t slots = 0;
    for (Job *j : jobs) slots = std::max(slots, j->params().slots);
    Engine eng;
    RK(eng.init(n_max, slots, mem_budget));
    // the jobs use the engine's stream only while it exists
    struct Detach {
        const std::vector<Job *> &js;
        ~Detach() {
            for (Job *j : js) j->detach();
        }
    } detach{jobs};
    for (Job *j : jobs) RK(j->begin(sink, eng.stream()));
    std::vector<Job *> act;
    std::vector<JobRequest> reqs;
    for (;;) {
        act.clear();
        reqs.clear();
        for (Job *j : jobs) {
            if (j->done()) continue;
            JobRequest r;
            if (!j->next_request(r)) {
                set_error("sample index space exhausted");
                return SILVAN_E_STATE;
            }
            act.push_back(j);
            reqs.push_back(r);
        }
        if (act.empty()) break;
        std::vector<uint64_t> nrec;
        RK(eng.round(act, reqs, nrec));
        for (size_t i = 0; i < act.size(); i++) RK(act[i]->on_drawn(reqs[i], nrec[i]));
        const size_t na = std::max<size_t>(1, act.size());
        for (Job *j : act)
            j->set_lookahead(eng.free_samples(j->graph(), true) / na,
                             eng.free_samples(j->graph(), false) / na);
    }
    for (size_t i = 0; i < jobs.size(); i++) RK(jobs[i]->finish(&results[i]));
    return SILVAN_OK;
}

// ---------------------------------------------------------------------------
// Job: reads and the replay hook
// ---------------------------------------------------------------------------
int Job::read_estimates(double *out, uint32_t n) {
    if (n != n_) {
        set_error("estimate buffer size does not match the graph");
        return SILVAN_E_BADARG;
    }
    // approx / num_samples on the device (the same IEEE division), then one copy
    double *est = nullptr;
    RK(dmalloc(&est, n));
    CK(divide_estimates(jc_.approx, (double)pass_samples_, est, n, stream_));
    cudaError_t e = cudaMemcpyAsync(out, est, sizeof(double) * n, cudaMemcpyDeviceToHost, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    dfree(est);
    CK(e);
    return SILVAN_OK;
}

int Job::read_counters(double *approx, double *wimpy, int64_t *mcrade, int32_t *part) {
    const uint32_t n = n_;
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
    if (phase_ != kDone || absolute_) {
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
    RK(borrow_engine());
    struct Return {
        Job *j;
        ~Return() { j->return_engine(); }
    } ret{this};
    stream_ = own_engine_->stream();
    pl.assign(count, 0);
    np.assign(count, 0);
    vis.assign(count, 0);
    status.assign(count, 0);
    recs.clear();
    const double save_alpha = alpha_;
    alpha_ = alpha;
    std::vector<Job *> jobs{this};
    std::vector<JobRequest> reqs(1);
    std::vector<uint64_t> nrec;
    for (uint32_t done = 0; done < count;) {
        const uint32_t c = std::min<uint32_t>(count - done, kRoundSamples);
        reqs[0].first_global = first + done;
        reqs[0].count = c;
        reqs[0].pass = 1;
        reqs[0].alpha = alpha;
        RK(own_engine_->round(jobs, reqs, nrec));
        CK(cudaMemcpy(pl.data() + done, rb_.pl, sizeof(int32_t) * c, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(np.data() + done, rb_.np, sizeof(int32_t) * c, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(vis.data() + done, rb_.vis, sizeof(uint64_t) * c, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(status.data() + done, rb_.status, sizeof(int32_t) * c,
                      cudaMemcpyDeviceToHost));
        const size_t r0 = recs.size();
        recs.resize(r0 + nrec[0]);
        if (nrec[0])
            CK(cudaMemcpy(recs.data() + r0, rb_.recs, sizeof(PathRec) * nrec[0],
                          cudaMemcpyDeviceToHost));
        for (size_t i = r0; i < recs.size(); i++) recs[i].sample += done;
        done += c;
    }
    alpha_ = save_alpha;
    return SILVAN_OK;
}

}  // namespace silvan
