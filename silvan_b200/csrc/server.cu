// Estimation server: continuous batching of progressive-sampling jobs.
//
// Requests (a host graph plus the binary's flags) are queued by any thread.
// An uploader thread admits queued requests in arrival order while their
// device memory (CSR + counters + round buffers) fits the budget and puts
// each admitted job's graph and state on the device; the server thread keeps
// them there and runs rounds: each round is one persistent sampler launch
// serving the next schedule interval of every active job, followed by each
// job's ordered commit and schedule evaluation (engine.cu).  Uploads overlap
// the rounds of the requests already running.  A job that reaches its
// stopping decision releases its memory, its estimates are copied to the host
// and the next queued request can be admitted -- requests arriving while
// others run join at the next round.  Each job follows exactly its stand-alone
// schedule, so its result does not depend on the mix.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "engine.h"
#include "server.h"

namespace silvan {

// Predicted CTA time of one serving round over all slots: long enough to
// amortise a launch, short enough that a small request never waits long
// behind a large one.
constexpr double kServeRoundMs = 3.0;

struct ServerRequest {
    uint64_t id = 0;
    HostGraph host;
    std::vector<uint32_t> cc;
    uint32_t ncomp = 0, diameter = 0;
    silvan_params_t params{};
    int32_t state = SILVAN_REQ_QUEUED;
    double t_submit = 0, t_admit = 0, t_done = 0;
    uint64_t bytes = 0;
    std::unique_ptr<DeviceGraph> graph;
    std::unique_ptr<Job> job;
    silvan_result_t result{};
    std::vector<double> estimates;
    std::vector<uint32_t> topk_nodes;
    std::vector<double> topk_values;
    std::string error;  // message of a failed request (set on the thread that failed it)
};

struct Server {
    uint64_t n_max = 0, budget = 0, used = 0;
    uint32_t slots = 0;
    Engine eng;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<ServerRequest *> pending;
    std::deque<ServerRequest *> ready;      // uploaded, waiting for the server thread
    std::vector<ServerRequest *> active;
    uint64_t in_upload = 0;                 // admitted, not yet ready
    std::map<uint64_t, std::unique_ptr<ServerRequest>> all;
    uint64_t next_id = 1;
    std::atomic<bool> stop{false};
    std::thread th, up_th;
    int device = 0;
    int fatal = 0;
    uint64_t rounds = 0, max_active = 0, samples = 0;
    int init_rc = SILVAN_OK;
    std::mutex init_mu;
    std::condition_variable init_cv;
    bool init_done = false;

    // time accounting of the server thread (seconds): total, longest
    double t_acc[4] = {0, 0, 0, 0}, t_max[4] = {0, 0, 0, 0};
    void account(int what, double t0) {
        const double dt = now_seconds() - t0;
        std::lock_guard<std::mutex> lk(mu);
        t_acc[what] += dt;
        t_max[what] = std::max(t_max[what], dt);
    }

    static uint64_t job_bytes(uint64_t n, uint64_t D) {
        // counters + node buckets + round buffers at their initial capacity
        return n * (8 + 8 + 8ull * kTrials + 4 + 1 + 4 + 4 + 4 + 4 + 8) + (D + 1) * 8 +
               65536ull * 36 + (1ull << 20) * 20 + (64ull << 20);
    }

    void loop(int device) {
        cudaSetDevice(device);
        {
            std::lock_guard<std::mutex> lk(init_mu);
            init_rc = eng.init(n_max, slots, 0);
            init_done = true;
        }
        init_cv.notify_all();
        if (init_rc != SILVAN_OK) return;
        std::vector<Job *> jobs;
        std::vector<JobRequest> reqs;
        while (!stop.load()) {
            // requests whose graph and state the uploader has put on the device
            std::vector<ServerRequest *> start;
            {
                std::unique_lock<std::mutex> lk(mu);
                if (active.empty() && ready.empty())
                    cv.wait_for(lk, std::chrono::milliseconds(20));
                while (!ready.empty()) {
                    start.push_back(ready.front());
                    ready.pop_front();
                }
            }
            for (ServerRequest *r : start) {
                int rc = r->job->begin(nullptr, eng.stream());
                if (rc != SILVAN_OK) {
                    finish(r, rc);
                    continue;
                }
                std::lock_guard<std::mutex> lk(mu);
                active.push_back(r);
            }
            if (active.empty()) continue;
            max_active = std::max<uint64_t>(max_active, active.size());
            jobs.clear();
            reqs.clear();
            std::vector<ServerRequest *> owners;
            for (ServerRequest *r : active) {
                JobRequest q;
                if (!r->job->next_request(q)) {
                    finish(r, SILVAN_E_STATE);
                    continue;
                }
                jobs.push_back(r->job.get());
                reqs.push_back(q);
                owners.push_back(r);
            }
            if (jobs.empty()) continue;
            // short rounds: a small request does not wait behind a large one
            eng.fair_share(jobs, reqs, kServeRoundMs);
            std::vector<uint64_t> nrec;
            const double t_round = now_seconds();
            int rc = eng.round(jobs, reqs, nrec);
            account(1, t_round);
            rounds++;
            for (const JobRequest &q : reqs) samples += q.count;
            if (rc != SILVAN_OK) {
                // a device error poisons every job in the round
                for (ServerRequest *r : owners) finish(r, rc);
                continue;
            }
            const size_t na = std::max<size_t>(1, owners.size());

            for (size_t i = 0; i < owners.size(); i++) {
                ServerRequest *r = owners[i];
                const double t_commit = now_seconds();
                int e = r->job->on_drawn(reqs[i], nrec[i]);
                r->job->set_lookahead(eng.free_samples(r->graph.get(), true) / na,
                                      eng.free_samples(r->graph.get(), false) / na);
                account(2, t_commit);
                if (e != SILVAN_OK) finish(r, e);
                else if (r->job->done()) finish(r, SILVAN_OK);
            }
        }
    }

    // Admission by device-memory budget, in arrival order, and the upload of
    // each admitted request's graph and job state, on a thread of its own so
    // that the rounds of the active requests go on meanwhile (the copies run
    // on the legacy stream, the rounds on the engine's non-blocking stream).
    void uploader() {
        cudaSetDevice(device);
        while (!stop.load()) {
            ServerRequest *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait_for(lk, std::chrono::milliseconds(20), [this]() {
                    return stop.load() || (!pending.empty() &&
                                           (used + pending.front()->bytes <= budget ||
                                            (active.empty() && ready.empty() && !in_upload)));
                });
                if (stop.load() || pending.empty()) continue;
                r = pending.front();
                if (used + r->bytes > budget && !(active.empty() && ready.empty() && !in_upload))
                    continue;
                pending.pop_front();
                used += r->bytes;
                in_upload++;
                r->state = SILVAN_REQ_RUNNING;
                r->t_admit = now_seconds();
            }
            const double t_adm = now_seconds();
            r->graph.reset(new DeviceGraph());
            r->graph->host = std::move(r->host);
            r->graph->cc = std::move(r->cc);
            r->graph->ncomp = r->ncomp;
            r->graph->diameter = r->diameter;
            int rc = r->graph->upload();
            if (rc == SILVAN_OK) {
                r->job.reset(new Job(r->graph.get(), r->params));
                rc = r->job->init();
            }
            // the upload and the set-up ran on the legacy stream: done before the
            // request's first round on the engine's stream
            if (rc == SILVAN_OK)
                rc = cuda_status(cudaStreamSynchronize(cudaStreamLegacy), "request upload");
            account(0, t_adm);
            if (rc != SILVAN_OK) {
                finish(r, rc);
                std::lock_guard<std::mutex> lk(mu);
                in_upload--;
                continue;
            }
            std::lock_guard<std::mutex> lk(mu);
            in_upload--;
            ready.push_back(r);
            cv.notify_all();
        }
    }

    // Completes a request: keeps its outputs on the host, frees its device state.
    void finish(ServerRequest *r, int rc) {
        if (rc != SILVAN_OK) r->error = last_error_cstr();
        const double t_fin = now_seconds();
        struct Acc {
            Server *s;
            double t;
            ~Acc() { s->account(3, t); }
        } acc{this, t_fin};
        if (rc == SILVAN_OK && r->job) {
            r->job->finish(&r->result);
            r->estimates.resize(r->graph->n);
            r->job->read_estimates(r->estimates.data(), r->graph->n);
            if (r->params.k > 0) {
                uint32_t cap = r->result.numresults_topk + 1, cnt = 0;
                r->topk_nodes.resize(cap);
                r->topk_values.resize(cap);
                r->job->read_topk(r->topk_nodes.data(), r->topk_values.data(), cap, &cnt);
                r->topk_nodes.resize(cnt);
                r->topk_values.resize(cnt);
            }
        }
        if (r->job) r->job->detach();
        r->job.reset();
        r->graph.reset();
        std::lock_guard<std::mutex> lk(mu);
        for (size_t i = 0; i < active.size(); i++)
            if (active[i] == r) {
                active.erase(active.begin() + i);
                break;
            }
        used -= r->bytes;
        r->t_done = now_seconds();
        r->state = rc == SILVAN_OK ? SILVAN_REQ_DONE : rc;
        cv.notify_all();
    }
};

int server_create(uint64_t n_max, uint64_t budget, uint32_t slots, Server **out) {
    int dev = 0;
    cudaGetDevice(&dev);
    Server *s = new Server();
    s->n_max = n_max;
    s->slots = slots;
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        budget = fr / 3;
    }
    s->budget = budget;
    s->device = dev;
    s->th = std::thread([s, dev]() { s->loop(dev); });
    std::unique_lock<std::mutex> lk(s->init_mu);
    s->init_cv.wait(lk, [s]() { return s->init_done; });
    if (s->init_rc != SILVAN_OK) {
        int rc = s->init_rc;
        lk.unlock();
        s->stop = true;
        s->th.join();
        delete s;
        return rc;
    }
    s->up_th = std::thread([s]() { s->uploader(); });
    *out = s;
    return SILVAN_OK;
}

int server_submit(Server *s, const HostGraph &h, const std::vector<uint32_t> &cc, uint32_t ncomp,
                  uint32_t diameter, const silvan_params_t &p, uint64_t *id) {
    if (h.n > s->n_max) {
        set_error("graph larger than the server's slots");
        return SILVAN_E_BADARG;
    }
    if (!(p.eps > 0 && p.eps < 1) || !(p.delta > 0 && p.delta < 1)) {
        set_error("eps and delta must lie in (0, 1)");
        return SILVAN_E_BADARG;
    }
    std::unique_ptr<ServerRequest> r(new ServerRequest());
    r->host = h;
    r->cc = cc;
    r->ncomp = ncomp;
    r->diameter = diameter;
    r->params = p;
    r->t_submit = now_seconds();
    HostGraph &hh = r->host;
    r->bytes = 4ull * (hh.n + 1) * (hh.directed ? 2 : 1) + 4ull * hh.out_adj.size() +
               4ull * hh.in_adj.size() + 4ull * hh.n + Server::job_bytes(hh.n, diameter);
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    *id = r->id;
    s->pending.push_back(r.get());
    s->all[r->id] = std::move(r);
    s->cv.notify_all();
    return SILVAN_OK;
}

int server_poll(Server *s, uint64_t id, int32_t *state, silvan_result_t *res, double *latency,
                double *queue_s) {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) {
        set_error("unknown request id");
        return SILVAN_E_BADARG;
    }
    ServerRequest *r = it->second.get();
    if (state) *state = r->state;
    if (r->state == SILVAN_REQ_DONE) {
        if (res) *res = r->result;
        if (latency) *latency = r->t_done - r->t_submit;
        if (queue_s) *queue_s = r->t_admit - r->t_submit;
    }
    if (r->state < 0) set_error(r->error);
    return SILVAN_OK;
}

int server_wait(Server *s, uint64_t id, double timeout_s) {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end()) {
        set_error("unknown request id");
        return SILVAN_E_BADARG;
    }
    ServerRequest *r = it->second.get();
    bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [r]() {
        return r->state != SILVAN_REQ_QUEUED && r->state != SILVAN_REQ_RUNNING;
    });
    if (!ok) {
        set_error("request still running");
        return SILVAN_E_TIMEOUT;
    }
    if (r->state == SILVAN_REQ_DONE) return SILVAN_OK;
    set_error(r->error);
    return r->state;
}

int server_estimates(Server *s, uint64_t id, double *out, uint32_t n, uint32_t *topk_nodes,
                     double *topk_values, uint32_t topk_cap, uint32_t *topk_count) {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->all.find(id);
    if (it == s->all.end() || it->second->state != SILVAN_REQ_DONE) {
        set_error("request not finished");
        return SILVAN_E_STATE;
    }
    ServerRequest *r = it->second.get();
    if (out) {
        if (n != r->estimates.size()) {
            set_error("estimate buffer size does not match the graph");
            return SILVAN_E_BADARG;
        }
        std::copy(r->estimates.begin(), r->estimates.end(), out);
    }
    if (topk_count) *topk_count = (uint32_t)r->topk_nodes.size();
    for (uint32_t i = 0; i < topk_cap && i < r->topk_nodes.size(); i++) {
        if (topk_nodes) topk_nodes[i] = r->topk_nodes[i];
        if (topk_values) topk_values[i] = r->topk_values[i];
    }
    return SILVAN_OK;
}

int server_stats(Server *s, silvan_server_stats_t *st) {
    std::lock_guard<std::mutex> lk(s->mu);
    st->rounds = s->rounds;
    st->samples = s->samples;
    st->max_active = s->max_active;
    st->queued = s->pending.size();
    st->active = s->active.size();
    st->bytes_in_use = s->used;
    st->budget = s->budget;
    st->slots = s->eng.slots();
    st->admit_s = s->t_acc[0];
    st->round_s = s->t_acc[1];
    st->commit_s = s->t_acc[2];
    st->finish_s = s->t_acc[3];
    st->admit_max_s = s->t_max[0];
    st->round_max_s = s->t_max[1];
    st->commit_max_s = s->t_max[2];
    st->finish_max_s = s->t_max[3];
    return SILVAN_OK;
}

void server_destroy(Server *s) {
    s->stop = true;
    s->cv.notify_all();
    if (s->up_th.joinable()) s->up_th.join();
    if (s->th.joinable()) s->th.join();
    for (auto &kv : s->all) {
        kv.second->job.reset();
        kv.second->graph.reset();
    }
    delete s;
}

}  // namespace silvan
