// extern "C" entry points of include/silvan.h.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "engine.h"
#include "ingest.h"
#include "brandes.h"
#include "gen.h"
#include "server.h"
#include "silvan.h"

namespace silvan {
const char *last_error_cstr();
int replay_samples_noalloc(const DeviceGraph &G, uint64_t seed, uint32_t first, uint32_t count,
                           double alpha, uint32_t np_cap, int32_t *d_path_length,
                           int32_t *d_num_paths, uint64_t *d_vis_edges, int32_t *d_status,
                           uint32_t *d_records, uint64_t record_cap,
                           unsigned long long *d_record_count, cudaStream_t stream);
}

struct silvan_graph_s {
    silvan::DeviceGraph g;
};
struct silvan_host_graph_s {
    silvan::HostGraph host;
    std::vector<uint32_t> cc;
    uint32_t ncomp = 0, diameter = 0;
    double seconds = 0;
};
struct silvan_server_s {
    silvan::Server *s;
};
struct silvan_job_s {
    silvan::Job *job;
    silvan_graph_s *graph;
};

using namespace silvan;

namespace {

int check_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_error("no CUDA device available: the sampler runs on the GPU only");
        return SILVAN_E_NOGPU;
    }
    return SILVAN_OK;
}

int finish_graph(silvan_graph_s *G, bool have_cc, silvan_graph_t *out) {
    double t0 = now_seconds();
    if (!have_cc) {
        G->g.ncomp = compute_scc(G->g.host, G->g.cc);
        G->g.diameter = estimate_diameter(G->g.host, G->g.cc, G->g.ncomp);
    }
    G->g.diameter_seconds = now_seconds() - t0;
    int rc = G->g.upload();
    if (rc != SILVAN_OK) {
        delete G;
        return rc;
    }
    *out = G;
    return SILVAN_OK;
}

}  // namespace

extern "C" {

void silvan_params_default(silvan_params_t *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->eps = 0.01;
    p->delta = 0.05;
    p->k = 0;
    p->m_hat = 1;
    p->alpha = 2.3;
    p->alpha_given = 0;
    p->form = SILVAN_FORM_BATCHED;
    p->a = 2.0;
    p->seed = 42;
    p->verbose = 60;
    p->np_cap = 0;
    p->slots = 0;
    p->threads = 1;
    p->block = 0;
    p->backtrack = SILVAN_BACKTRACK_REFERENCE;
    p->assist_items = 0;
    p->wait_polls = 0;
    p->serial_checks = 0;
}

const char *silvan_last_error(void) { return last_error_cstr(); }
const char *silvan_version(void) { return "silvan-b200 0.1"; }

int silvan_graph_load(const char *path, int directed, silvan_graph_t *out) {
    if (!path || !out) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    int rc = check_device();
    if (rc) return rc;
    silvan_graph_s *G = new (std::nothrow) silvan_graph_s();
    if (!G) return SILVAN_E_OOM;
    // parsed and built on the device (ingest.cu); the host loader
    // (silvan_host_graph_load) gives the same graph
    std::string err;
    rc = device_ingest(path, directed != 0, G->g, err);
    if (rc != SILVAN_OK) {
        if (!err.empty()) set_error(err);
        delete G;
        return rc;
    }
    *out = G;
    return SILVAN_OK;
}

int silvan_graph_upload(uint32_t n, int directed, const uint64_t *out_off,
                        const uint32_t *out_adj, const uint64_t *in_off, const uint32_t *in_adj,
                        const uint32_t *cc, uint32_t n_components, uint32_t diameter,
                        silvan_graph_t *out) {
    if (!out_off || !out_adj || !out || (directed && (!in_off || !in_adj))) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    int rc = check_device();
    if (rc) return rc;
    silvan_graph_s *G = new (std::nothrow) silvan_graph_s();
    if (!G) return SILVAN_E_OOM;
    if (cc) {
        // the caller's arrays go to the device as they are (validated there)
        G->g.ncomp = n_components;
        G->g.diameter = diameter;
        G->g.diameter_seconds = 0;
        rc = G->g.upload_raw(n, directed != 0, out_off, out_adj, in_off, in_adj, cc);
        if (rc != SILVAN_OK) {
            delete G;
            return rc;
        }
        *out = G;
        return SILVAN_OK;
    }
    // components and the diameter bound are computed on the host
    HostGraph &h = G->g.host;
    h.n = n;
    h.directed = directed != 0;
    h.out_off.assign(out_off, out_off + n + 1);
    h.out_adj.assign(out_adj, out_adj + out_off[n]);
    if (h.directed) {
        h.in_off.assign(in_off, in_off + n + 1);
        h.in_adj.assign(in_adj, in_adj + in_off[n]);
    }
    for (uint32_t i = 0; i < n; i++) {
        for (uint64_t e = h.out_off[i]; e < h.out_off[i + 1]; e++)
            if (h.out_adj[e] >= n || (e > h.out_off[i] && h.out_adj[e] <= h.out_adj[e - 1])) {
                set_error("CSR rows must hold ascending unique ids < n");
                delete G;
                return SILVAN_E_BADARG;
            }
    }
    return finish_graph(G, false, out);
}

int silvan_graph_from_pairs(const uint32_t *pairs, uint64_t count, int directed,
                            silvan_graph_t *out) {
    if ((!pairs && count) || !out) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    int rc = check_device();
    if (rc) return rc;
    std::vector<std::pair<uint32_t, uint32_t>> pv(count);
    for (uint64_t i = 0; i < count; i++) {
        if (pairs[2 * i] > kMaxNodeId || pairs[2 * i + 1] > kMaxNodeId) {
            set_error("node id too large");
            return SILVAN_E_PARSE;
        }
        pv[i] = {pairs[2 * i], pairs[2 * i + 1]};
    }
    silvan_graph_s *G = new (std::nothrow) silvan_graph_s();
    if (!G) return SILVAN_E_OOM;
    build_csr(pv, directed != 0, G->g.host);
    return finish_graph(G, false, out);
}

namespace {
int host_finish(silvan_host_graph_s *H, silvan_host_graph_t *out) {
    double t0 = now_seconds();
    H->ncomp = compute_scc(H->host, H->cc);
    H->diameter = estimate_diameter(H->host, H->cc, H->ncomp);
    H->seconds = now_seconds() - t0;
    *out = H;
    return SILVAN_OK;
}
}  // namespace

int silvan_host_graph_load(const char *path, int directed, silvan_host_graph_t *out) {
    if (!path || !out) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    silvan_host_graph_s *H = new (std::nothrow) silvan_host_graph_s();
    if (!H) return SILVAN_E_OOM;
    std::string err;
    int rc = load_edge_list(path, directed != 0, H->host, err);
    if (rc != SILVAN_OK) {
        set_error(err);
        delete H;
        return rc;
    }
    return host_finish(H, out);
}

int silvan_host_graph_from_pairs(const uint32_t *pairs, uint64_t count, int directed,
                                 silvan_host_graph_t *out) {
    if ((!pairs && count) || !out) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    std::vector<std::pair<uint32_t, uint32_t>> pv(count);
    for (uint64_t i = 0; i < count; i++) {
        if (pairs[2 * i] > kMaxNodeId || pairs[2 * i + 1] > kMaxNodeId) {
            set_error("node id too large");
            return SILVAN_E_PARSE;
        }
        pv[i] = {pairs[2 * i], pairs[2 * i + 1]};
    }
    silvan_host_graph_s *H = new (std::nothrow) silvan_host_graph_s();
    if (!H) return SILVAN_E_OOM;
    build_csr(pv, directed != 0, H->host);
    return host_finish(H, out);
}

int silvan_host_graph_info(silvan_host_graph_t g, silvan_graph_info_t *info) {
    if (!g || !info) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    info->n = g->host.n;
    info->n_components = g->ncomp;
    info->m = g->host.num_edges();
    info->diameter = g->diameter;
    info->directed = g->host.directed ? 1 : 0;
    return SILVAN_OK;
}

int silvan_host_graph_csr(silvan_host_graph_t g, uint64_t *out_off, uint32_t *out_adj,
                          uint64_t *in_off, uint32_t *in_adj, uint32_t *cc) {
    if (!g) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    const HostGraph &h = g->host;
    if (out_off) std::copy(h.out_off.begin(), h.out_off.end(), out_off);
    if (out_adj) std::copy(h.out_adj.begin(), h.out_adj.end(), out_adj);
    const uint64_t *io = h.in_offsets();
    if (in_off) std::copy(io, io + h.n + 1, in_off);
    if (in_adj) {
        const uint32_t *ia = h.in_neighbours();
        std::copy(ia, ia + io[h.n], in_adj);
    }
    if (cc) std::copy(g->cc.begin(), g->cc.end(), cc);
    return SILVAN_OK;
}

int silvan_host_graph_destroy(silvan_host_graph_t g) {
    delete g;
    return SILVAN_OK;
}

int silvan_graph_from_host(silvan_host_graph_t h, silvan_graph_t *out) {
    if (!h || !out) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    int rc = check_device();
    if (rc) return rc;
    silvan_graph_s *G = new (std::nothrow) silvan_graph_s();
    if (!G) return SILVAN_E_OOM;
    G->g.host = h->host;
    G->g.cc = h->cc;
    G->g.ncomp = h->ncomp;
    G->g.diameter = h->diameter;
    rc = G->g.upload();
    G->g.diameter_seconds = h->seconds;
    if (rc != SILVAN_OK) {
        delete G;
        return rc;
    }
    *out = G;
    return SILVAN_OK;
}

int silvan_graph_info(silvan_graph_t g, silvan_graph_info_t *info) {
    if (!g || !info) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    info->n = g->g.n;
    info->n_components = g->g.ncomp;
    info->m = g->g.m;
    info->diameter = g->g.diameter;
    info->directed = g->g.directed ? 1 : 0;
    return SILVAN_OK;
}

int silvan_graph_csr(silvan_graph_t g, uint64_t *out_off, uint32_t *out_adj, uint64_t *in_off,
                     uint32_t *in_adj, uint32_t *cc) {
    if (!g) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    const DeviceGraph &G = g->g;
    const uint32_t n = G.n;
    if (G.has_host) {
        const HostGraph &h = G.host;
        if (out_off) std::copy(h.out_off.begin(), h.out_off.end(), out_off);
        if (out_adj) std::copy(h.out_adj.begin(), h.out_adj.end(), out_adj);
        const uint64_t *io = h.in_offsets();
        if (in_off) std::copy(io, io + h.n + 1, in_off);
        if (in_adj) {
            const uint32_t *ia = h.in_neighbours();
            std::copy(ia, ia + io[h.n], in_adj);
        }
        if (cc) std::copy(G.cc.begin(), G.cc.end(), cc);
        return SILVAN_OK;
    }
    // uploaded from caller arrays: read the device copy back
    std::vector<uint32_t> off32(n + 1);
    auto get = [&](const uint32_t *doff, const uint32_t *dadj, uint64_t cnt, uint64_t *off,
                   uint32_t *adj) -> int {
        if (off) {
            if (cudaMemcpy(off32.data(), doff, sizeof(uint32_t) * (n + 1),
                           cudaMemcpyDeviceToHost) != cudaSuccess)
                return SILVAN_E_CUDA;
            for (uint32_t i = 0; i <= n; i++) off[i] = off32[i];
        }
        if (adj && cnt &&
            cudaMemcpy(adj, dadj, sizeof(uint32_t) * cnt, cudaMemcpyDeviceToHost) != cudaSuccess)
            return SILVAN_E_CUDA;
        return SILVAN_OK;
    };
    int rc = get(G.d_out_off, G.d_out_adj, G.m, out_off, out_adj);
    if (rc == SILVAN_OK) rc = get(G.d_in_off, G.d_in_adj, G.m_in, in_off, in_adj);
    if (rc == SILVAN_OK && cc &&
        cudaMemcpy(cc, G.d_cc, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = SILVAN_E_CUDA;
    if (rc != SILVAN_OK) set_error("device read failed");
    return rc;
}

int silvan_graph_destroy(silvan_graph_t g) {
    delete g;
    return SILVAN_OK;
}

int silvan_job_create(silvan_graph_t g, const silvan_params_t *p, silvan_job_t *out) {
    if (!g || !p || !out) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    silvan_job_s *J = new (std::nothrow) silvan_job_s();
    if (!J) return SILVAN_E_OOM;
    J->graph = g;
    J->job = new (std::nothrow) Job(&g->g, *p);
    if (!J->job) {
        delete J;
        return SILVAN_E_OOM;
    }
    int rc = J->job->init();
    if (rc != SILVAN_OK) {
        delete J->job;
        delete J;
        return rc;
    }
    *out = J;
    return SILVAN_OK;
}

int silvan_job_run(silvan_job_t j, silvan_result_t *res, void *log) {
    if (!j) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return j->job->run(res, (FILE *)log);
}

int silvan_run_rounds(silvan_job_t j, uint32_t rounds, silvan_status_t *st, void *log) {
    if (!j) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return j->job->step(rounds, st, (FILE *)log);
}

int silvan_job_result(silvan_job_t j, silvan_result_t *res) {
    if (!j || !res) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return j->job->finish(res);
}

int silvan_jobs_run_batched(silvan_job_t *jobs, uint32_t count, uint64_t mem_budget,
                            silvan_result_t *results, void *log) {
    if ((!jobs && count) || (!results && count)) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    std::vector<Job *> js(count);
    for (uint32_t i = 0; i < count; i++) {
        if (!jobs[i]) {
            set_error("null job");
            return SILVAN_E_BADARG;
        }
        js[i] = jobs[i]->job;
    }
    return run_batched(js, mem_budget, results, (FILE *)log);
}

int silvan_read_estimates(silvan_job_t j, double *out, uint32_t n) {
    if (!j || !out) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return j->job->read_estimates(out, n);
}

int silvan_read_topk(silvan_job_t j, uint32_t *nodes, double *values, uint32_t cap,
                     uint32_t *count) {
    if (!j) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return j->job->read_topk(nodes, values, cap, count);
}

int silvan_read_counters(silvan_job_t j, double *approx, double *wimpy, int64_t *mcrade,
                         int32_t *partition_index) {
    if (!j) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return j->job->read_counters(approx, wimpy, mcrade, partition_index);
}

int silvan_job_destroy(silvan_job_t j) {
    if (!j) return SILVAN_OK;
    delete j->job;
    delete j;
    return SILVAN_OK;
}

int silvan_server_create(uint64_t n_max, uint64_t budget, uint32_t slots, silvan_server_t *out) {
    if (!out || n_max < 2) {
        set_error("bad argument");
        return SILVAN_E_BADARG;
    }
    int rc = check_device();
    if (rc) return rc;
    Server *s = nullptr;
    rc = server_create(n_max, budget, slots, &s);
    if (rc != SILVAN_OK) return rc;
    *out = new silvan_server_s{s};
    return SILVAN_OK;
}

int silvan_server_submit(silvan_server_t s, silvan_host_graph_t g, const silvan_params_t *p,
                         uint64_t *id) {
    if (!s || !g || !p || !id) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return server_submit(s->s, g->host, g->cc, g->ncomp, g->diameter, *p, id);
}

int silvan_server_poll(silvan_server_t s, uint64_t id, int32_t *state, silvan_result_t *res,
                       double *latency_s, double *queued_s) {
    if (!s) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return server_poll(s->s, id, state, res, latency_s, queued_s);
}

int silvan_server_wait(silvan_server_t s, uint64_t id, double timeout_s) {
    if (!s) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return server_wait(s->s, id, timeout_s);
}

int silvan_server_estimates(silvan_server_t s, uint64_t id, double *out, uint32_t n,
                            uint32_t *topk_nodes, double *topk_values, uint32_t topk_cap,
                            uint32_t *topk_count) {
    if (!s) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return server_estimates(s->s, id, out, n, topk_nodes, topk_values, topk_cap, topk_count);
}

int silvan_server_stats(silvan_server_t s, silvan_server_stats_t *st) {
    if (!s || !st) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    return server_stats(s->s, st);
}

int silvan_server_destroy(silvan_server_t s) {
    if (!s) return SILVAN_OK;
    server_destroy(s->s);
    delete s;
    return SILVAN_OK;
}

int silvan_replay_samples(silvan_graph_t g, uint64_t seed, uint32_t first, uint32_t count,
                          double alpha, uint32_t np_cap, int32_t *path_length, int32_t *num_paths,
                          uint64_t *vis_edges, uint32_t *nent, int32_t *sample_status,
                          uint32_t *ent_node, int32_t *ent_cnt, uint64_t ent_cap,
                          uint64_t *ent_total) {
    if (!g || !path_length || !num_paths || !vis_edges || !nent || !sample_status) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    silvan_params_t p;
    silvan_params_default(&p);
    p.seed = seed;
    p.np_cap = np_cap;
    Job job(&g->g, p);
    int rc = job.init();
    if (rc != SILVAN_OK) return rc;
    std::vector<int32_t> pl, np, status;
    std::vector<uint64_t> vis;
    std::vector<PathRec> recs;
    rc = job.replay(first, count, alpha, pl, np, vis, status, recs);
    if (rc != SILVAN_OK) return rc;
    std::sort(recs.begin(), recs.end(), [](const PathRec &a, const PathRec &b) {
        return a.sample != b.sample ? a.sample < b.sample : a.node < b.node;
    });
    if (ent_total) *ent_total = recs.size();
    for (uint32_t i = 0; i < count; i++) {
        path_length[i] = pl[i];
        num_paths[i] = np[i];
        vis_edges[i] = vis[i];
        sample_status[i] = status[i];
        nent[i] = 0;
    }
    for (const PathRec &r : recs) nent[r.sample]++;
    if (recs.size() > ent_cap) {
        set_error("entry buffer too small");
        return SILVAN_E_CAPACITY;
    }
    for (size_t i = 0; i < recs.size(); i++) {
        if (ent_node) ent_node[i] = recs[i].node;
        if (ent_cnt) ent_cnt[i] = (int32_t)recs[i].count;
    }
    return SILVAN_OK;
}

int silvan_exact_betweenness(silvan_graph_t g, double *out, uint32_t n) {
    if (!g || !out) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    if (n != g->g.n) {
        set_error("output size does not match the graph");
        return SILVAN_E_BADARG;
    }
    return exact_betweenness(g->g, out);
}

int silvan_replay_samples_noalloc(silvan_graph_t g, uint64_t seed, uint32_t first,
                                  uint32_t count, double alpha, uint32_t np_cap,
                                  int32_t *d_path_length, int32_t *d_num_paths,
                                  uint64_t *d_vis_edges, int32_t *d_status,
                                  uint32_t *d_records, uint64_t record_cap,
                                  unsigned long long *d_record_count, void *stream) {
    if (!g) {
        set_error("null graph");
        return SILVAN_E_BADARG;
    }
    return replay_samples_noalloc(g->g, seed, first, count, alpha, np_cap, d_path_length,
                                  d_num_paths, d_vis_edges, d_status, d_records, record_cap,
                                  d_record_count, (cudaStream_t)stream);
}

int silvan_generate(int kind, uint32_t a, uint32_t b, uint32_t c, double x, double y,
                    uint64_t seed, uint32_t *pairs, uint64_t cap, uint64_t *count) {
    if (!count) {
        set_error("null argument");
        return SILVAN_E_BADARG;
    }
    EdgeList e;
    switch (kind) {
        case 0: e = gen_ba(a, b, seed); break;
        case 1: e = gen_er(a, x, seed); break;
        case 2: e = gen_rmat(a, b, 0.57, 0.19, 0.19, seed, c != 0); break;
        case 3: e = gen_grid(a, x, y, seed); break;
        default: set_error("unknown generator"); return SILVAN_E_BADARG;
    }
    *count = e.size();
    if (e.size() > cap || (!pairs && !e.empty())) {
        set_error("pair buffer too small");
        return SILVAN_E_CAPACITY;
    }
    for (size_t i = 0; i < e.size(); i++) {
        pairs[2 * i] = e[i].first;
        pairs[2 * i + 1] = e[i].second;
    }
    return SILVAN_OK;
}

}  // extern "C"
