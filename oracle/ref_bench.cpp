// Test infrastructure (oracle / CPU baseline): times the reference's own
// estimator -- silvan/src/*.cpp unmodified, including its MMIX LCG Rand_gen
// and its OpenMP threads, compiled with the reference's flags -- on a graph
// given as CSR.  Built into oracle/_ref/libsilvan_refbench.so by
// oracle/Makefile; only bench.py's reference arm and CPU-baseline leg load it.
//
// The reference can only construct its graph from a file through std::set
// insertion (silvan/src/Graph.cpp:37-90), which takes about a minute for a
// 16M-edge R-MAT and lies outside its own "Total time" window
// (silvan/src/Probabilistic.cpp:810).  The harness constructs the estimator
// on a two-node file and then installs the CSR rows in the reference's own
// per-node arrays, re-allocating the per-node counters for the real size.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <iostream>
#include <sstream>
#include <string>
#include <map>
#include <set>
#include <vector>
#include <utility>
#include <algorithm>
#include <ctype.h>
#include <unistd.h>
#include <omp.h>

#define private public
#define protected public
#include "Graph.h"
#include "Sp_sampler.h"
#include "Probabilistic.h"
#undef private
#undef protected

namespace {
struct CoutCapture {
    std::ostringstream buf;
    std::streambuf *old;
    CoutCapture() { old = std::cout.rdbuf(buf.rdbuf()); }
    ~CoutCapture() { std::cout.rdbuf(old); }
};

double last_value(const std::string &text, const std::string &pattern) {
    size_t pos = text.rfind(pattern);
    if (pos == std::string::npos) return -1.0;
    return std::strtod(text.c_str() + pos + pattern.size(), nullptr);
}

uint32_t **rows(uint32_t n, const uint64_t *off, const uint32_t *adj, uint32_t **deg) {
    uint32_t **r = (uint32_t **)malloc(sizeof(uint32_t *) * n);
    *deg = (uint32_t *)malloc(sizeof(uint32_t) * n);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t d = (uint32_t)(off[i + 1] - off[i]);
        (*deg)[i] = d;
        r[i] = (uint32_t *)malloc(sizeof(uint32_t) * (d ? d : 1));
        std::memcpy(r[i], adj + off[i], sizeof(uint32_t) * d);
    }
    return r;
}
}  // namespace

extern "C" int refbench_run(uint32_t n, int directed, const uint64_t *out_off,
                            const uint32_t *out_adj, const uint64_t *in_off,
                            const uint32_t *in_adj, double eps, double delta, uint32_t k,
                            double alpha, int alpha_given, double a, int mhat, int threads,
                            double *total_time, uint64_t *pass1, uint64_t *pass2,
                            uint64_t *vis_edges, char *stdout_buf, uint64_t stdout_cap) {
    if (threads > 0) omp_set_num_threads(threads);
    char path[] = "/tmp/silvan_refbench_XXXXXX";
    int fd = mkstemp(path);
    if (fd < 0) return -1;
    const char two[] = "0 1\n";
    if (write(fd, two, sizeof(two) - 1) != (ssize_t)(sizeof(two) - 1)) {
        close(fd);
        return -1;
    }
    close(fd);
    std::string text;
    {
        CoutCapture cap;
        Probabilistic *p = new Probabilistic(std::string(path), directed != 0, 1.0, alpha,
                                             alpha_given != 0, a, mhat != 0, std::string(""));
        unlink(path);
        // install the CSR in the reference's per-node arrays
        for (uint32_t i = 0; i < p->nodes_num; i++) free(p->adj[i]);
        free(p->adj);
        free(p->degrees);
        if (directed) {
            for (uint32_t i = 0; i < p->nodes_num; i++) free(p->inc[i]);
            free(p->inc);
            free(p->in_degrees);
        }
        free(p->cc);
        p->nodes_num = n;
        p->edges_num = out_off[n];
        p->adj = rows(n, out_off, out_adj, &p->degrees);
        if (directed) {
            p->inc = rows(n, in_off, in_adj, &p->in_degrees);
        } else {
            p->inc = p->adj;
            p->in_degrees = p->degrees;
        }
        p->cc = (uint32_t *)malloc(sizeof(uint32_t) * n);
        free(p->approx);
        free(p->approx_toadd);
        free(p->emp_wimpy_vars);
        free(p->mcrade);
        free(p->partition_index);
        p->approx = (double *)calloc(n, sizeof(double));
        p->approx_toadd = (double *)calloc(n, sizeof(double));
        p->emp_wimpy_vars = (double *)calloc(n, sizeof(double));
        p->mcrade = (int64_t *)calloc((uint64_t)n * p->mctrials, sizeof(int64_t));
        p->partition_index = (int *)calloc(n, sizeof(int));
        p->run(k, delta, eps);
        *pass2 = p->num_samples;
        *vis_edges = p->vis_edges;
        text = cap.buf.str();
        delete p;
    }
    *total_time = last_value(text, "Total time: ");
    *pass1 = (uint64_t)last_value(text, "First pass finished after ");
    if (stdout_buf && stdout_cap) {
        size_t l = std::min<size_t>(stdout_cap - 1, text.size());
        std::memcpy(stdout_buf, text.data(), l);
        stdout_buf[l] = 0;
    }
    return 0;
}

// A bounded sample of the reference's hot path: `count` calls of its own
// Sp_sampler::random_path (silvan/src/Sp_sampler.cpp:41-238, its own LCG
// streams, one sampler per OpenMP thread as in Probabilistic.cpp:825-830) on
// the CSR graph, timed over the parallel region.  Used where a complete
// estimation would take minutes on the host (the 2048 x 2048 grid).
extern "C" int refbench_sample(uint32_t n, int directed, const uint64_t *out_off,
                               const uint32_t *out_adj, const uint64_t *in_off,
                               const uint32_t *in_adj, double alpha, int threads,
                               uint64_t count, double *seconds, uint64_t *vis_edges,
                               uint64_t *paths) {
    if (threads > 0) omp_set_num_threads(threads);
    char path[] = "/tmp/silvan_refbench_XXXXXX";
    int fd = mkstemp(path);
    if (fd < 0) return -1;
    const char two[] = "0 1\n";
    if (write(fd, two, sizeof(two) - 1) != (ssize_t)(sizeof(two) - 1)) {
        close(fd);
        return -1;
    }
    close(fd);
    CoutCapture cap;
    Graph *g = new Graph(std::string(path), directed != 0);
    unlink(path);
    for (uint32_t i = 0; i < g->nodes_num; i++) free(g->adj[i]);
    free(g->adj);
    free(g->degrees);
    if (directed) {
        for (uint32_t i = 0; i < g->nodes_num; i++) free(g->inc[i]);
        free(g->inc);
        free(g->in_degrees);
    }
    free(g->cc);
    g->nodes_num = n;
    g->edges_num = out_off[n];
    g->adj = rows(n, out_off, out_adj, &g->degrees);
    if (directed) {
        g->inc = rows(n, in_off, in_adj, &g->in_degrees);
    } else {
        g->inc = g->adj;
        g->in_degrees = g->degrees;
    }
    g->cc = (uint32_t *)malloc(sizeof(uint32_t) * n);
    g->estimate_diameter();  // component ids for the void test (outside the timing)
    uint64_t next = 0, vis = 0, np_total = 0;
    const double t0 = omp_get_wtime();
#pragma omp parallel reduction(+ : vis, np_total)
    {
        Sp_sampler sp(g, 1234u + 77u * (uint32_t)omp_get_thread_num());
        for (;;) {
            uint64_t i;
#pragma omp atomic capture
            i = next++;
            if (i >= count) break;
            int pl = 0, np = 0;
            std::map<uint32_t, int> m = sp.random_path(pl, np, alpha);
            vis += sp.vis_edges;
            np_total += (uint64_t)(np > 0 ? np : 0);
        }
    }
    *seconds = omp_get_wtime() - t0;
    *vis_edges = vis;
    *paths = np_total;
    delete g;
    return 0;
}

extern "C" int refbench_max_threads() { return omp_get_max_threads(); }

// ---------------------------------------------------------------------------
// The benchmark graphs without the product library: bench.py's reference arm
// must not load libsilvan_b200.so, so this harness carries the project's
// seeded generators (silvan_b200/csrc/gen.cpp, compiled in by the Makefile)
// and its own CSR build with the reference loader's semantics
// (silvan/src/Graph.cpp:37-90: rows sorted ascending without duplicates,
// self-loops kept, n = max id + 1, each undirected edge in both rows; for
// directed graphs the in-rows hold the reverse edges).  The arm prints a
// checksum of the CSR, and so does the GPU arm, so the two can be seen to
// run on the same graph.
// ---------------------------------------------------------------------------
#include "gen.h"

namespace {
struct BuiltGraph {
    uint32_t n = 0;
    std::vector<uint64_t> out_off, in_off;
    std::vector<uint32_t> out_adj, in_adj;
};

void csr_rows(uint32_t n, std::vector<std::pair<uint32_t, uint32_t>> &e, std::vector<uint64_t> &off,
              std::vector<uint32_t> &adj) {
    std::sort(e.begin(), e.end());
    e.erase(std::unique(e.begin(), e.end()), e.end());
    off.assign((size_t)n + 1, 0);
    adj.resize(e.size());
    for (size_t i = 0; i < e.size(); i++) {
        off[e[i].first + 1]++;
        adj[i] = e[i].second;
    }
    for (uint32_t i = 0; i < n; i++) off[i + 1] += off[i];
}
}  // namespace

// kind: 0 = BA(n=a, m=b), 1 = ER(n=a, mean degree=x), 2 = R-MAT(scale=a,
// edge factor=b, directed=c; a,b,c probabilities .57,.19,.19), 3 = grid(side=a,
// delete fraction x, shortcut fraction y).  Returns a handle (nullptr on
// failure) whose sizes refbench_graph_info reports.
extern "C" void *refbench_graph_new(int kind, uint32_t a, uint32_t b, uint32_t c, double x,
                                    double y, uint64_t seed, int directed) {
    silvan::EdgeList e;
    switch (kind) {
    case 0: e = silvan::gen_ba(a, b, seed); break;
    case 1: e = silvan::gen_er(a, x, seed); break;
    case 2: e = silvan::gen_rmat(a, b, 0.57, 0.19, 0.19, seed, c != 0); break;
    case 3: e = silvan::gen_grid(a, x, y, seed); break;
    default: return nullptr;
    }
    BuiltGraph *g = new BuiltGraph();
    uint32_t mx = 0;
    for (auto &p : e) mx = std::max(mx, std::max(p.first, p.second));
    g->n = e.empty() ? 0 : mx + 1;
    std::vector<std::pair<uint32_t, uint32_t>> fwd, rev;
    fwd.reserve(directed ? e.size() : 2 * e.size());
    for (auto &p : e) {
        fwd.push_back(p);
        if (directed) rev.emplace_back(p.second, p.first);
        else fwd.emplace_back(p.second, p.first);
    }
    csr_rows(g->n, fwd, g->out_off, g->out_adj);
    if (directed) csr_rows(g->n, rev, g->in_off, g->in_adj);
    return g;
}

extern "C" void refbench_graph_info(void *h, uint32_t *n, uint64_t *m_out, uint64_t *m_in) {
    BuiltGraph *g = static_cast<BuiltGraph *>(h);
    *n = g->n;
    *m_out = g->out_adj.size();
    *m_in = g->in_adj.size();
}

extern "C" void refbench_graph_csr(void *h, uint64_t *out_off, uint32_t *out_adj,
                                   uint64_t *in_off, uint32_t *in_adj) {
    BuiltGraph *g = static_cast<BuiltGraph *>(h);
    std::memcpy(out_off, g->out_off.data(), sizeof(uint64_t) * g->out_off.size());
    std::memcpy(out_adj, g->out_adj.data(), sizeof(uint32_t) * g->out_adj.size());
    if (!g->in_off.empty()) {
        std::memcpy(in_off, g->in_off.data(), sizeof(uint64_t) * g->in_off.size());
        std::memcpy(in_adj, g->in_adj.data(), sizeof(uint32_t) * g->in_adj.size());
    }
}

extern "C" void refbench_graph_free(void *h) { delete static_cast<BuiltGraph *>(h); }
