// Test infrastructure (oracle): C entry points around the reference's own
// classes, compiled together with the unmodified reference sources
// (silvan/src/Graph.cpp, Sp_sampler.cpp, Probabilistic.cpp, Ranking_list.cpp,
// utilities.cpp) and the Philox Rand_gen of ref_rand_philox.cpp into
// oracle/_ref/libsilvan_ref.so.  Only tests and the fixture generator load it.
//
// Sp_sampler::random_path is wrapped at link time (-Wl,--wrap) so that every
// sample drawn by Probabilistic::run (silvan/src/Probabilistic.cpp:472) gets
// the next global sample index before its first draw; with one OpenMP thread
// the run is then a deterministic function of (graph, flags, job seed).
// Private members are reached by redefining the access keywords around the
// reference headers in this file only (after every standard header they use
// has been included); no reference file is edited.
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <iostream>
#include <sstream>
#include <string>
#include <map>
#include <vector>
#include <set>
#include <utility>
#include <ctype.h>
#include <omp.h>

#define private public
#define protected public
#include "Graph.h"
#include "Sp_sampler.h"
#include "Probabilistic.h"
#undef private
#undef protected

extern "C" {
extern uint64_t ref_job_seed;
extern uint32_t ref_sample_index;
extern int ref_rng_zero_modulus;
}

static uint32_t g_next_sample = 0;

// Per-sample record kept while recording is on.
struct SampleRec {
    uint32_t index;
    int path_length;
    int num_paths;
    uint64_t vis_edges;
    std::vector<std::pair<uint32_t, int>> nodes;
};
static bool g_recording = false;
static std::vector<SampleRec> g_records;

std::map<uint32_t, int> real_random_path(Sp_sampler *self, int &pl, int &np, double alpha)
    __asm__("__real__ZN10Sp_sampler11random_pathERiS0_d");
std::map<uint32_t, int> wrap_random_path(Sp_sampler *self, int &pl, int &np, double alpha)
    __asm__("__wrap__ZN10Sp_sampler11random_pathERiS0_d");

std::map<uint32_t, int> wrap_random_path(Sp_sampler *self, int &pl, int &np, double alpha) {
    ref_sample_index = g_next_sample++;
    std::map<uint32_t, int> r = real_random_path(self, pl, np, alpha);
    if (g_recording) {
        SampleRec rec;
        rec.index = ref_sample_index;
        rec.path_length = pl;
        rec.num_paths = np;
        rec.vis_edges = self->vis_edges;
        for (const auto &e : r) rec.nodes.push_back(e);
        g_records.push_back(std::move(rec));
    }
    return r;
}

struct CoutCapture {
    std::ostringstream buf;
    std::streambuf *old;
    CoutCapture() { old = std::cout.rdbuf(buf.rdbuf()); }
    ~CoutCapture() { std::cout.rdbuf(old); }
};

static std::string g_last_stdout;

extern "C" {

// ---- graph -----------------------------------------------------------------

void *ref_graph_load(const char *path, int directed) {
    return new Graph(std::string(path), directed != 0);
}

void ref_graph_free(void *g) { delete (Graph *)g; }

uint32_t ref_graph_nn(void *g) { return ((Graph *)g)->get_nn(); }
uint64_t ref_graph_ne(void *g) { return ((Graph *)g)->get_ne(); }

// Copies the adjacency out as CSR (out-edges, then in-edges).
void ref_graph_csr(void *gp, uint64_t *out_off, uint32_t *out_adj, uint64_t *in_off,
                   uint32_t *in_adj) {
    Graph *g = (Graph *)gp;
    uint32_t n = g->get_nn();
    uint64_t p = 0, q = 0;
    for (uint32_t i = 0; i < n; i++) {
        out_off[i] = p;
        for (uint32_t j = 0; j < g->degrees[i]; j++) out_adj[p++] = g->adj[i][j];
        in_off[i] = q;
        for (uint32_t j = 0; j < g->in_degrees[i]; j++) in_adj[q++] = g->inc[i][j];
    }
    out_off[n] = p;
    in_off[n] = q;
}

// Runs the reference's SCC + AllCCUpperBound; copies cc ids out.
uint32_t ref_graph_diameter(void *gp, uint32_t *cc_out, uint32_t *n_components) {
    Graph *g = (Graph *)gp;
    uint32_t d;
    {
        CoutCapture cap;
        d = g->estimate_diameter();
    }
    for (uint32_t i = 0; i < g->get_nn(); i++) cc_out[i] = g->cc[i];
    *n_components = g->n_components;
    return d;
}

// ---- per-sample replay -------------------------------------------------------

// Draws samples [first, first+count) with the reference sampler; the cc ids
// must have been computed (ref_graph_diameter).  Entries are the path_map
// (node, count) pairs in ascending node order, concatenated over samples.
// Returns the number of entries, or -1 if ent_cap is too small, -2 if a
// zero modulus (wrapped path count) was requested.
int64_t ref_replay(void *gp, uint64_t seed, uint32_t first, uint32_t count, double alpha,
                   int32_t *pl, int32_t *np, uint64_t *vis, uint32_t *nent,
                   uint32_t *ent_node, int32_t *ent_cnt, uint64_t ent_cap) {
    Graph *g = (Graph *)gp;
    ref_job_seed = seed;
    ref_rng_zero_modulus = 0;
    Sp_sampler sp(g, 0);
    uint64_t e = 0;
    g_records.clear();
    g_recording = true;
    g_next_sample = first;
    for (uint32_t i = 0; i < count; i++) {
        int path_length = 0, num_paths = 0;
        std::map<uint32_t, int> m;
        {
            CoutCapture cap;  // the sampler prints diagnostics on inconsistent cc ids
            m = sp.random_path(path_length, num_paths, alpha);
        }
        pl[i] = path_length;
        np[i] = num_paths;
        vis[i] = sp.vis_edges;
        nent[i] = (uint32_t)m.size();
        for (const auto &kv : m) {
            if (e >= ent_cap) {
                g_recording = false;
                return -1;
            }
            ent_node[e] = kv.first;
            ent_cnt[e] = kv.second;
            e++;
        }
    }
    g_recording = false;
    g_records.clear();
    if (ref_rng_zero_modulus) return -2;
    return (int64_t)e;
}

// ---- full run ----------------------------------------------------------------

struct RefRunResult {
    uint32_t n;
    uint32_t graph_diameter;
    uint64_t num_samples;      // pass-2 samples
    uint64_t n_pairs;          // as left by run() (pass-2 samples + tau)
    uint64_t vis_edges;
    uint64_t first_pass_samples;
    int32_t iteration_index;
    int32_t num_partitions;
    double omega;
    double first_stopping_samples;
    double last_stopping_samples;
    double alpha_sp_sampling;
    double sup_bcest;
    double sup_emp_wimpy_var;
    double eps_final_topk;
    uint32_t numresults_topk;
    uint32_t union_sample;
    int32_t zero_modulus;
    int32_t pad;
};

static Probabilistic *g_prob = nullptr;
static uint64_t g_first_pass_samples = 0;

// Runs Probabilistic::run with one OpenMP thread and keeps the object for the
// accessors below.  Stdout is captured (ref_last_stdout).
int ref_run(const char *path, int directed, double eps, double delta, uint32_t k, double alpha,
            int alpha_given, double a, int mhat, uint64_t seed, const char *output_file,
            double verbose, RefRunResult *res) {
    omp_set_num_threads(1);
    if (g_prob) {
        delete g_prob;
        g_prob = nullptr;
    }
    ref_job_seed = seed;
    ref_rng_zero_modulus = 0;
    g_next_sample = 0;
    g_recording = false;
    {
        CoutCapture cap;
        g_prob = new Probabilistic(std::string(path), directed != 0, verbose, alpha,
                                   alpha_given != 0, a, mhat != 0,
                                   std::string(output_file ? output_file : ""));
        g_prob->run(k, delta, eps);
        g_last_stdout = cap.buf.str();
    }
    Probabilistic *p = g_prob;
    res->n = p->get_nn();
    res->graph_diameter = (uint32_t)p->graph_diameter;
    res->num_samples = p->num_samples;
    res->n_pairs = p->n_pairs;
    res->vis_edges = p->vis_edges;
    res->first_pass_samples = 0;
    res->iteration_index = p->iteration_index;
    res->num_partitions = p->number_of_non_empty_partitions;
    res->omega = p->omega;
    res->first_stopping_samples = p->first_stopping_samples;
    res->last_stopping_samples = p->last_stopping_samples;
    res->alpha_sp_sampling = p->alpha_sp_sampling;
    res->sup_bcest = p->sup_bcest;
    res->sup_emp_wimpy_var = p->sup_emp_wimpy_var;
    res->eps_final_topk = p->eps_final_topk;
    res->numresults_topk = p->numresults_topk;
    res->union_sample = p->union_sample;
    res->zero_modulus = ref_rng_zero_modulus;
    (void)g_first_pass_samples;
    return 0;
}

const char *ref_last_stdout() { return g_last_stdout.c_str(); }

void ref_run_arrays(double *approx, double *wimpy, int64_t *mcrade, int32_t *partition_index) {
    Probabilistic *p = g_prob;
    uint32_t n = p->get_nn();
    std::memcpy(approx, p->approx, sizeof(double) * n);
    std::memcpy(wimpy, p->emp_wimpy_vars, sizeof(double) * n);
    std::memcpy(mcrade, p->mcrade, sizeof(int64_t) * (uint64_t)n * p->mctrials);
    std::memcpy(partition_index, p->partition_index, sizeof(int32_t) * n);
}

// Ranking list after the run: union_sample (element, value) pairs.
void ref_run_ranking(uint32_t *elements, double *values) {
    Probabilistic *p = g_prob;
    for (uint32_t i = 0; i < p->union_sample; i++) {
        elements[i] = p->top_k->get(i);
        values[i] = p->top_k->get_value(i);
    }
}

void ref_run_partitions(double *epsilon_partition, int32_t *partition_ids) {
    Probabilistic *p = g_prob;
    for (int i = 0; i < p->number_of_non_empty_partitions; i++)
        epsilon_partition[i] = p->epsilon_partition[i];
    int j = 0;
    for (const auto &kv : p->partitions_ids_map) partition_ids[j++] = kv.first;
}

void ref_run_sp_lengths(uint64_t *out) {
    Probabilistic *p = g_prob;
    for (int i = 0; i <= p->graph_diameter; i++) out[i] = p->sp_lengths[i];
}

void ref_run_free() {
    if (g_prob) {
        delete g_prob;
        g_prob = nullptr;
    }
}

}  // extern "C"
