// silvan: drop-in replacement for the reference binary (silvan/main.cpp).
// Same flags, same positional arguments, same exit codes and the stdout lines
// that scripts/run_silvan.py scrapes; the estimator runs on the GPU through
// the C-ABI of include/silvan.h.
//
//   silvan [-dhm] [-v verbosity] [-k k_value] [-o output] [-a a_emp_peeling]
//          [-s alpha] epsilon delta graph
//
// Options beyond the reference's (long options, so that the reference's
// short-option set is unchanged): --plain (one launch sequence per 11-sample
// block), --seed N (job seed), --np-cap N (paths per sample), --slots N,
// --block N (threads per sampler slot; default autotuned), --sigma-weighted
// (the path-count-weighted backtrack instead of the reference's rule),
// --assist-items N (BFS levels of at least N adjacency entries are expanded
// by several sampler CTAs; 0 = default, 4294967295 = never).
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <getopt.h>
#include <iostream>
#include <string>
#include <vector>

#include "silvan.h"

namespace {

const std::string kErr = "ERROR: ";

bool directed = false;
double verb = 60;
double delta_ = 0, err_ = 0;
const char *graph_file = nullptr;
std::string output_file;
int64_t k = 0;
double sampling_rate = 2.3;
bool alpha_given = false;
double peeling_a = 2.0;
bool m_hat = true;
bool plain = false;
uint64_t seed = 42;
uint32_t np_cap = 0, slots = 0, block = 0, assist_items = 0;
bool sigma_weighted = false;

// silvan/main.cpp:51-68
void usage(const char *b) {
    std::cerr << b << ": compute betweenness centrality approximations for all nodes" << std::endl;
    std::cerr << "USAGE: " << b
              << " [-dhm] [-v verbosity] [-k k_value] [-o output] [-a a_emp_peeling] [-s alpha] "
                 "epsilon delta graph"
              << std::endl;
    std::cerr << "\t-d: consider the graph as directed" << std::endl;
    std::cerr << "\t-k: compute the top-k betweenness centralities (if 0, compute all of them "
                 "with absolute error) "
              << std::endl;
    std::cerr << "\t-h: print this help message" << std::endl;
    std::cerr << "\t-v: print additional messages (verbosity is the time in second between "
                 "subsequent outputs)"
              << std::endl;
    std::cerr << "\t-o: path for the output file (if empty, do not write the output)" << std::endl;
    std::cerr << "\t-a: parameter a for empirical peeling (def. = 2)" << std::endl;
    std::cerr << "\t-s: parameter alpha for sampling shortest paths (def. = 2.3)" << std::endl;
    std::cerr << "\t-m: disable the computation of m_hat" << std::endl;
    std::cerr << "\terr: accuracy (0 < epsilon < 1), relative accuracy if k > 0" << std::endl;
    std::cerr << "\tdelta: confidence (0 < delta < 1)" << std::endl;
    std::cerr << "\tgraph: graph edge list file" << std::endl;
    std::cerr << "\t--plain: one launch sequence per 11-sample block (default: batched)"
              << std::endl;
    std::cerr << "\t--seed N, --np-cap N, --slots N, --block N: job seed, paths per sample, "
                 "sampler slots, threads per slot"
              << std::endl;
    std::cerr << "\t--sigma-weighted: pick predecessors by path count (not the reference's rule)"
              << std::endl;
    std::cerr << "\t--assist-items N: levels of at least N entries on several CTAs "
                 "(0 default, 4294967295 never)"
              << std::endl;
}

// silvan/main.cpp:74-153: 0 ok, 1 error, 2 help
int parse(int argc, char **argv) {
    static struct option longopts[] = {{"plain", no_argument, nullptr, 1},
                                       {"seed", required_argument, nullptr, 2},
                                       {"np-cap", required_argument, nullptr, 3},
                                       {"slots", required_argument, nullptr, 4},
                                       {"block", required_argument, nullptr, 5},
                                       {"sigma-weighted", no_argument, nullptr, 6},
                                       {"assist-items", required_argument, nullptr, 7},
                                       {nullptr, 0, nullptr, 0}};
    int opt;
    while ((opt = getopt_long(argc, argv, "dhmk:o:s:a:v:", longopts, nullptr)) != -1) {
        errno = 0;
        switch (opt) {
            case 'd': directed = true; break;
            case 'h': return 2;
            case 'm': m_hat = false; break;
            case 'o':
                std::cerr << "Writing output to " << optarg << std::endl;
                output_file = optarg;
                break;
            case 's':
                sampling_rate = std::strtod(optarg, nullptr);
                alpha_given = true;
                break;
            case 'a':
                peeling_a = std::strtod(optarg, nullptr);
                if (errno == ERANGE || peeling_a <= 1)
                    std::cerr << kErr << "The value a should be >= 1. Empirical peeling disabled."
                              << std::endl;
                alpha_given = true;
                break;
            case 'k':
                k = (int64_t)std::strtod(optarg, nullptr);
                if (errno == ERANGE || k < 0 || k > UINT_MAX) {
                    std::cerr << kErr << "The value k should be between 0 and 2^32-1." << std::endl;
                    return 1;
                }
                break;
            case 'v':
                verb = std::strtod(optarg, nullptr);
                if (errno == ERANGE || verb < 0) {
                    std::cerr << kErr
                              << "The verbosity should be a positive number, or 0 to produce no "
                                 "output."
                              << std::endl;
                    return 1;
                }
                break;
            case 1: plain = true; break;
            case 2: seed = std::strtoull(optarg, nullptr, 10); break;
            case 3: np_cap = (uint32_t)std::strtoul(optarg, nullptr, 10); break;
            case 4: slots = (uint32_t)std::strtoul(optarg, nullptr, 10); break;
            case 5: block = (uint32_t)std::strtoul(optarg, nullptr, 10); break;
            case 6: sigma_weighted = true; break;
            case 7: assist_items = (uint32_t)std::strtoul(optarg, nullptr, 10); break;
            default: break;
        }
    }
    if (optind != argc - 3) {
        std::cerr << kErr << "Wrong number of arguments" << std::endl;
        return 1;
    }
    errno = 0;
    err_ = std::strtod(argv[argc - 3], nullptr);
    if (errno == ERANGE || err_ >= 1.0 || err_ <= 0.0) {
        std::cerr << kErr << "The error err should be greater than 0 and smaller than 1"
                  << std::endl;
        return 1;
    }
    errno = 0;
    delta_ = std::strtod(argv[argc - 2], nullptr);
    if (errno == ERANGE || delta_ >= 1.0 || delta_ <= 0.0) {
        std::cerr << kErr << "Delta should be greater than 0 and smaller than 1" << std::endl;
        return 1;
    }
    graph_file = argv[argc - 1];
    std::ifstream infile(graph_file);
    if (!infile.good()) {
        std::cerr << "Problems with input graph file" << std::endl;
        return 1;
    }
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    int pr = parse(argc, argv);
    if (pr != 0) {
        usage(argv[0]);
        return pr != 2;
    }
    silvan_graph_t g = nullptr;
    int rc = silvan_graph_load(graph_file, directed ? 1 : 0, &g);
    if (rc != SILVAN_OK) {
        std::cerr << kErr << silvan_last_error() << std::endl;
        return 1;
    }
    silvan_graph_info_t info;
    silvan_graph_info(g, &info);
    // Probabilistic constructor + estimate_diameter output
    // (silvan/src/Graph.cpp:93-101,275)
    if (verb > 0) {
        std::cout << (directed ? "Directed graph\n" : "Undirected graph\n");
        std::cout << "Number of nodes: " << info.n << std::endl;
        std::cout << "Number of edges: " << info.m << std::endl;
    }
    std::cout << "n_components " << info.n_components << std::endl;
    std::cout.flush();

    silvan_params_t p;
    silvan_params_default(&p);
    p.eps = err_;
    p.delta = delta_;
    p.k = (uint32_t)k;
    p.m_hat = m_hat ? 1 : 0;
    p.alpha = sampling_rate;
    p.alpha_given = alpha_given ? 1 : 0;
    p.a = peeling_a;
    p.verbose = verb;
    p.seed = seed;
    p.form = plain ? SILVAN_FORM_PLAIN : SILVAN_FORM_BATCHED;
    p.np_cap = np_cap;
    p.slots = slots;
    p.block = block;
    p.assist_items = assist_items;
    p.backtrack = sigma_weighted ? SILVAN_BACKTRACK_SIGMA_WEIGHTED : SILVAN_BACKTRACK_REFERENCE;
    silvan_job_t j = nullptr;
    rc = silvan_job_create(g, &p, &j);
    if (rc != SILVAN_OK) {
        std::cerr << kErr << silvan_last_error() << std::endl;
        silvan_graph_destroy(g);
        return 1;
    }
    silvan_result_t res;
    rc = silvan_job_run(j, &res, stdout);
    if (rc != SILVAN_OK) {
        std::cerr << kErr << silvan_last_error() << " (status " << rc << ")" << std::endl;
        silvan_job_destroy(j);
        silvan_graph_destroy(g);
        return 1;
    }
    // output file (silvan/src/Probabilistic.cpp:1116-1136)
    if (!output_file.empty()) {
        std::ofstream of(output_file);
        if (k > 0) {
            std::vector<uint32_t> nodes(res.numresults_topk + 1);
            std::vector<double> vals(res.numresults_topk + 1);
            uint32_t cnt = 0;
            silvan_read_topk(j, nodes.data(), vals.data(), (uint32_t)nodes.size(), &cnt);
            for (uint32_t i = 0; i < cnt; i++) of << (uint64_t)nodes[i] << "," << vals[i] << "\n";
        } else {
            std::vector<double> est(info.n);
            silvan_read_estimates(j, est.data(), info.n);
            for (uint32_t i = 0; i < info.n; i++) of << (uint64_t)i << "," << est[i] << "\n";
        }
    }
    silvan_job_destroy(j);
    silvan_graph_destroy(g);
    std::cout << "run finished" << std::endl;
    return 0;
}
