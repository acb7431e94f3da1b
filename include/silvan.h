/*
 * silvan.h -- C-ABI of the B200 progressive-sampling betweenness estimator.
 *
 * The reference (SILVAN) has no in-process API: its boundary is the binary's
 * command line (silvan/main.cpp:38-154) driving Probabilistic::run
 * (silvan/src/Probabilistic.cpp:775-1139), which calls Sp_sampler::random_path
 * once per sample (silvan/src/Sp_sampler.cpp:41-238).  The entry points below
 * replace that chain one-for-one; each comment names the reference interface
 * it stands in for.  Plain pointers and sizes only; the caller owns every
 * host buffer, a handle owns its device memory.
 *
 * Conventions
 *   - Every call returns int: SILVAN_OK (0) or a negative SILVAN_E_* code;
 *     silvan_last_error() returns a message for the calling thread.
 *   - Nothing traps.  Conditions under which the reference divides by zero
 *     or loops for hours are reported as status codes.
 *   - A job is bound to one CUDA stream.  Calls on one job are not
 *     thread-safe; different jobs may be driven from different host threads.
 */
#ifndef SILVAN_H
#define SILVAN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define SILVAN_OK 0
#define SILVAN_E_BADARG -1    /* invalid argument or handle                  */
#define SILVAN_E_IO -2        /* graph file cannot be read                   */
#define SILVAN_E_PARSE -3     /* node id the reference cannot represent      */
#define SILVAN_E_OOM -4       /* device or host allocation failed            */
#define SILVAN_E_CUDA -5      /* CUDA runtime error                          */
#define SILVAN_E_OVERFLOW -6  /* wrapped 64-bit path count reached 0; the
                                 reference divides by zero there
                                 (silvan/src/Rand_gen.cpp:24)                */
#define SILVAN_E_NP_CAP -7    /* alpha * W paths for one sample exceed the
                                 job's cap (silvan/src/Sp_sampler.cpp:166-170
                                 can ask for ~2^31 backtracks per sample)    */
#define SILVAN_E_TIMEOUT -8   /* a bounded device wait expired               */
#define SILVAN_E_CAPACITY -9  /* a per-round buffer is too small             */
#define SILVAN_E_STATE -10    /* call out of order                           */
#define SILVAN_E_NOGPU -11    /* no usable CUDA device                       */

/* ---- handles ------------------------------------------------------------- */
typedef struct silvan_graph_s *silvan_graph_t;
typedef struct silvan_job_s *silvan_job_t;

typedef struct {
    uint32_t n;             /* nodes (1 + largest id)                       */
    uint32_t n_components;  /* strongly connected components                */
    uint64_t m;             /* directed edge entries (edges_num)            */
    uint32_t diameter;      /* AllCCUpperBound diameter bound               */
    int32_t directed;
} silvan_graph_info_t;

/* Execution forms of the sampling loop. */
#define SILVAN_FORM_PLAIN 0    /* one launch sequence per 11-sample block   */
#define SILVAN_FORM_BATCHED 1  /* persistent sampler per schedule interval  */

/* Estimator parameters: the binary's flags (silvan/main.cpp:20-33,63-137). */
typedef struct {
    double eps;          /* accuracy, absolute (k == 0) or relative (k > 0) */
    double delta;        /* confidence                                      */
    uint32_t k;          /* -k: top-k relative mode when > 0                */
    int32_t m_hat;       /* 0 disables m_hat (-m)                           */
    double alpha;        /* -s: multi-path sampling rate (default 2.3)      */
    int32_t alpha_given; /* -s or -a given: keeps alpha fixed in pass 2     */
    int32_t form;        /* SILVAN_FORM_*                                   */
    double a;            /* -a: empirical peeling base (default 2); <= 1 off */
    uint64_t seed;       /* Philox key of the job (default 42)              */
    double verbose;      /* -v: seconds between progress lines (default 60) */
    uint32_t np_cap;     /* max paths per sample (0 = default 2^24)         */
    uint32_t slots;      /* concurrent sampler slots (0 = autotuned)        */
    uint32_t threads;    /* divisor of union_sample (0 = 1, parity mode)    */
    uint32_t block;      /* threads per sampler slot: 0 = autotuned per graph
                            and round, else 128, 256, 512 or 1024            */
    uint32_t backtrack;  /* SILVAN_BACKTRACK_*                               */
    uint32_t assist_items; /* BFS levels of at least this many adjacency
                            entries are expanded by several sampler CTAs
                            together (same results): 0 = default (128 x the
                            CTA size while samples remain to be handed out,
                            64 x once all are taken), 0xffffffff = never    */
    uint32_t wait_polls; /* polls after which a wait between the CTAs that
                            share a level gives up (the sample then reports
                            SILVAN_E_TIMEOUT and the job fails; later jobs
                            are unaffected): 0 = default (2^20, far above
                            any real wait), 0xffffffff = no polls at all (a
                            hook for tests of that failure path)            */
    uint32_t serial_checks; /* absolute mode: 0 = default, the commit of the
                            samples after a stopping-rule check runs while
                            the host evaluates the check (and is undone if
                            the check stops the run); 1 = each check is
                            evaluated before any later sample is committed.
                            The results are the same.                       */
} silvan_params_t;

/* Predecessor choice of the random backtrack.  REFERENCE is the rule of
 * silvan/src/Sp_sampler.cpp:241-265 as written (its running counter adds
 * n_paths of the sample's endpoint, 1, per predecessor: bit-exact parity).
 * SIGMA_WEIGHTED adds n_paths of each predecessor instead (in 64 bits), so
 * every shortest path is equally likely; it is an option of this library and
 * outside the reference's parity. */
#define SILVAN_BACKTRACK_REFERENCE 0
#define SILVAN_BACKTRACK_SIGMA_WEIGHTED 1

/* Fills p with the reference defaults. */
void silvan_params_default(silvan_params_t *p);

/* Result of a finished run: the values the reference prints. */
typedef struct {
    uint64_t first_pass_samples; /* "First pass finished after N iteration" */
    uint64_t num_samples;        /* pass-2 samples ("Finished after")       */
    uint64_t vis_edges;          /* edges visited, both passes              */
    uint64_t void_samples;       /* pass-2 void samples                     */
    uint64_t backtracked_paths;  /* sum of num_paths over counted samples   */
    uint32_t tau;
    uint32_t diameter;
    int32_t iteration_index;
    int32_t num_partitions;
    int32_t stop_reason;         /* 1 = eps condition, 2 = omega reached    */
    uint32_t union_sample;
    uint32_t numresults_topk;
    uint32_t checks;             /* stopping-rule evaluations               */
    double omega;
    double first_stopping_samples;
    double last_stopping_samples;
    double alpha_sp_sampling;    /* alpha used in pass 2                    */
    double eps_stop;             /* sup eps at the stop, -1 if none          */
    double eps_final_topk;
    double sup_bcest;            /* max approx / num_samples                */
    double sup_emp_wimpy_var;    /* max wimpy / num_samples                 */
    double max_num_samples;      /* m_hat after pass 1                      */
    double time_total_s;         /* "Total time" window                     */
    double time_first_pass_s;
    double time_sampling_s;      /* device time in the sampler              */
    double time_apply_s;         /* device time in counter application     */
    double time_device_s;        /* device time of the whole run (events)   */
    uint64_t ball_nodes;         /* nodes visited by all samples            */
    uint64_t pred_entries;       /* predecessor entries of all samples      */
    uint64_t kernel_launches;    /* kernels launched by the run             */
    uint32_t sampler_launches;   /* persistent sampler launches (own engine) */
    uint32_t sampler_block;      /* CTA size that drew most samples          */
    uint64_t samples_drawn;      /* samples drawn, speculative ones included */
    uint32_t assisted_levels;    /* BFS levels expanded by several CTAs (own
                                    engine; see silvan_params_t::assist_items) */
    uint32_t overlapped_checks;  /* checks during whose evaluation the next
                                    samples were committed (and kept)      */
    uint64_t helper_tiles;       /* tiles of those levels done by helpers    */
} silvan_result_t;

/* ---- graphs (reference: Graph, silvan/src/Graph.cpp) ------------------- */

/* Graph(filename, directed) (silvan/src/Graph.cpp:37-90) followed by
 * compute_cc + estimate_diameter (silvan/src/Graph.cpp:109-316).  The edge
 * list is parsed and the CSR built on the device, with the reference
 * loader's line semantics (the same graph as silvan_host_graph_load); the
 * components and the diameter bound are computed on a host copy. */
int silvan_graph_load(const char *path, int directed, silvan_graph_t *out);

/* Same, from host CSR arrays (rows ascending, unique).  in_off/in_adj are
 * ignored for undirected graphs.  cc may be NULL, in which case the
 * components and the diameter bound are computed on the host. */
int silvan_graph_upload(uint32_t n, int directed, const uint64_t *out_off,
                        const uint32_t *out_adj, const uint64_t *in_off,
                        const uint32_t *in_adj, const uint32_t *cc,
                        uint32_t n_components, uint32_t diameter,
                        silvan_graph_t *out);

int silvan_graph_info(silvan_graph_t g, silvan_graph_info_t *info);

/* Host CSR of a loaded graph (out rows, then in rows; in rows alias the
 * out rows for undirected graphs).  Sizes from silvan_graph_info. */
int silvan_graph_csr(silvan_graph_t g, uint64_t *out_off, uint32_t *out_adj,
                     uint64_t *in_off, uint32_t *in_adj, uint32_t *cc);

int silvan_graph_destroy(silvan_graph_t g);

/* ---- host-only ingest ------------------------------------------------------
 * The same ingest without a device: edge-list parse, CSR, components and
 * diameter bound (silvan/src/Graph.cpp:37-316).  Useful to prepare graphs on
 * machines without a GPU; silvan_graph_from_host uploads one. */
typedef struct silvan_host_graph_s *silvan_host_graph_t;
int silvan_host_graph_load(const char *path, int directed, silvan_host_graph_t *out);
int silvan_host_graph_from_pairs(const uint32_t *pairs, uint64_t count, int directed,
                                 silvan_host_graph_t *out);
int silvan_host_graph_info(silvan_host_graph_t g, silvan_graph_info_t *info);
int silvan_host_graph_csr(silvan_host_graph_t g, uint64_t *out_off, uint32_t *out_adj,
                          uint64_t *in_off, uint32_t *in_adj, uint32_t *cc);
int silvan_host_graph_destroy(silvan_host_graph_t g);
int silvan_graph_from_host(silvan_host_graph_t h, silvan_graph_t *out);

/* ---- jobs (reference: Probabilistic, silvan/include/Probabilistic.h) ---- */

/* Probabilistic(...) constructor: allocates the device counters. */
int silvan_job_create(silvan_graph_t g, const silvan_params_t *p, silvan_job_t *out);

/* Probabilistic::run(k, delta, err): pass 1, empirical peeling, bounds,
 * pass 2 with the progressive stopping rule.  Status lines of the
 * reference are written to `log` when it is not NULL. */
int silvan_job_run(silvan_job_t j, silvan_result_t *res, void *log /* FILE* */);

/* get_centrality(v) for every node: approx[v] / num_samples. */
int silvan_read_estimates(silvan_job_t j, double *out, uint32_t n);

/* Ranked output of top-k mode: the numresults_topk (node, estimate) pairs in
 * ranking order (silvan/src/Probabilistic.cpp:1121-1127). */
int silvan_read_topk(silvan_job_t j, uint32_t *nodes, double *values, uint32_t cap,
                     uint32_t *count);

/* Raw pass-2 counters: approx (double), emp_wimpy_vars (double), mcrade
 * (int64, n x 25, node-major) and partition_index (int32).  Any pointer may
 * be NULL. */
int silvan_read_counters(silvan_job_t j, double *approx, double *wimpy, int64_t *mcrade,
                         int32_t *partition_index);

int silvan_job_destroy(silvan_job_t j);

/* ---- step-wise interface ------------------------------------------------- */

/* Progress of the sampling loop. */
typedef struct {
    uint64_t samples;       /* samples committed in the current pass        */
    uint64_t void_samples;  /* void samples of the current pass              */
    uint64_t vis_edges;     /* edges visited in the current pass             */
    uint64_t backtracked_paths;
    int32_t pass;           /* 1 or 2                                       */
    int32_t done;           /* 1 once the stopping rule has fired           */
} silvan_status_t;

/* Advances the estimator by at most `rounds` rounds of its own schedule.  A
 * round draws the samples up to the next point at which the reference acts
 * (the end of pass 1, a stopping-rule evaluation, the omega cap; every
 * 11-sample block in the plain form), commits them in sample order
 * (Probabilistic::one_round, silvan/src/Probabilistic.cpp:468-559) and
 * evaluates that point.  The first call starts the run; results are read
 * with silvan_job_result once status.done is set. */
int silvan_run_rounds(silvan_job_t j, uint32_t rounds, silvan_status_t *st, void *log);

/* Result of a finished job (after silvan_job_run or the last round). */
int silvan_job_result(silvan_job_t j, silvan_result_t *res);

/* ---- multi-graph batching ------------------------------------------------- */

/* Runs `count` jobs (on the same or different graphs) to completion with one
 * persistent sampler launch per round serving every unfinished job, each job
 * following its own schedule (no counterpart in the reference, which runs one
 * graph per process).  Sampler slots are sized for the largest graph; they
 * take at most mem_budget bytes (0 = half of the free device memory).
 * results[i] receives job i's result.  Each job's estimates are the same as
 * when it runs alone. */
int silvan_jobs_run_batched(silvan_job_t *jobs, uint32_t count, uint64_t mem_budget,
                            silvan_result_t *results, void *log);

/* ---- serving ---------------------------------------------------------------
 * An estimation server with continuous batching (no counterpart in the
 * reference, which runs one estimation per process).  Requests are submitted
 * from any thread; one server thread owns the device, admits queued requests
 * in arrival order while their device memory fits the budget, keeps their
 * graphs and sampler state on the device, and serves every active request in
 * each round's single persistent sampler launch.  A request's result is the
 * same as when it runs alone. */
typedef struct silvan_server_s *silvan_server_t;

#define SILVAN_REQ_QUEUED 1
#define SILVAN_REQ_RUNNING 2
#define SILVAN_REQ_DONE 3   /* negative values: the request failed (SILVAN_E_*) */

typedef struct {
    uint64_t rounds;        /* sampler rounds run                             */
    uint64_t samples;       /* samples drawn over all requests                */
    uint64_t max_active;    /* most requests served by one round              */
    uint64_t queued, active;
    uint64_t bytes_in_use;  /* device bytes held by admitted requests        */
    uint64_t budget;        /* admission budget                               */
    uint32_t slots;         /* sampler slots                                  */
    uint32_t pad;
    /* where the server thread's time went (seconds, totals and the longest
     * single occurrence): admitting requests (upload, job set-up), sampler
     * rounds, committing and evaluating, finishing (read-back, release) */
    double admit_s, round_s, commit_s, finish_s;
    double admit_max_s, round_max_s, commit_max_s, finish_max_s;
} silvan_server_stats_t;

/* n_max: largest graph (nodes) the server accepts; the sampler slots are
 * sized for it.  budget: device bytes for admitted requests (0 = a third of
 * the free memory).  slots: 0 = occupancy x SM count. */
int silvan_server_create(uint64_t n_max, uint64_t budget, uint32_t slots, silvan_server_t *out);
/* Queues an estimation of graph g (copied; g may be destroyed afterwards). */
int silvan_server_submit(silvan_server_t s, silvan_host_graph_t g, const silvan_params_t *p,
                         uint64_t *id);
/* state: SILVAN_REQ_*; once done, res, the latency from submission to the
 * result and the time spent queued are filled. */
int silvan_server_poll(silvan_server_t s, uint64_t id, int32_t *state, silvan_result_t *res,
                       double *latency_s, double *queued_s);
/* Blocks until the request finished or timeout_s passed (SILVAN_E_TIMEOUT). */
int silvan_server_wait(silvan_server_t s, uint64_t id, double timeout_s);
/* Estimates (approx / num_samples, n entries) and, in top-k mode, the ranked
 * output of a finished request.  Any pointer may be NULL. */
int silvan_server_estimates(silvan_server_t s, uint64_t id, double *out, uint32_t n,
                            uint32_t *topk_nodes, double *topk_values, uint32_t topk_cap,
                            uint32_t *topk_count);
int silvan_server_stats(silvan_server_t s, silvan_server_stats_t *st);
int silvan_server_destroy(silvan_server_t s);

/* ---- exact betweenness (validation) --------------------------------------- */

/* Exact betweenness of every node (Brandes, on the device), normalised by
 * n (n - 1) over ordered pairs: the quantity the estimator approximates, for
 * checking the (eps, delta) guarantee.  No counterpart in the reference,
 * which has no exact algorithm.  out has n entries. */
int silvan_exact_betweenness(silvan_graph_t g, double *out, uint32_t n);

/* ---- per-sample replay (parity hook) -------------------------------------- */

/* Runs the device sampler for global sample indices [first, first+count)
 * and returns, per sample, what Sp_sampler::random_path returns
 * (silvan/src/Sp_sampler.cpp:41-238): path_length, num_paths, vis_edges and
 * the path map (node -> count, ascending node id), concatenated in
 * ent_node/ent_cnt with nent[i] entries for sample i.  sample_status[i] is 0
 * or a SILVAN_E_* code for that sample.  Returns SILVAN_E_CAPACITY when
 * ent_cap is too small (*ent_total then holds the size needed). */
int silvan_replay_samples(silvan_graph_t g, uint64_t seed, uint32_t first, uint32_t count,
                          double alpha, uint32_t np_cap, int32_t *path_length,
                          int32_t *num_paths, uint64_t *vis_edges, uint32_t *nent,
                          int32_t *sample_status, uint32_t *ent_node, int32_t *ent_cnt,
                          uint64_t ent_cap, uint64_t *ent_total);

/* No counterpart in the reference.  The same per-sample sampler as
 * silvan_replay_samples, for callers that cannot let a library allocate
 * device memory: a process that shares the GPU under a quota it already
 * holds in full, or a runtime that gives its libraries only buffers it
 * allocated itself.  It calls no cudaMalloc/cudaFree or other allocating
 * routine: the sampler's scratch is a fixed 64 MiB static device array (held
 * by every GPU that loads the library until exit), which limits a call to
 * graphs of at most 1,489,408 nodes and to 65536 samples (SILVAN_E_CAPACITY
 * beyond, with the limit in silvan_last_error()).  The graph's device must
 * be current (SILVAN_E_BADARG otherwise).  Every output is a DEVICE buffer
 * supplied by the caller; d_records receives (node, sample, count) triples,
 * unordered, whose sample field is the index relative to `first` (0 for
 * sample `first`), and *d_record_count their number (when it exceeds
 * record_cap the surplus is dropped and the affected samples carry
 * SILVAN_E_CAPACITY; slots below record_cap that such a sample had reserved
 * hold placeholders with count 0 and node 0xFFFFFFFF, to be skipped).  The
 * work is queued on `stream` (a cudaStream_t, NULL
 * for the default stream); outputs are ready when the stream reaches it.  The
 * first call on a device looks up the scratch's device address (and caches
 * it: the cache does not survive cudaDeviceReset), so it should come before
 * any stream capture.  All calls share the scratch, so calls that overlap on
 * the GPU race. */
int silvan_replay_samples_noalloc(silvan_graph_t g, uint64_t seed, uint32_t first,
                                  uint32_t count, double alpha, uint32_t np_cap,
                                  int32_t *d_path_length, int32_t *d_num_paths,
                                  uint64_t *d_vis_edges, int32_t *d_status,
                                  uint32_t *d_records, uint64_t record_cap,
                                  unsigned long long *d_record_count, void *stream);

/* ---- synthetic workloads --------------------------------------------------- */

/* Generators of the measured workloads; they write at most cap (u, v) pairs
 * to pairs[2*i], pairs[2*i+1] and return the count in *count (when the
 * buffer is too small, *count is the size needed and SILVAN_E_CAPACITY is
 * returned).  kind: 0 = BA(n=a, m=b), 1 = ER(n=a, mean degree=x),
 * 2 = R-MAT(scale=a, edge factor=b, directed=c), 3 = grid(side=a, delete
 * fraction x, shortcut fraction y). */
int silvan_generate(int kind, uint32_t a, uint32_t b, uint32_t c, double x, double y,
                    uint64_t seed, uint32_t *pairs, uint64_t cap, uint64_t *count);

/* Builds a graph handle directly from (u, v) pairs with the loader's
 * semantics (dedup, sorted rows, reverse edges when undirected). */
int silvan_graph_from_pairs(const uint32_t *pairs, uint64_t count, int directed,
                            silvan_graph_t *out);

/* ---- misc ------------------------------------------------------------------ */
const char *silvan_last_error(void);
const char *silvan_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SILVAN_H */
