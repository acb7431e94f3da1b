// Test infrastructure (oracle) -- NOT part of the product.  A plain,
// single-threaded C++ restatement of SILVAN's progressive-sampling estimator
// in "parity mode" (the reference's one-thread semantics with the Philox
// stream of oracle_philox.h replacing the LCG).  Only tests/, the smoke check
// and bench.py's CPU-baseline leg load it (as oracle/_ref/liboracle.so).
// It is itself checked against the reference sources compiled with the same
// stream (oracle/_ref/libsilvan_ref.so, built by oracle/Makefile).
//
// Each function cites the reference code it restates (paths relative to the
// SILVAN repository).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "oracle_philox.h"

namespace {

struct OGraph {
    uint32_t n = 0;
    bool directed = false;
    uint64_t m = 0;
    std::vector<uint64_t> out_off, in_off;
    std::vector<uint32_t> out_adj, in_adj;
    std::vector<uint32_t> cc;
    const uint64_t *ioff() const { return directed ? in_off.data() : out_off.data(); }
    const uint32_t *iadj() const { return directed ? in_adj.data() : out_adj.data(); }
};

// One stream of draws for one sample (silvan/src/Rand_gen.cpp:15-25 with the
// LCG replaced by Philox; get_max keeps the low 32 bits of the draw).
struct Stream {
    uint64_t seed;
    uint32_t sample, kind, draw = 0;
    bool zero_mod = false;
    uint64_t get() { return oracle_draw(seed, sample, kind, draw++); }
    uint64_t get_max(uint64_t m) {
        uint32_t r = (uint32_t)get();
        if (m == 0) {
            zero_mod = true;
            return 0;
        }
        return r % m;
    }
};

struct SampleOut {
    int path_length = 0;
    int num_paths = 0;
    uint64_t vis_edges = 0;
    std::vector<std::pair<uint32_t, int>> nodes;  // ascending node id
    bool zero_mod = false;
};

// Per-sampler scratch (silvan/src/Sp_sampler.cpp:13-29).
struct Scratch {
    std::vector<uint32_t> ball, dist, q;
    std::vector<uint64_t> sigma;
    std::vector<std::vector<uint32_t>> pred;
    explicit Scratch(uint32_t n) : ball(n, 0), dist(n, 0), q(n, 0), sigma(n, 0), pred(n) {}
};

enum { UNVISITED = 0, SIDE_U = 1, SIDE_V = 2 };

// Walks predecessor lists from `start` to an endpoint
// (silvan/src/Sp_sampler.cpp:241-265).  The running counter adds
// n_paths[v] of the sample's endpoint v, which is always 1, so the chosen
// predecessor is pred[start][min(r, |pred|-1)] with r = draw mod sigma(start).
// With `weighted` the counter adds n_paths[w] of the predecessor itself (in
// 64 bits), the rule that picks each shortest path with equal probability;
// it is an option of this library, not the reference's behaviour.
void backtrack(const Scratch &s, Stream &rng, uint32_t u, uint32_t v, uint32_t start,
               std::vector<uint32_t> &path, bool weighted) {
    while (start != u && start != v) {
        path.push_back(start);
        uint32_t r = (uint32_t)rng.get_max(s.sigma[start]);
        const std::vector<uint32_t> &p = s.pred[start];
        uint32_t w = 0;
        uint32_t acc = 0;
        uint64_t acc64 = 0;
        for (uint32_t t = 0; t < p.size(); t++) {
            w = p[t];
            if (weighted) {
                acc64 += s.sigma[w];
                if (acc64 > r) break;
            } else {
                acc += (uint32_t)s.sigma[v];
                if (acc > r) break;
            }
        }
        start = w;
    }
}

// silvan/src/Sp_sampler.cpp:41-238 (random_path).
void sample_one(const OGraph &g, Scratch &s, uint64_t seed, uint32_t index, double alpha,
                SampleOut &out, bool weighted = false) {
    Stream rng{seed, index, 0};
    out = SampleOut();
    const uint32_t n = g.n;
    uint32_t v = (uint32_t)rng.get_max(n);
    uint32_t u = (uint32_t)rng.get_max(n);
    while (u == v) v = (uint32_t)rng.get_max(n);
    // void test on component ids (:62-74)
    if (g.directed ? (g.cc[u] < g.cc[v]) : (g.cc[u] != g.cc[v])) {
        out.zero_mod = rng.zero_mod;
        return;
    }
    uint32_t end_q = 2;
    s.q[0] = u;
    s.q[1] = v;
    s.ball[u] = SIDE_U;
    s.ball[v] = SIDE_V;
    s.sigma[u] = 1;
    s.dist[u] = 0;
    s.sigma[v] = 1;
    s.dist[v] = 0;
    uint32_t start_u = 0, end_u = 1, start_v = 1, end_v = 2;
    uint32_t sum_u = 0, sum_v = 0;
    bool stop = false;
    std::vector<std::pair<uint32_t, uint32_t>> meet;
    uint64_t vis = 0;
    while (!stop) {
        // expand the side with the smaller degree sum, u on ties (:91-113)
        bool side_u = (sum_u <= sum_v);
        uint32_t lo, hi;
        uint32_t *new_end;
        uint32_t *sum;
        const uint64_t *off;
        const uint32_t *adj;
        if (side_u) {
            lo = start_u;
            hi = end_u;
            start_u = end_q;
            end_u = end_q;
            new_end = &end_u;
            sum_u = 0;
            sum = &sum_u;
            off = g.out_off.data();
            adj = g.out_adj.data();
        } else {
            lo = start_v;
            hi = end_v;
            start_v = end_q;
            end_v = end_q;
            new_end = &end_v;
            sum_v = 0;
            sum = &sum_v;
            off = g.ioff();
            adj = g.iadj();
        }
        for (uint32_t i = lo; i < hi; i++) {  // (:116-140)
            uint32_t x = s.q[i];
            for (uint64_t e = off[x]; e < off[x + 1]; e++) {
                vis++;
                uint32_t y = adj[e];
                if (s.ball[y] == UNVISITED) {
                    *sum += (uint32_t)(off[y + 1] - off[y]);
                    s.sigma[y] = s.sigma[x];
                    s.ball[y] = s.ball[x];
                    s.q[end_q++] = y;
                    (*new_end)++;
                    s.pred[y].push_back(x);
                    s.dist[y] = s.dist[x] + 1;
                } else if (s.ball[y] != s.ball[x]) {
                    stop = true;
                    meet.emplace_back(x, y);
                } else if (s.dist[y] == s.dist[x] + 1) {
                    s.sigma[y] += s.sigma[x];
                    s.pred[y].push_back(x);
                }
            }
        }
        if (*sum == 0) stop = true;  // (:141-143)
    }
    out.vis_edges = vis;
    auto reset = [&]() {
        for (uint32_t i = 0; i < end_q; i++) {
            s.ball[s.q[i]] = UNVISITED;
            s.pred[s.q[i]].clear();
        }
    };
    if (meet.empty()) {  // (:146-157)
        reset();
        out.zero_mod = rng.zero_mod;
        return;
    }
    uint64_t W = 0;  // (:159-161), wrapping
    for (auto &p : meet) W += s.sigma[p.first] * s.sigma[p.second];
    int np = 1;  // (:166-170); out-of-range double->int gives INT_MIN on x86
    if (alpha > 0. && W > 1) {
        double t = alpha * (double)W;
        np = (t >= 2147483648.0 || t < -2147483648.0 || t != t) ? INT32_MIN : (int)t;
    }
    out.num_paths = np;
    std::map<uint32_t, int> hits;
    std::vector<uint32_t> path;
    for (int j = 0; j < np; j++) {  // (:172-197)
        uint32_t r = (uint32_t)rng.get_max(W);
        path.clear();
        uint64_t cum = 0;
        for (auto &p : meet) {
            cum += s.sigma[p.first] * s.sigma[p.second];
            if (cum > r) {
                backtrack(s, rng, u, v, p.first, path, weighted);
                backtrack(s, rng, u, v, p.second, path, weighted);
                break;
            }
        }
        if (j == 0) out.path_length = (int)path.size();
        for (uint32_t w : path) hits[w] += 1;
    }
    for (auto &kv : hits) out.nodes.push_back(kv);
    reset();
    out.zero_mod = rng.zero_mod;
}

// ---------------------------------------------------------------------------
// Fixed-length descending list (silvan/src/Ranking_list.cpp:8-43): on equal
// values the most recent update goes first.
struct Ranking {
    std::vector<uint32_t> el;
    std::vector<double> val;
    explicit Ranking(uint32_t k) : el(k), val(k, 0.0) {
        for (uint32_t i = 0; i < k; i++) el[i] = i;
    }
    void put(uint32_t e, double nv) {
        uint32_t k = (uint32_t)el.size();
        uint32_t i;
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

struct Params {
    double eps, delta;
    uint32_t k;
    double alpha;
    int alpha_given;
    double a;
    int mhat;
    uint64_t seed;
    uint32_t threads;  // union_sample divisor (1 in parity mode)
    int weighted;      // sigma-weighted backtrack (an option, not the reference)
};

struct Result {
    uint32_t graph_diameter;
    uint32_t tau;
    uint64_t first_pass_samples;
    uint64_t num_samples;
    uint64_t vis_edges;
    int32_t iteration_index;
    int32_t num_partitions;
    double omega;
    double first_stopping_samples;
    double last_stopping_samples;
    double alpha_sp_sampling;
    double sup_bcest;
    double sup_emp_wimpy_var;
    double eps_final_topk;
    double eps_stop;  // sup eps at the stopping check, or -1
    uint32_t numresults_topk;
    uint32_t union_sample;
    int32_t stop_reason;  // 1 = eps condition, 2 = omega cap
    int32_t zero_modulus;
    uint64_t checks;
};

struct Run {
    const OGraph &g;
    Params p;
    uint32_t D;
    bool absolute;
    std::vector<double> approx, approx_toadd, wimpy;
    std::vector<int64_t> mcrade;
    std::vector<int> part;
    std::map<int, int> part_map;
    int nparts = 0;
    std::vector<uint64_t> sp_lengths;
    uint64_t n_pairs = 0, num_samples = 0, vis_edges = 0, void_samples = 0;
    uint64_t distinct = 0;
    double sup_bcest = 0, sup_wv = 0;
    bool firstpass = true;
    double alpha;
    Ranking *topk = nullptr;
    uint32_t union_sample = 0, k = 0;
    uint32_t next_index = 0;  // global sample index
    Scratch scratch;
    std::vector<double> eps_part;
    double omega = 0, first_stop = 0, last_stop = 0, dfpb = 0;
    uint64_t next_stop = 0;
    int iteration = 0;
    double eps_final_topk = 0;
    uint32_t numresults_topk = 0;
    bool zero_mod = false;
    double eps_stop = -1;
    uint64_t checks = 0;
    const int T = 25;  // mctrials (silvan/include/Probabilistic.h:89)

    Run(const OGraph &g_, const Params &p_, uint32_t D_)
        : g(g_), p(p_), D(D_), scratch(g_.n) {}

    // silvan/src/Probabilistic.cpp:468-559
    void one_round() {
        SampleOut s;
        uint32_t idx = next_index++;
        sample_one(g, scratch, p.seed, idx, alpha, s, p.weighted != 0);
        if (s.zero_mod) zero_mod = true;
        n_pairs++;
        vis_edges += s.vis_edges;
        num_samples++;
        if (s.path_length <= 0) {
            void_samples++;
            return;
        }
        int sig[25];
        if (!firstpass) {
            Stream r{p.seed, idx, 1};
            for (int j = 0; j < T; j++) sig[j] = (r.get_max(100000000) >= 50000000.0) * 2 - 1;
        }
        double one_over = 1. / (double)s.num_paths;
        for (auto &kv : s.nodes) {
            uint32_t u = kv.first;
            double x = kv.second * one_over;
            if (x > 0.) {
                approx[u] += x;
                wimpy[u] += x * x;
                topk->put(u, approx[u]);
                if (!firstpass) {
                    int64_t *m = &mcrade[(uint64_t)u * T];
                    for (int j = 0; j < T; j++) m[j] = (int64_t)((double)m[j] + sig[j] * x);
                }
                if (firstpass && !absolute) {
                    if (approx_toadd[u] == 0 && approx[u] >= 3) {
                        distinct++;
                        approx_toadd[u] = 1;
                    }
                }
                if (approx[u] > sup_bcest) sup_bcest = approx[u];
                if (wimpy[u] > sup_wv) sup_wv = wimpy[u];
            }
        }
        sp_lengths[s.path_length] += 1;
    }

    // silvan/src/Probabilistic.cpp:712-726
    double ub_top1(double est, double delta) {
        double lt = log(1. / delta);
        double c = lt / (double)num_samples;
        double ub = est + c + sqrt(2 * c * est + pow(c, 2.));
        return fmin(ub, 1.0);
    }

    // silvan/src/Probabilistic.cpp:729-766
    double ub_avg_diam(double delta) {
        double avg = 0.;
        int Di = (int)D;
        for (int i = 0; i <= Di; i++) avg += (double)i * sp_lengths[i] / (double)(num_samples);
        double lt = log(1. / delta);
        double c = (Di - 2) * lt / (double)num_samples;
        double ub_b = avg + c + sqrt(2 * c * avg + pow(c, 2.));
        double var = 0.;
        for (int i = 0; i <= Di; i++)
            for (int j = i + 1; j <= Di; j++)
                var += pow(i - j, 2.0) * sp_lengths[i] / (double)num_samples * sp_lengths[j] /
                       (double)(num_samples - 1);
        lt = log(2. / delta);
        double ub_eb = avg + 7. / 3. * (Di - 2) * lt / (double)num_samples +
                       sqrt(2 * var * lt / (double)num_samples);
        double ub = fmin(ub_b, ub_eb);
        ub = fmin(ub, (double)(Di - 2));
        return ub;
    }

    // silvan/src/Probabilistic.cpp:80-85
    static double nsb(double x, double rho, double d, double e) {
        double vx = x * (1. - x);
        double ah = e / vx;
        double den = vx * ((1 + ah) * log(1 + ah) - ah);
        return log(2 * rho / (x * d)) / (den);
    }

    // silvan/src/Probabilistic.cpp:87-174
    static double ub_samples(double max_bc, double max_var, double avg_spl, double eps,
                             double db) {
        double xh = 0., lo = fmax(0.5 - sqrt(eps / 3.), 0.), hi = 0.5;
        while (hi - lo > 0.0001) {
            xh = (hi + lo) / 2.;
            double vx = xh * (1. - xh);
            double ah = eps / vx;
            double f = vx * ((1 + ah) * log(1 + ah) - ah);
            if (f <= 2 * pow(eps, 2)) hi = xh;
            else lo = xh;
        }
        xh = hi;
        double xhigh = fmin(xh, max_bc);
        if (max_var < 0.25) {
            double xv = 0.5 - sqrt(0.25 - max_var);
            xhigh = fmin(xhigh, xv);
        }
        double step = xhigh / 1000.;
        double bh = nsb(xhigh, avg_spl, db, eps);
        double b = bh + 1;
        while (b >= bh) {
            double xl = xhigh - step;
            if (xl > 0.) {
                b = nsb(xl, avg_spl, db, eps);
                if (b > bh) {
                    xhigh = xl;
                    bh = b;
                }
            } else {
                b = bh - 1;
            }
        }
        return bh;
    }

    // silvan/src/Probabilistic.cpp:689-708
    double eps_mcrade(double sw, double mc, double d, double m, double nn) {
        mc = fmax(mc, 0.);
        double lt = log(5. / d) / m;
        double var_ub = sw + lt + sqrt(pow(lt, 2.) + 2 * lt * sw);
        var_ub = fmin(var_ub, 0.25);
        double era = mc + sqrt(4 * sw * lt / (double)T);
        double ra = era + lt + sqrt(pow(lt, 2.) + 2 * lt * era);
        if (nn == 1) ra = 0;
        double e = 2 * ra + sqrt(2 * lt * (var_ub + 4 * ra)) + lt / 3;
        double e2 = 2 * ra + sqrt(lt / 2.);
        e = fmin(e, e2);
        if (nn >= 1) {
            double eu = sqrt(2 * var_ub * log(5. / d * nn) / m) + log(5. / d * nn) / m / 3;
            e = fmin(e, eu);
        }
        return e;
    }

    // silvan/src/Probabilistic.cpp:179-245
    double rel_bound(double bc, double delta, double rho, double m, bool upper) {
        double up = 1.0, lo = 0.;
        if (upper) lo = bc;
        else up = bc;
        for (int i = 0; i < 30; i++) {
            double t = (up + lo) / 2.;
            double vt = t * (1. - t);
            double ltm = log(2. / delta * fmin((double)g.n, rho / t)) / m;
            double st = sqrt(2. * ltm * vt);
            if (upper) {
                double qc = bc + ltm / 3. + st;
                if (qc >= t) lo = t;
                else up = t;
            } else {
                double qc = bc - ltm / 3. - st;
                if (qc <= t) up = t;
                else lo = t;
            }
        }
        return upper ? up : lo;
    }

    // silvan/src/Probabilistic.cpp:587-687
    bool check_topk() {
        double ms = (double)num_samples;
        double dpb = p.delta / pow(2., iteration);
        eps_final_topk = 1.0;
        double lb_topk = 0.0, ub_topk = 1.0;
        Ranking sub(k), slb(k);
        uint32_t ins = 0;
        bool rel = true;
        for (uint64_t i = 0; i < union_sample && rel; i++) {
            uint32_t node = topk->el[i];
            double an = topk->val[i] / ms;
            double ec = eps_part[part_map[part[node]]];
            double lbb = an - ec, ubb = an + ec;
            double adu = ub_avg_diam(dpb);
            double lbr = rel_bound(an, dpb, adu, ms, false);
            double ubr = rel_bound(an, dpb, adu, ms, true);
            lbb = fmax(lbb, lbr);
            ubb = fmin(ubb, ubr);
            sub.put(node, ubb);
            slb.put(node, lbb);
            ins++;
            if (ins >= k) {
                ub_topk = fmin(ub_topk, sub.val[k - 1]);
                lb_topk = fmax(lb_topk, slb.val[k - 1]);
            }
            if (ubb > lb_topk) {
                eps_final_topk = fmin(eps_final_topk, ec);
                bool lc = lbb >= an / (1. + p.eps);
                bool uc = ubb <= an / (1. - p.eps);
                rel = rel && lc && uc;
            } else {
                eps_final_topk = fmin(eps_final_topk, lb_topk - an);
            }
        }
        if (rel) {
            uint32_t cnt = 0;
            for (uint32_t i = 0; i < ins; i++) {
                uint32_t node = topk->el[i];
                double an = topk->val[i] / ms;
                double ec = eps_part[part_map[part[node]]];
                if (an + ec > lb_topk) cnt++;
            }
            numresults_topk = cnt;
        }
        return rel;
    }

    // silvan/src/Probabilistic.cpp:251-414
    bool check(uint64_t status_n_pairs, uint32_t status_top0) {
        checks++;
        double ms = (double)num_samples;
        double dpb = 1.0;
        if (absolute && p.mhat) dpb = dfpb;
        else dpb = p.delta / pow(2., iteration);
        if (absolute) {  // second phase has started
            double adu = ub_avg_diam(dpb);
            double t1 = approx[status_top0] / ms;
            double t1u = ub_top1(t1, dpb);
            double wvu = ub_top1(sup_wv / ms, dpb);
            if (p.mhat) {
                uint64_t mns = (uint64_t)ub_samples(t1u, wvu, adu, p.eps, dpb);
                if (last_stop > (double)mns) {
                    last_stop = (double)mns;
                    omega = last_stop;
                    double mni = log((double)mns / (double)first_stop) / log(1.2) + 1;
                    dfpb = p.delta / (floor(mni));
                }
            }
        }
        std::vector<int> cnt(nparts, 0);
        std::vector<double> swp(nparts, 0.0);
        std::vector<int64_t> mx((size_t)nparts * T, -(int64_t)status_n_pairs);
        for (uint32_t v = 0; v < g.n; v++) {
            int pi = part_map[part[v]];
            swp[pi] = fmax(swp[pi], wimpy[v]);
            cnt[pi]++;
            for (int j = 0; j < T; j++)
                mx[(size_t)pi * T + j] = std::max(mx[(size_t)pi * T + j], mcrade[(uint64_t)v * T + j]);
        }
        eps_part.assign(nparts, 1.0);
        for (int i = 0; i < nparts; i++) {
            double avg = 0.0;
            for (int j = 0; j < T; j++) avg += mx[(size_t)i * T + j] / (double)T;
            avg = avg / ms;
            double sw = swp[i] / ms;
            double dp = dpb / nparts;
            eps_part[i] = eps_mcrade(sw, avg, dp, ms, cnt[i]);
        }
        if (absolute) {
            double sup = 0;
            for (int i = 0; i < nparts; i++) sup = fmax(sup, eps_part[i]);
            if (sup <= p.eps) eps_stop = sup;
            return sup <= p.eps;
        }
        return check_topk();
    }

    // silvan/src/Probabilistic.cpp:775-1139, one thread
    void run(Result &res) {
        const uint32_t n = g.n;
        absolute = (p.k == 0);
        alpha = p.alpha;
        approx.assign(n, 0);
        approx_toadd.assign(n, 0);
        wimpy.assign(n, 0);
        mcrade.assign((uint64_t)n * T, 0);
        part.assign(n, 0);
        uint32_t tau = (uint32_t)fmax(1. / p.eps * (log(1. / p.delta)), 1000.);
        tau = (uint32_t)fmax((double)tau, 2 * (int)D * (log(1. / p.delta)));
        res.tau = tau;
        double a = p.a;
        bool peel = a > 1;
        if (!peel) a = 100 * tau;
        union_sample = std::min(n, (uint32_t)fmax(2 * sqrt((double)g.m) / p.threads, p.k + 20.));
        k = std::min(p.k, n);
        sp_lengths.assign((size_t)D + 1, 0);
        topk = new Ranking(union_sample);
        firstpass = true;
        bool stop1 = false;
        while (!stop1) {
            for (int i = 0; i <= 10; i++) one_round();
            if (absolute) stop1 = n_pairs >= tau;
            else stop1 = distinct >= 1.5 * p.k && n_pairs >= tau;
        }
        res.first_pass_samples = num_samples;
        // empirical peeling (:853-871)
        std::map<int, int> ne;
        for (uint32_t i = 0; i < n; i++) {
            double ew = wimpy[i] / (double)num_samples;
            double mi = fmin(1. / ew, (double)num_samples);
            int idx = (int)(log(mi) / log(a) + 1);
            if (!peel) idx = 0;
            part[i] = idx;
            ne[idx] = ne[idx] + 1;
        }
        nparts = (int)ne.size();
        int pidx = 0;
        for (auto &e : ne) part_map[e.first] = pidx++;
        firstpass = false;
        double mns = 0.;
        if (absolute) {  // (:906-942)
            double adu = ub_avg_diam(p.delta / 8.);
            std::fill(sp_lengths.begin(), sp_lengths.end(), 0);
            double t1u = ub_top1(sup_bcest / (double)num_samples, p.delta / 8.);
            double wvu = ub_top1(sup_wv / (double)num_samples, p.delta / 8.);
            if (!p.alpha_given && wvu > 0.9 * t1u) alpha = -1.;
            if (p.mhat) mns = ub_samples(t1u, wvu, adu, p.eps, p.delta / 2.);
        }
        iteration = 1;
        n_pairs = 0;
        double kth = 1.0;
        if (!absolute) {
            kth = topk->val[p.k] / (double)num_samples + 1.0 / (double)num_samples;
        }
        delete topk;
        topk = new Ranking(union_sample);
        std::fill(approx.begin(), approx.end(), 0);
        std::fill(approx_toadd.begin(), approx_toadd.end(), 0);
        std::fill(wimpy.begin(), wimpy.end(), 0);
        std::fill(mcrade.begin(), mcrade.end(), 0);
        sup_bcest = 0;
        omega = pow(10., 15);
        if (mns > 0.) omega = mns;
        // first sample size by bisection (:973-1025)
        double lo = 1. / p.eps * log(2. / p.delta), hi = omega;
        double svn = sup_wv / (double)num_samples + 1 / (double)num_samples;
        while (hi - lo > 10) {
            num_samples = (uint64_t)((hi + lo) / 2.);
            double eg;
            if (absolute)
                eg = sqrt(2 * svn * log(2. / p.delta) / (double)num_samples) +
                     log(2. / p.delta) / (double)num_samples / 3.;
            else
                eg = sqrt(2 * kth * log(2. / p.delta / kth) / (double)num_samples) +
                     log(2. / p.delta / kth) / (double)num_samples / 3.;
            if (absolute) {
                if (eg > p.eps) lo = (double)num_samples;
                else hi = (double)num_samples;
            } else {
                bool v1 = kth + eg > kth / (1. - p.eps);
                bool v2 = kth - eg < kth / (1. + p.eps);
                bool v3 = eg >= kth * p.eps * pow((1 - p.eps) / (1 + p.eps), 2.);
                if (v1 || v2 || v3) lo = (double)num_samples;
                else hi = (double)num_samples;
            }
        }
        first_stop = (double)num_samples;
        num_samples = 0;
        sup_wv = 0;
        if (p.mhat) {
            double mni = log((double)mns / (double)first_stop) / log(1.2) + 1;
            dfpb = p.delta / (floor(mni));
        }
        last_stop = omega;
        if (first_stop >= last_stop / 4) first_stop = last_stop / 4;
        next_stop = (uint64_t)first_stop;
        bool stop = false;
        int reason = 0;
        while (!stop) {  // (:1060-1101)
            for (int i = 0; i <= 10; i++) one_round();
            if (p.mhat && (double)num_samples >= omega) {
                stop = true;
                reason = 2;
            }
            if (!stop && (double)num_samples < last_stop && num_samples >= next_stop) {
                stop = check(n_pairs, topk->el[0]);
                if (stop) reason = 1;
                else {
                    next_stop = (uint64_t)(next_stop * 1.2);
                    iteration += 1;
                }
            }
        }
        res.graph_diameter = D;
        res.num_samples = num_samples;
        res.vis_edges = vis_edges;
        res.iteration_index = iteration;
        res.num_partitions = nparts;
        res.omega = omega;
        res.first_stopping_samples = first_stop;
        res.last_stopping_samples = last_stop;
        res.alpha_sp_sampling = alpha;
        res.sup_bcest = sup_bcest;
        res.sup_emp_wimpy_var = sup_wv;
        res.eps_final_topk = eps_final_topk;
        res.eps_stop = eps_stop;
        res.numresults_topk = numresults_topk;
        res.union_sample = union_sample;
        res.stop_reason = reason;
        res.zero_modulus = zero_mod ? 1 : 0;
        res.checks = checks;
    }
};

Run *g_run = nullptr;

}  // namespace

extern "C" {

void *orc_graph_new(uint32_t n, int directed, const uint64_t *out_off, const uint32_t *out_adj,
                    const uint64_t *in_off, const uint32_t *in_adj, const uint32_t *cc) {
    OGraph *g = new OGraph();
    g->n = n;
    g->directed = directed != 0;
    g->out_off.assign(out_off, out_off + n + 1);
    g->out_adj.assign(out_adj, out_adj + out_off[n]);
    g->m = out_off[n];
    if (g->directed) {
        g->in_off.assign(in_off, in_off + n + 1);
        g->in_adj.assign(in_adj, in_adj + in_off[n]);
    }
    g->cc.assign(cc, cc + n);
    return g;
}

void orc_graph_free(void *g) { delete (OGraph *)g; }

// Exact betweenness (Brandes, "A faster algorithm for betweenness
// centrality", J. Math. Sociol. 2001) normalised the way SILVAN estimates it:
// the sum over ordered pairs (s, t), s != t, of sigma_st(v) / sigma_st,
// divided by n (n - 1).  Path counts are doubles.  The reference has no exact
// algorithm of its own; this is the ground truth of the (eps, delta) check.
void orc_brandes(void *gp, double *bc) {
    const OGraph &g = *(const OGraph *)gp;
    const uint32_t n = g.n;
    std::vector<double> acc(n, 0.0);
#pragma omp parallel
    {
        std::vector<double> local(n, 0.0), sigma(n), delta(n);
        std::vector<int64_t> dist(n);
        std::vector<uint32_t> order;
        order.reserve(n);
#pragma omp for schedule(dynamic, 16)
        for (int64_t s = 0; s < (int64_t)n; s++) {
            std::fill(sigma.begin(), sigma.end(), 0.0);
            std::fill(delta.begin(), delta.end(), 0.0);
            std::fill(dist.begin(), dist.end(), -1);
            order.clear();
            sigma[s] = 1.0;
            dist[s] = 0;
            order.push_back((uint32_t)s);
            for (size_t h = 0; h < order.size(); h++) {
                const uint32_t x = order[h];
                for (uint64_t e = g.out_off[x]; e < g.out_off[x + 1]; e++) {
                    const uint32_t y = g.out_adj[e];
                    if (dist[y] < 0) {
                        dist[y] = dist[x] + 1;
                        order.push_back(y);
                    }
                    if (dist[y] == dist[x] + 1) sigma[y] += sigma[x];
                }
            }
            for (size_t h = order.size(); h-- > 1;) {
                const uint32_t y = order[h];
                for (uint64_t e = g.ioff()[y]; e < g.ioff()[y + 1]; e++) {
                    const uint32_t x = g.iadj()[e];
                    if (dist[x] >= 0 && dist[x] + 1 == dist[y])
                        delta[x] += sigma[x] / sigma[y] * (1.0 + delta[y]);
                }
                local[y] += delta[y];
            }
        }
#pragma omp critical
        for (uint32_t v = 0; v < n; v++) acc[v] += local[v];
    }
    const double norm = (double)n * (double)(n - 1);
    for (uint32_t v = 0; v < n; v++) bc[v] = acc[v] / norm;
}

// Per-sample replay of samples [first, first+count).  Entries are the
// (node, count) pairs of each sample in ascending node order.  Returns the
// number of entries, -1 if ent_cap is too small, -2 on a zero modulus.
int64_t orc_replay(void *gp, uint64_t seed, uint32_t first, uint32_t count, double alpha,
                   int32_t *pl, int32_t *np, uint64_t *vis, uint32_t *nent, uint32_t *ent_node,
                   int32_t *ent_cnt, uint64_t ent_cap) {
    const OGraph &g = *(OGraph *)gp;
    Scratch s(g.n);
    uint64_t e = 0;
    bool zm = false;
    for (uint32_t i = 0; i < count; i++) {
        SampleOut o;
        sample_one(g, s, seed, first + i, alpha, o);
        zm = zm || o.zero_mod;
        pl[i] = o.path_length;
        np[i] = o.num_paths;
        vis[i] = o.vis_edges;
        nent[i] = (uint32_t)o.nodes.size();
        for (auto &kv : o.nodes) {
            if (e >= ent_cap) return -1;
            ent_node[e] = kv.first;
            ent_cnt[e] = kv.second;
            e++;
        }
    }
    return zm ? -2 : (int64_t)e;
}

// Full estimator run in parity mode.  res must point to an OrcResult
// (layout of `Result` above).
int orc_run(void *gp, uint32_t diameter, double eps, double delta, uint32_t k, double alpha,
            int alpha_given, double a, int mhat, uint64_t seed, uint32_t threads, int weighted,
            void *res) {
    delete g_run;
    Params p{eps, delta, k, alpha, alpha_given, a, mhat, seed, threads ? threads : 1, weighted};
    g_run = new Run(*(OGraph *)gp, p, diameter);
    g_run->run(*(Result *)res);
    return 0;
}

uint64_t orc_result_size() { return sizeof(Result); }

void orc_run_arrays(double *approx, double *wimpy, int64_t *mcrade, int32_t *partition_index) {
    Run *r = g_run;
    uint32_t n = r->g.n;
    std::memcpy(approx, r->approx.data(), sizeof(double) * n);
    std::memcpy(wimpy, r->wimpy.data(), sizeof(double) * n);
    std::memcpy(mcrade, r->mcrade.data(), sizeof(int64_t) * (uint64_t)n * 25);
    std::memcpy(partition_index, r->part.data(), sizeof(int32_t) * n);
}

void orc_run_ranking(uint32_t *elements, double *values) {
    Run *r = g_run;
    for (uint32_t i = 0; i < r->union_sample; i++) {
        elements[i] = r->topk->el[i];
        values[i] = r->topk->val[i];
    }
}

void orc_run_sp_lengths(uint64_t *out) {
    Run *r = g_run;
    for (size_t i = 0; i < r->sp_lengths.size(); i++) out[i] = r->sp_lengths[i];
}

void orc_run_partitions(double *eps, int32_t *ids) {
    Run *r = g_run;
    for (int i = 0; i < r->nparts; i++) eps[i] = i < (int)r->eps_part.size() ? r->eps_part[i] : 1.0;
    int j = 0;
    for (auto &kv : r->part_map) ids[j++] = kv.first;
}

void orc_run_free() {
    delete g_run;
    g_run = nullptr;
}

}  // extern "C"

extern "C" {
// Philox4x32-10 block (for known-answer tests of the oracle stream).
void orc_philox4x32(const uint32_t *ctr, const uint32_t *key, uint32_t *out) {
    oracle_philox4x32_10(ctr, key, out);
}
}
