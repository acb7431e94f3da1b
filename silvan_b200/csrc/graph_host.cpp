// Host side of the graph store (see graph_host.h).
#include "graph_host.h"

#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <deque>

#include "silvan.h"

namespace silvan {

namespace {

inline bool c_isspace(unsigned char ch) {
    return ch == ' ' || ch == '\t' || ch == '\n' || ch == '\v' || ch == '\f' || ch == '\r';
}

// One "%u" conversion of sscanf in the C locale, restricted to what the
// reference can represent: optional '+', decimal digits, value <= kMaxNodeId.
// Returns 1 on a conversion, 0 on a matching failure (nothing stored),
// -1 on a value the reference cannot hold (a '-' sign or an id > kMaxNodeId).
int scan_u(const char *&p, const char *end, uint32_t &out) {
    while (p < end && c_isspace((unsigned char)*p)) p++;
    const char *q = p;
    bool neg = false;
    if (q < end && (*q == '+' || *q == '-')) {
        neg = (*q == '-');
        q++;
    }
    if (q >= end || *q < '0' || *q > '9') return 0;
    uint64_t v = 0;
    bool big = false;
    while (q < end && *q >= '0' && *q <= '9') {
        v = v * 10 + (uint64_t)(*q - '0');
        if (v > kMaxNodeId) big = true;
        if (v > (1ull << 40)) v = (1ull << 40);  // stays "big", no wrap
        q++;
    }
    p = q;
    if (neg || big) return -1;
    out = (uint32_t)v;
    return 1;
}

void sort_unique(std::vector<uint64_t> &keys) {
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
}

void keys_to_csr(const std::vector<uint64_t> &keys, uint32_t n, std::vector<uint64_t> &off,
                 std::vector<uint32_t> &adj) {
    off.assign((size_t)n + 1, 0);
    adj.resize(keys.size());
    for (uint64_t k : keys) off[(k >> 32) + 1]++;
    for (uint32_t i = 0; i < n; i++) off[i + 1] += off[i];
    for (size_t i = 0; i < keys.size(); i++) adj[i] = (uint32_t)keys[i];
}

}  // namespace

void build_csr(const std::vector<std::pair<uint32_t, uint32_t>> &pairs, bool directed,
               HostGraph &g) {
    uint32_t n = 0;
    for (auto &p : pairs) n = std::max(n, std::max(p.first, p.second) + 1);
    g.n = n;
    g.directed = directed;
    std::vector<uint64_t> keys;
    keys.reserve(pairs.size() * (directed ? 1 : 2));
    for (auto &p : pairs) {
        keys.push_back(((uint64_t)p.first << 32) | p.second);
        if (!directed) keys.push_back(((uint64_t)p.second << 32) | p.first);
    }
    sort_unique(keys);
    keys_to_csr(keys, n, g.out_off, g.out_adj);
    g.in_off.clear();
    g.in_adj.clear();
    if (directed) {
        keys.clear();
        for (auto &p : pairs) keys.push_back(((uint64_t)p.second << 32) | p.first);
        sort_unique(keys);
        keys_to_csr(keys, n, g.in_off, g.in_adj);
    }
}

int load_edge_list(const char *path, bool directed, HostGraph &g, std::string &err) {
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        err = std::string("cannot open graph file: ") + path;
        return SILVAN_E_IO;
    }
    std::vector<char> data;
    {
        char buf[1 << 16];
        size_t r;
        while ((r = std::fread(buf, 1, sizeof buf, f)) > 0) data.insert(data.end(), buf, buf + r);
        std::fclose(f);
    }
    std::vector<std::pair<uint32_t, uint32_t>> pairs;
    pairs.reserve(data.size() / 8 + 1);
    uint32_t u = 0, v = 0;  // silvan/src/Graph.cpp:42: kept across lines
    const char *p = data.data(), *end = data.data() + data.size();
    uint64_t lineno = 0;
    while (p < end) {
        const char *eol = (const char *)std::memchr(p, '\n', (size_t)(end - p));
        const char *lend = eol ? eol : end;
        lineno++;
        if (lend == p || *p != '#') {
            const char *q = p;
            int r = scan_u(q, lend, u);
            if (r == 1) {
                while (q < lend && c_isspace((unsigned char)*q)) q++;
                r = scan_u(q, lend, v);
            }
            if (r < 0) {
                err = "graph file line " + std::to_string(lineno) +
                      ": node id is negative or larger than " + std::to_string(kMaxNodeId);
                return SILVAN_E_PARSE;
            }
            pairs.emplace_back(u, v);
        }
        p = eol ? eol + 1 : end;
    }
    build_csr(pairs, directed, g);
    return SILVAN_OK;
}

uint32_t compute_scc(const HostGraph &g, std::vector<uint32_t> &cc) {
    // Iterative Tarjan with the visiting order of silvan/src/Graph.cpp:125-191:
    // roots ascending; on first visit every unvisited neighbour is pushed on
    // the DFS stack in row order (the last pushed is explored first); an
    // on-stack neighbour lowers the node's lowlink with its lowlink; when a
    // node is popped the second time its lowlink is passed to its DFS parent
    // and, if it is a root, its component is numbered.
    const uint32_t n = g.n;
    cc.assign(n, 0);
    std::vector<uint32_t> index(n), low(n), parent(n), scc_stack;
    std::vector<uint32_t> dfs;
    std::vector<uint8_t> state(n, 0), onstack(n, 0);
    scc_stack.reserve(n);
    dfs.reserve(g.num_edges() + 1);
    uint32_t counter = 0, ncomp = 0;
    for (uint32_t root = 0; root < n; root++) {
        if (state[root] != 0) continue;
        dfs.clear();
        dfs.push_back(root);
        parent[root] = root;
        while (!dfs.empty()) {
            uint32_t x = dfs.back();
            if (state[x] == 0) {
                state[x] = 1;
                index[x] = low[x] = counter++;
                scc_stack.push_back(x);
                onstack[x] = 1;
                for (uint64_t e = g.out_off[x]; e < g.out_off[x + 1]; e++) {
                    uint32_t w = g.out_adj[e];
                    if (state[w] == 0) {
                        parent[w] = x;
                        dfs.push_back(w);
                    } else if (onstack[w]) {
                        low[x] = std::min(low[x], low[w]);
                    }
                }
            } else {
                dfs.pop_back();
                if (state[x] == 1) {
                    uint32_t px = parent[x];
                    low[px] = std::min(low[px], low[x]);
                    if (low[x] == index[x]) {
                        uint32_t w;
                        do {
                            w = scc_stack.back();
                            scc_stack.pop_back();
                            onstack[w] = 0;
                            cc[w] = ncomp;
                        } while (w != x);
                        ncomp++;
                    }
                    state[x] = 2;
                }
            }
        }
    }
    return ncomp;
}

uint32_t estimate_diameter(const HostGraph &g, const std::vector<uint32_t> &cc, uint32_t ncomp) {
    const uint32_t n = g.n;
    // pivot: largest out+in degree, first index on ties (Graph.cpp:205-215)
    std::vector<uint32_t> pivot(ncomp, UINT32_MAX);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t &p = pivot[cc[i]];
        if (p == UINT32_MAX ||
            g.out_degree(i) + g.in_degree(i) > g.out_degree(p) + g.in_degree(p))
            p = i;
    }
    // eccentricity of each pivot inside its component, forward and backward
    // (Graph.cpp:237-268); the distance arrays are shared across components
    // because every BFS stays inside its own component.
    std::vector<int32_t> dist_f(n, -1), dist_b(n, -1);
    std::vector<uint32_t> q(n);
    auto ecc = [&](uint32_t start, bool backward, std::vector<int32_t> &dist) -> uint32_t {
        const uint64_t *off = backward ? g.in_offsets() : g.out_off.data();
        const uint32_t *adj = backward ? g.in_neighbours() : g.out_adj.data();
        uint32_t head = 0, tail = 0;
        q[tail++] = start;
        dist[start] = 0;
        while (head < tail) {
            uint32_t x = q[head++];
            for (uint64_t e = off[x]; e < off[x + 1]; e++) {
                uint32_t y = adj[e];
                if (dist[y] == -1 && cc[y] == cc[x]) {
                    dist[y] = dist[x] + 1;
                    q[tail++] = y;
                }
            }
        }
        return (uint32_t)dist[q[tail - 1]];
    };
    std::vector<uint32_t> ecc_f(ncomp), ecc_b(ncomp);
    for (uint32_t c = 0; c < ncomp; c++) {
        ecc_f[c] = ecc(pivot[c], false, dist_f);
        ecc_b[c] = ecc(pivot[c], true, dist_b);
    }
    return diameter_recursion(g, cc, ncomp, ecc_f, ecc_b);
}

uint32_t diameter_recursion(const HostGraph &g, const std::vector<uint32_t> &cc, uint32_t ncomp,
                            const std::vector<uint32_t> &ecc_f, const std::vector<uint32_t> &ecc_b) {
    const uint32_t n = g.n;
    std::vector<uint32_t> ecc_fp(ncomp);
    // Components complete in reverse topological order, so every edge between
    // components goes to a smaller id and the DP below (Graph.cpp:298-306) can
    // run in ascending id order over the edges of each component.
    std::vector<uint64_t> start(ncomp + 1, 0);
    for (uint32_t i = 0; i < n; i++) start[cc[i] + 1]++;
    for (uint32_t c = 0; c < ncomp; c++) start[c + 1] += start[c];
    std::vector<uint32_t> members(n);
    {
        std::vector<uint64_t> cur(start.begin(), start.end() - 1);
        for (uint32_t i = 0; i < n; i++) members[cur[cc[i]]++] = i;
    }
    uint32_t diam = 0;
    for (uint32_t c = 0; c < ncomp; c++) {
        uint32_t best = ecc_f[c];
        for (uint64_t k = start[c]; k < start[c + 1]; k++) {
            uint32_t x = members[k];
            for (uint64_t e = g.out_off[x]; e < g.out_off[x + 1]; e++) {
                uint32_t d = cc[g.out_adj[e]];
                if (d != c) best = std::max(best, ecc_f[c] + 1 + ecc_b[d] + ecc_fp[d]);
            }
        }
        ecc_fp[c] = best;
        diam = std::max(diam, ecc_fp[c] + ecc_b[c]);
    }
    return diam;
}

}  // namespace silvan
