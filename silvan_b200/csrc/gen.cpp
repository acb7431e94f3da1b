// Seeded synthetic graph generators for the workloads this library is
// measured on (the paper's SNAP/KONECT datasets are not available offline):
// Barabasi-Albert, Erdos-Renyi G(n, M), R-MAT and a perturbed 4-neighbour
// grid.  Labels are consecutive integers.  Every generator is a plain
// function of its arguments and seed.  Undirected graphs are emitted with
// each edge once; the edge-list loader adds the reverse direction exactly
// like the reference loader does (silvan/src/Graph.cpp:53-55).
#include "gen.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <unordered_set>
#include <vector>

namespace {

// splitmix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) seeds a xoshiro256** state (Blackman, Vigna 2018).
struct Rng {
    uint64_t s[4];
    static uint64_t splitmix(uint64_t &x) {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (int i = 0; i < 4; i++) s[i] = splitmix(x);
    }
    static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    // uniform in [0, m) by 128-bit multiply (Lemire); the tiny bias is
    // irrelevant for workload generation.
    uint64_t below(uint64_t m) { return (uint64_t)(((__uint128_t)next() * m) >> 64); }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

inline uint64_t key(uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | b; }

}  // namespace

namespace silvan {

std::vector<std::pair<uint32_t, uint32_t>> gen_ba(uint32_t n, uint32_t m, uint64_t seed) {
    std::vector<std::pair<uint32_t, uint32_t>> e;
    if (n <= m || m == 0) return e;
    Rng rng(seed);
    std::vector<uint32_t> rep;
    rep.reserve((size_t)2 * n * m);
    // initial star on m+1 nodes, centre 0
    for (uint32_t i = 1; i <= m; i++) {
        e.emplace_back(0u, i);
        rep.push_back(0u);
        rep.push_back(i);
    }
    std::vector<uint32_t> tg(m);
    for (uint32_t src = m + 1; src < n; src++) {
        uint32_t got = 0;
        while (got < m) {
            uint32_t t = rep[rng.below(rep.size())];
            bool dup = false;
            for (uint32_t q = 0; q < got; q++)
                if (tg[q] == t) dup = true;
            if (!dup) tg[got++] = t;
        }
        for (uint32_t q = 0; q < m; q++) {
            e.emplace_back(src, tg[q]);
            rep.push_back(tg[q]);
            rep.push_back(src);
        }
    }
    return e;
}

std::vector<std::pair<uint32_t, uint32_t>> gen_er(uint32_t n, double mean_degree, uint64_t seed) {
    std::vector<std::pair<uint32_t, uint32_t>> e;
    if (n < 2) return e;
    Rng rng(seed);
    uint64_t M = (uint64_t)(mean_degree * n / 2.0 + 0.5);
    uint64_t maxm = (uint64_t)n * (n - 1) / 2;
    if (M > maxm) M = maxm;
    std::unordered_set<uint64_t> seen;
    seen.reserve(M * 2);
    e.reserve(M);
    while (e.size() < M) {
        uint32_t a = (uint32_t)rng.below(n), b = (uint32_t)rng.below(n);
        if (a == b) continue;
        uint32_t lo = std::min(a, b), hi = std::max(a, b);
        if (seen.insert(key(lo, hi)).second) e.emplace_back(a, b);
    }
    return e;
}

std::vector<std::pair<uint32_t, uint32_t>> gen_rmat(uint32_t scale, uint32_t edge_factor, double a,
                                                    double b, double c, uint64_t seed,
                                                    bool directed) {
    std::vector<std::pair<uint32_t, uint32_t>> e;
    Rng rng(seed);
    uint64_t draws = (uint64_t)edge_factor << scale;
    std::vector<uint64_t> keys;
    keys.reserve(draws);
    const double ab = a + b, abc = a + b + c;
    for (uint64_t i = 0; i < draws; i++) {
        uint32_t u = 0, v = 0;
        for (uint32_t l = 0; l < scale; l++) {
            double r = rng.unit();
            uint32_t bu = 0, bv = 0;
            if (r < a) {
            } else if (r < ab) {
                bv = 1;
            } else if (r < abc) {
                bu = 1;
            } else {
                bu = 1;
                bv = 1;
            }
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        if (u == v) continue;  // self-loops removed
        if (!directed && u > v) std::swap(u, v);
        keys.push_back(key(u, v));
    }
    // duplicates removed (the list comes out sorted; the loader sorts anyway)
    std::vector<uint64_t> sorted = keys;
    std::sort(sorted.begin(), sorted.end());
    sorted.erase(std::unique(sorted.begin(), sorted.end()), sorted.end());
    e.reserve(sorted.size());
    for (uint64_t k : sorted) e.emplace_back((uint32_t)(k >> 32), (uint32_t)k);
    return e;
}

std::vector<std::pair<uint32_t, uint32_t>> gen_grid(uint32_t side, double delete_frac,
                                                    double shortcut_frac, uint64_t seed) {
    std::vector<std::pair<uint32_t, uint32_t>> base;
    Rng rng(seed);
    uint64_t nn = (uint64_t)side * side;
    base.reserve((size_t)2 * nn);
    for (uint32_t r = 0; r < side; r++)
        for (uint32_t c = 0; c < side; c++) {
            uint32_t id = r * side + c;
            if (c + 1 < side) base.emplace_back(id, id + 1);
            if (r + 1 < side) base.emplace_back(id, id + side);
        }
    uint64_t E = base.size();
    uint64_t ndel = (uint64_t)(delete_frac * (double)E + 0.5);
    // partial Fisher-Yates: the first ndel slots are the deleted edges
    for (uint64_t i = 0; i < ndel && i < E; i++) {
        uint64_t j = i + rng.below(E - i);
        std::swap(base[i], base[j]);
    }
    std::vector<std::pair<uint32_t, uint32_t>> e(base.begin() + std::min(ndel, E), base.end());
    std::sort(e.begin(), e.end());
    std::unordered_set<uint64_t> seen;
    seen.reserve(e.size() * 2);
    for (auto &p : e) seen.insert(key(p.first, p.second));
    uint64_t nsc = (uint64_t)(shortcut_frac * (double)E + 0.5);
    uint64_t added = 0;
    while (added < nsc) {
        uint32_t a = (uint32_t)rng.below(nn), b = (uint32_t)rng.below(nn);
        if (a == b) continue;
        uint32_t lo = std::min(a, b), hi = std::max(a, b);
        if (!seen.insert(key(lo, hi)).second) continue;
        e.emplace_back(lo, hi);
        added++;
    }
    return e;
}

bool write_edge_list(const char *path, const std::vector<std::pair<uint32_t, uint32_t>> &e) {
    FILE *f = std::fopen(path, "wb");
    if (!f) return false;
    std::vector<char> buf;
    buf.reserve(1 << 22);
    char tmp[32];
    for (auto &p : e) {
        int l = std::snprintf(tmp, sizeof tmp, "%u %u\n", p.first, p.second);
        buf.insert(buf.end(), tmp, tmp + l);
        if (buf.size() > (1u << 22)) {
            std::fwrite(buf.data(), 1, buf.size(), f);
            buf.clear();
        }
    }
    std::fwrite(buf.data(), 1, buf.size(), f);
    return std::fclose(f) == 0;
}

}  // namespace silvan
