// Seeded synthetic graph generators (see gen.cpp).
#pragma once
#include <cstdint>
#include <utility>
#include <vector>

namespace silvan {

using EdgeList = std::vector<std::pair<uint32_t, uint32_t>>;

// Barabasi-Albert: star on m+1 nodes, then each new node attaches to m
// distinct existing nodes chosen proportionally to degree.  Undirected.
EdgeList gen_ba(uint32_t n, uint32_t m, uint64_t seed);
// Erdos-Renyi G(n, M) with M = round(n * mean_degree / 2) distinct edges,
// no self-loops.  Undirected.
EdgeList gen_er(uint32_t n, double mean_degree, uint64_t seed);
// R-MAT with 2^scale ids and edge_factor * 2^scale draws of quadrant
// probabilities (a, b, c, 1-a-b-c); self-loops and duplicates removed.
EdgeList gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                  uint64_t seed, bool directed);
// side x side 4-neighbour grid; delete_frac of its edges removed uniformly at
// random, then shortcut_frac * (grid edges) random long-range edges added.
EdgeList gen_grid(uint32_t side, double delete_frac, double shortcut_frac, uint64_t seed);

bool write_edge_list(const char *path, const EdgeList &e);

}  // namespace silvan
