// Host side of the graph store: edge-list ingest with the reference loader's
// semantics, CSR layout, strongly connected components and the diameter
// upper bound that sizes the estimator (the reference's silvan/src/Graph.cpp).
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace silvan {

// Compressed sparse rows, neighbours ascending and unique per row (the
// reference keeps them in std::set, silvan/src/Graph.cpp:39-56).  For an
// undirected graph the in-rows alias the out-rows, as `inc = adj` does in
// silvan/src/Graph.cpp:67-69.
struct HostGraph {
    uint32_t n = 0;
    bool directed = false;
    std::vector<uint64_t> out_off;  // n + 1
    std::vector<uint32_t> out_adj;
    std::vector<uint64_t> in_off;   // n + 1, directed only
    std::vector<uint32_t> in_adj;   // directed only

    uint64_t num_edges() const { return out_adj.size(); }  // edges_num of the reference
    const uint64_t *in_offsets() const { return directed ? in_off.data() : out_off.data(); }
    const uint32_t *in_neighbours() const { return directed ? in_adj.data() : out_adj.data(); }
    uint32_t out_degree(uint32_t v) const { return (uint32_t)(out_off[v + 1] - out_off[v]); }
    uint32_t in_degree(uint32_t v) const {
        const uint64_t *o = in_offsets();
        return (uint32_t)(o[v + 1] - o[v]);
    }
};

// Largest node id accepted by the loader.  The reference computes
// n = 1 + max id in uint32_t (silvan/src/Graph.cpp:48) and cannot hold ids
// near 2^32; larger ids are rejected here instead.
constexpr uint32_t kMaxNodeId = 0x7FFFFFFEu;

// Reads a `u v` edge list with the reference's line semantics
// (silvan/src/Graph.cpp:45-57): a line whose first character is '#' is
// skipped; every other line goes through sscanf("%u %u") and the pair left
// in (u, v) is inserted, so a line that fails to parse re-inserts the
// previous pair (or (0, 0) before the first pair).  Self-loops are kept.
// Returns 0, or a negative SILVAN_E_* code with a message in err.
int load_edge_list(const char *path, bool directed, HostGraph &g, std::string &err);

// Builds the CSR from (u, v) pairs with the same semantics as the loader
// (dedup, ascending rows, reverse direction added when undirected,
// n = 1 + max id).
void build_csr(const std::vector<std::pair<uint32_t, uint32_t>> &pairs, bool directed,
               HostGraph &g);

// Strongly connected components in the numbering of the reference's
// iterative Tarjan (silvan/src/Graph.cpp:109-199): reverse topological order,
// components numbered as they complete.  Returns the number of components.
uint32_t compute_scc(const HostGraph &g, std::vector<uint32_t> &cc);

// AllCCUpperBound diameter bound (silvan/src/Graph.cpp:205-316).
uint32_t estimate_diameter(const HostGraph &g, const std::vector<uint32_t> &cc, uint32_t ncomp);
// The AllCCUpperBound recursion over the condensation (Graph.cpp:298-306)
// from every component's forward and backward pivot eccentricity.
uint32_t diameter_recursion(const HostGraph &g, const std::vector<uint32_t> &cc, uint32_t ncomp,
                            const std::vector<uint32_t> &ecc_f, const std::vector<uint32_t> &ecc_b);

}  // namespace silvan
