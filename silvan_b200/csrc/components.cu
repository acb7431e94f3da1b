// Components and the diameter bound of an undirected graph on the device,
// identical to the reference's compute_cc + estimate_diameter
// (silvan/src/Graph.cpp:109-316) for undirected graphs:
//   * Tarjan's iterative DFS starts from the roots in ascending id order and
//     an undirected component is one strongly connected component, numbered
//     when its DFS finishes, so component c is the one whose smallest node id
//     is the c-th smallest of all components' smallest ids;
//   * the pivot of a component is its node of largest degree sum, the lowest
//     id on ties (compute_pivot, :204-214);
//   * no edge joins two components, so the AllCCUpperBound recursion reduces
//     to max over components of ecc_f(pivot) + ecc_b(pivot) = 2 ecc(pivot),
//     the eccentricity being the distance of the last node of the BFS from
//     the pivot (compute_ecc_in_scc, :238-270).
// Components: lock-free union-find over the edges that always links the
// larger root under the smaller one (so every root is its component's
// smallest id), then every node's root and a prefix count of the roots.
// Eccentricities: one breadth-first search from all pivots at once (the
// components are disjoint), level by level.
//
// Directed graphs: their component numbers are the completion order of the
// reference's sequential DFS (the void test of the sampler compares them, so
// the numbering must be that DFS's, and a depth-first order is inherently
// sequential); the host computes them, and device_directed_bound computes
// the pivots, the eccentricities and the AllCCUpperBound recursion from them
// on the device.
#include <cub/cub.cuh>

#include <vector>

#include "components.h"

namespace silvan {

namespace {

#define CC_CK(x)                                                                    \
    do {                                                                            \
        cudaError_t e_ = (x);                                                       \
        if (e_ != cudaSuccess) return cuda_status(e_, "device components");         \
    } while (0)
#define CC_RK(x)                                                                    \
    do {                                                                            \
        int r_ = (x);                                                               \
        if (r_ != SILVAN_OK) return r_;                                             \
    } while (0)

__device__ __forceinline__ uint32_t find_root(uint32_t *parent, uint32_t x) {
    uint32_t p = __ldcg(&parent[x]);
    while (p != x) {
        const uint32_t gp = __ldcg(&parent[p]);
        if (gp != p) parent[x] = gp;  // path halving; a stale value is still an ancestor
        x = p;
        p = gp;
    }
    return x;
}

__global__ void cc_init_kernel(uint32_t *parent, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        parent[v] = v;
}

// One warp per row: every edge (u, w) unites the two sets.
__global__ void cc_union_kernel(const uint32_t *off, const uint32_t *adj, uint32_t n,
                                uint32_t *parent) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
        for (uint32_t k = off[u] + lane; k < off[u + 1]; k += 32) {
            const uint32_t w = adj[k];
            if (w <= u) continue;  // each undirected edge once
            uint32_t a = find_root(parent, u), b = find_root(parent, w);
            while (a != b) {
                if (a > b) {
                    const uint32_t t = a;
                    a = b;
                    b = t;
                }
                // link the larger root b under the smaller a, if b is still a root
                const uint32_t old = atomicCAS(&parent[b], b, a);
                if (old == b) break;
                a = find_root(parent, a);
                b = find_root(parent, old);
            }
        }
    }
}

// After the unions: every node's root, read-only (a compressing find here
// could overwrite another thread's final answer with an older ancestor).
__global__ void cc_compress_kernel(const uint32_t *parent, uint32_t n, uint32_t *root,
                                   uint32_t *is_root) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint32_t x = v, p = parent[v];
        while (p != x) {
            x = p;
            p = parent[x];
        }
        root[v] = x;
        is_root[v] = x == v ? 1u : 0u;
    }
}

// cc[v] = number of roots below v's root; the pivot key of each component:
// degree sum (2 x degree) in the high word, the inverted id in the low word.
__global__ void cc_number_kernel(const uint32_t *root, const uint32_t *rank, const uint32_t *off,
                                 uint32_t n, uint32_t *cc, unsigned long long *pivot_key) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t c = rank[root[v]];
        cc[v] = c;
        const unsigned long long deg2 = 2ull * (off[v + 1] - off[v]);
        atomicMax(&pivot_key[c], (deg2 << 32) | (0xffffffffull - v));
    }
}

__global__ void bfs_seed_kernel(const unsigned long long *pivot_key, uint32_t ncomp, int32_t *dist,
                                uint32_t *frontier) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncomp;
         c += gridDim.x * blockDim.x) {
        const uint32_t p = 0xffffffffu - (uint32_t)(pivot_key[c] & 0xffffffffull);
        dist[p] = 0;
        frontier[c] = p;
    }
}

// One warp per frontier node: unvisited neighbours join the next level.
__global__ void bfs_level_kernel(const uint32_t *off, const uint32_t *adj, const uint32_t *frontier,
                                 uint32_t count, int32_t level, int32_t *dist, uint32_t *next,
                                 uint32_t *next_count) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += warps) {
        const uint32_t u = frontier[i];
        for (uint32_t k = off[u] + lane; k < off[u + 1]; k += 32) {
            const uint32_t w = adj[k];
            if (__ldcg(&dist[w]) >= 0) continue;
            if (atomicCAS(&dist[w], -1, level + 1) == -1) next[atomicAdd(next_count, 1u)] = w;
        }
    }
}

__global__ void ecc_kernel(const int32_t *dist, const uint32_t *cc, uint32_t n, int32_t *ecc) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        atomicMax(&ecc[cc[v]], dist[v]);
}

__global__ void diam_kernel(const int32_t *ecc, uint32_t ncomp, unsigned int *diam) {
    uint32_t mx = 0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncomp;
         c += gridDim.x * blockDim.x)
        mx = max(mx, 2u * (uint32_t)ecc[c]);
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(diam, mx);
}

// ---- directed graphs: the diameter bound over given component ids --------

// Pivot key of every component: out + in degree in the high word, the
// inverted id in the low word (largest degree sum, lowest id on ties).
__global__ void dir_pivot_kernel(const uint32_t *oo, const uint32_t *io, const uint32_t *cc,
                                 uint32_t n, unsigned long long *pivot_key) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const unsigned long long d = (unsigned long long)(oo[v + 1] - oo[v]) + (io[v + 1] - io[v]);
        atomicMax(&pivot_key[cc[v]], (d << 32) | (0xffffffffull - v));
    }
}

__global__ void dir_seed_kernel(const unsigned long long *pivot_key, uint32_t ncomp,
                                int32_t *dist_f, int32_t *dist_b, uint32_t *frontier) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncomp;
         c += gridDim.x * blockDim.x) {
        const uint32_t p = 0xffffffffu - (uint32_t)(pivot_key[c] & 0xffffffffull);
        dist_f[p] = 0;
        dist_b[p] = 0;
        frontier[c] = p;
    }
}

// One level of the breadth-first searches from every pivot at once, each
// staying inside its pivot's component (the components are disjoint, so the
// searches never meet).
__global__ void dir_bfs_level_kernel(const uint32_t *off, const uint32_t *adj, const uint32_t *cc,
                                     const uint32_t *frontier, uint32_t count, int32_t level,
                                     int32_t *dist, uint32_t *next, uint32_t *next_count) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < count; i += warps) {
        const uint32_t u = frontier[i];
        const uint32_t cu = cc[u];
        for (uint32_t k = off[u] + lane; k < off[u + 1]; k += 32) {
            const uint32_t w = adj[k];
            if (cc[w] != cu || __ldcg(&dist[w]) >= 0) continue;
            if (atomicCAS(&dist[w], -1, level + 1) == -1) next[atomicAdd(next_count, 1u)] = w;
        }
    }
}

// Edges between different components, as (source component, target
// component); every one goes to a smaller id (Tarjan numbers a component
// after every component it reaches).
__global__ void dir_inter_kernel(const uint32_t *off, const uint32_t *adj, const uint32_t *cc,
                                 uint32_t n, uint2 *inter, unsigned long long *n_inter,
                                 unsigned long long cap, uint32_t *bad) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
        const uint32_t cu = cc[u];
        for (uint32_t k = off[u] + lane; k < off[u + 1]; k += 32) {
            const uint32_t cw = cc[adj[k]];
            if (cw == cu) continue;
            if (cw > cu) atomicExch(bad, 1u);
            const unsigned long long i = atomicAdd(n_inter, 1ull);
            if (i < cap) inter[i] = make_uint2(cu, cw);
        }
    }
}

// One pass of the AllCCUpperBound recursion (silvan/src/Graph.cpp:298-306)
// as a fixpoint: fp[c] = max(ecc_f[c], ecc_f[c] + 1 + ecc_b[d] + fp[d]) over
// the edges c -> d.  Passes repeat until nothing grows; the result is the
// recursion's, which the reference evaluates in ascending component order.
__global__ void dir_dp_kernel(const uint2 *inter, unsigned long long m, const int32_t *ecc_f,
                              const int32_t *ecc_b, int32_t *fp, uint32_t *changed) {
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < m;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint2 e = inter[i];
        const int32_t cand = ecc_f[e.x] + 1 + ecc_b[e.y] + __ldcg(&fp[e.y]);
        if (cand > __ldcg(&fp[e.x]) && atomicMax(&fp[e.x], cand) < cand) *changed = 1u;
    }
}

__global__ void dir_diam_kernel(const int32_t *fp, const int32_t *ecc_b, uint32_t ncomp,
                                unsigned int *diam) {
    uint32_t mx = 0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < ncomp;
         c += gridDim.x * blockDim.x)
        mx = max(mx, (uint32_t)(fp[c] + ecc_b[c]));
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(diam, mx);
}

}  // namespace

int device_directed_bound(DeviceGraph &G, cudaStream_t st) {
    const uint32_t n = G.n, ncomp = G.ncomp;
    std::vector<void *> bufs;
    struct Free {
        std::vector<void *> &b;
        ~Free() {
            for (void *p : b) device_free(p);
        }
    } fr{bufs};
    auto get = [&](void **p, size_t bytes) -> int {
        int rc = device_alloc(p, bytes);
        if (rc == SILVAN_OK) bufs.push_back(*p);
        return rc;
    };
    uint32_t *frontier = nullptr, *next = nullptr, *cnt = nullptr, *flag = nullptr;
    int32_t *dist_f = nullptr, *dist_b = nullptr, *ecc_f = nullptr, *ecc_b = nullptr, *fp = nullptr;
    unsigned long long *pivot_key = nullptr, *n_inter = nullptr;
    unsigned int *d_diam = nullptr;
    CC_RK(get((void **)&dist_f, 4ull * n));
    CC_RK(get((void **)&dist_b, 4ull * n));
    CC_RK(get((void **)&frontier, 4ull * n));
    CC_RK(get((void **)&next, 4ull * n));
    CC_RK(get((void **)&cnt, 16));
    CC_RK(get((void **)&flag, 16));
    CC_RK(get((void **)&n_inter, 8));
    CC_RK(get((void **)&d_diam, 4));
    CC_RK(get((void **)&pivot_key, 8ull * ncomp));
    CC_RK(get((void **)&ecc_f, 4ull * ncomp));
    CC_RK(get((void **)&ecc_b, 4ull * ncomp));
    CC_RK(get((void **)&fp, 4ull * ncomp));
    CC_CK(cudaMemsetAsync(pivot_key, 0, 8ull * ncomp, st));
    CC_CK(cudaMemsetAsync(ecc_f, 0, 4ull * ncomp, st));
    CC_CK(cudaMemsetAsync(ecc_b, 0, 4ull * ncomp, st));
    CC_CK(cudaMemsetAsync(dist_f, 0xff, 4ull * n, st));
    CC_CK(cudaMemsetAsync(dist_b, 0xff, 4ull * n, st));
    CC_CK(cudaMemsetAsync(d_diam, 0, 4, st));
    CC_CK(cudaMemsetAsync(n_inter, 0, 8, st));
    CC_CK(cudaMemsetAsync(flag, 0, 16, st));
    dir_pivot_kernel<<<592, 256, 0, st>>>(G.d_out_off, G.d_in_off, G.d_cc, n, pivot_key);
    dir_seed_kernel<<<64, 256, 0, st>>>(pivot_key, ncomp, dist_f, dist_b, frontier);
    CC_CK(cudaGetLastError());
    // eccentricity of every pivot inside its component, forward then backward
    // (compute_ecc_in_scc, silvan/src/Graph.cpp:238-270)
    for (int dir = 0; dir < 2; dir++) {
        const uint32_t *off = dir == 0 ? G.d_out_off : G.d_in_off;
        const uint32_t *adj = dir == 0 ? G.d_out_adj : G.d_in_adj;
        int32_t *dist = dir == 0 ? dist_f : dist_b;
        if (dir == 1) dir_seed_kernel<<<64, 256, 0, st>>>(pivot_key, ncomp, dist_f, dist_b, frontier);
        uint32_t count = ncomp;
        for (int32_t level = 0; count > 0; level++) {
            CC_CK(cudaMemsetAsync(cnt, 0, 4, st));
            dir_bfs_level_kernel<<<1184, 256, 0, st>>>(off, adj, G.d_cc, frontier, count, level,
                                                       dist, next, cnt);
            CC_CK(cudaGetLastError());
            CC_CK(cudaMemcpyAsync(&count, cnt, 4, cudaMemcpyDeviceToHost, st));
            CC_CK(cudaStreamSynchronize(st));
            std::swap(frontier, next);
        }
        ecc_kernel<<<592, 256, 0, st>>>(dist, G.d_cc, n, dir == 0 ? ecc_f : ecc_b);
        CC_CK(cudaGetLastError());
    }
    // the recursion over the condensation
    const uint64_t m = G.m;
    uint2 *inter = nullptr;
    CC_RK(get((void **)&inter, 8ull * std::max<uint64_t>(m, 1)));
    dir_inter_kernel<<<1184, 256, 0, st>>>(G.d_out_off, G.d_out_adj, G.d_cc, n, inter, n_inter, m,
                                           flag + 1);
    CC_CK(cudaMemcpyAsync(fp, ecc_f, 4ull * ncomp, cudaMemcpyDeviceToDevice, st));
    unsigned long long mi = 0;
    uint32_t badf = 0;
    CC_CK(cudaMemcpyAsync(&mi, n_inter, 8, cudaMemcpyDeviceToHost, st));
    CC_CK(cudaMemcpyAsync(&badf, flag + 1, 4, cudaMemcpyDeviceToHost, st));
    CC_CK(cudaStreamSynchronize(st));
    if (badf || mi > m) {
        set_error("component ids are not in the reference's completion order");
        return SILVAN_E_STATE;
    }
    // Pass p settles every component whose longest chain of descendants has
    // p edges, so shallow condensations (small-world graphs) take a few
    // passes; a deep one (a long chain of components) is finished by the
    // recursion in ascending order on the host copy, which directed graphs
    // keep for the component numbering.
    constexpr uint32_t kMaxPasses = 64;
    for (uint32_t pass = 0;; pass++) {
        uint32_t changed = 0;
        CC_CK(cudaMemsetAsync(flag, 0, 4, st));
        if (mi) dir_dp_kernel<<<1184, 256, 0, st>>>(inter, mi, ecc_f, ecc_b, fp, flag);
        CC_CK(cudaGetLastError());
        CC_CK(cudaMemcpyAsync(&changed, flag, 4, cudaMemcpyDeviceToHost, st));
        CC_CK(cudaStreamSynchronize(st));
        if (!changed) break;
        if (pass + 1 >= kMaxPasses) {
            if (!G.has_host || G.cc.size() != n) {
                set_error("diameter recursion needs the host copy of a deep condensation");
                return SILVAN_E_STATE;
            }
            std::vector<uint32_t> ef(ncomp), eb(ncomp);
            CC_CK(cudaMemcpyAsync(ef.data(), ecc_f, 4ull * ncomp, cudaMemcpyDeviceToHost, st));
            CC_CK(cudaMemcpyAsync(eb.data(), ecc_b, 4ull * ncomp, cudaMemcpyDeviceToHost, st));
            CC_CK(cudaStreamSynchronize(st));
            G.diameter = diameter_recursion(G.host, G.cc, ncomp, ef, eb);
            return SILVAN_OK;
        }
    }
    dir_diam_kernel<<<64, 256, 0, st>>>(fp, ecc_b, ncomp, d_diam);
    CC_CK(cudaGetLastError());
    unsigned int diam = 0;
    CC_CK(cudaMemcpyAsync(&diam, d_diam, 4, cudaMemcpyDeviceToHost, st));
    CC_CK(cudaStreamSynchronize(st));
    G.diameter = diam;
    return SILVAN_OK;
}

int device_undirected_components(DeviceGraph &G, cudaStream_t st) {
    const uint32_t n = G.n;
    std::vector<void *> bufs;
    struct Free {
        std::vector<void *> &b;
        ~Free() {
            for (void *p : b) device_free(p);
        }
    } fr{bufs};
    auto get = [&](void **p, size_t bytes) -> int {
        int rc = device_alloc(p, bytes);
        if (rc == SILVAN_OK) bufs.push_back(*p);
        return rc;
    };
    uint32_t *parent = nullptr, *root = nullptr, *is_root = nullptr, *rank = nullptr,
             *frontier = nullptr, *next = nullptr, *cnt = nullptr;
    int32_t *dist = nullptr, *ecc = nullptr;
    unsigned long long *pivot_key = nullptr;
    unsigned int *d_diam = nullptr;
    CC_RK(get((void **)&parent, 4ull * n));
    CC_RK(get((void **)&root, 4ull * n));
    CC_RK(get((void **)&is_root, 4ull * n));
    CC_RK(get((void **)&rank, 4ull * (n + 1)));
    CC_RK(get((void **)&dist, 4ull * n));
    CC_RK(get((void **)&frontier, 4ull * n));
    CC_RK(get((void **)&next, 4ull * n));
    CC_RK(get((void **)&cnt, 4));
    CC_RK(get((void **)&d_diam, 4));
    uint32_t *d_cc = nullptr;
    CC_RK(device_alloc((void **)&d_cc, 4ull * n));  // owned by the graph
    G.d_cc = d_cc;

    cc_init_kernel<<<592, 256, 0, st>>>(parent, n);
    cc_union_kernel<<<1184, 256, 0, st>>>(G.d_out_off, G.d_out_adj, n, parent);
    cc_compress_kernel<<<592, 256, 0, st>>>(parent, n, root, is_root);
    CC_CK(cudaGetLastError());
    size_t tb = 0;
    CC_CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, is_root, rank, n, st));
    void *tmp = nullptr;
    CC_RK(get(&tmp, tb));
    CC_CK(cub::DeviceScan::ExclusiveSum(tmp, tb, is_root, rank, n, st));
    uint32_t last_rank = 0, last_root = 0;
    CC_CK(cudaMemcpyAsync(&last_rank, rank + n - 1, 4, cudaMemcpyDeviceToHost, st));
    CC_CK(cudaMemcpyAsync(&last_root, is_root + n - 1, 4, cudaMemcpyDeviceToHost, st));
    CC_CK(cudaStreamSynchronize(st));
    const uint32_t ncomp = last_rank + last_root;
    CC_RK(get((void **)&pivot_key, 8ull * ncomp));
    CC_RK(get((void **)&ecc, 4ull * ncomp));
    CC_CK(cudaMemsetAsync(pivot_key, 0, 8ull * ncomp, st));
    CC_CK(cudaMemsetAsync(ecc, 0, 4ull * ncomp, st));
    CC_CK(cudaMemsetAsync(dist, 0xff, 4ull * n, st));
    CC_CK(cudaMemsetAsync(d_diam, 0, 4, st));
    cc_number_kernel<<<592, 256, 0, st>>>(root, rank, G.d_out_off, n, d_cc, pivot_key);
    bfs_seed_kernel<<<64, 256, 0, st>>>(pivot_key, ncomp, dist, frontier);
    CC_CK(cudaGetLastError());
    uint32_t count = ncomp;
    for (int32_t level = 0; count > 0; level++) {
        CC_CK(cudaMemsetAsync(cnt, 0, 4, st));
        bfs_level_kernel<<<1184, 256, 0, st>>>(G.d_out_off, G.d_out_adj, frontier, count, level,
                                               dist, next, cnt);
        CC_CK(cudaGetLastError());
        CC_CK(cudaMemcpyAsync(&count, cnt, 4, cudaMemcpyDeviceToHost, st));
        CC_CK(cudaStreamSynchronize(st));
        std::swap(frontier, next);
    }
    ecc_kernel<<<592, 256, 0, st>>>(dist, d_cc, n, ecc);
    diam_kernel<<<64, 256, 0, st>>>(ecc, ncomp, d_diam);
    CC_CK(cudaGetLastError());
    unsigned int diam = 0;
    CC_CK(cudaMemcpyAsync(&diam, d_diam, 4, cudaMemcpyDeviceToHost, st));
    CC_CK(cudaStreamSynchronize(st));
    G.ncomp = ncomp;
    G.diameter = diam;
    return SILVAN_OK;
}

}  // namespace silvan
