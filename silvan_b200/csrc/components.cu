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
// Directed graphs keep the host path: their component numbers are the
// completion order of the reference's sequential DFS, which the void test of
// the sampler compares.
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

}  // namespace

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
