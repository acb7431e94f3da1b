// Exact betweenness on the device (Brandes, "A faster algorithm for
// betweenness centrality", J. Math. Sociol. 2001), normalised the way SILVAN
// estimates it: the sum over ordered pairs (s, t), s != t, of
// sigma_st(v) / sigma_st, divided by n (n - 1).  It is the ground truth for
// checking the (eps, delta) guarantee on graphs too large for the CPU
// restatement; the reference has no exact algorithm of its own.
//
// One CTA per source at a time (persistent; slot b takes the sources b,
// b + slots, ..., so that the result does not depend on scheduling).
// Forward: level-synchronous BFS, the node claimed by atomicCAS on its
// distance, path counts summed with atomicAdd on doubles
// (integers below 2^53, so the sum is exact in any order).  Backward: each
// node pulls the dependencies of its successors on the next level in row
// order (no atomics, so the value does not depend on scheduling).  Every
// slot adds its sources' dependencies into its own row of partial sums; the
// rows are summed in slot order at the end.
#include "brandes.h"

#include <vector>

namespace silvan {

namespace {

#define BK(x)                                                                       \
    do {                                                                            \
        cudaError_t e_ = (x);                                                       \
        if (e_ != cudaSuccess) return cuda_status(e_, "exact betweenness");         \
    } while (0)
#define BR(x)                                                                       \
    do {                                                                            \
        int r_ = (x);                                                               \
        if (r_ != SILVAN_OK) return r_;                                             \
    } while (0)

constexpr int kBlock = 512;

struct BrandesArgs {
    const uint32_t *out_off, *out_adj;
    uint32_t n;
    int32_t *dist;       // slot-major, n per slot, -1 = unvisited
    double *sigma;
    double *delta;
    uint32_t *queue;
    uint32_t *levels;    // slot-major, n + 2 per slot: queue index where each level starts
    double *partial;     // slot-major, n per slot
};

__global__ void __launch_bounds__(kBlock) brandes_kernel(BrandesArgs A) {
    __shared__ uint32_t s_tail, s_nlev;
    const uint64_t base = (uint64_t)blockIdx.x * A.n;
    int32_t *dist = A.dist + base;
    double *sigma = A.sigma + base;
    double *delta = A.delta + base;
    uint32_t *queue = A.queue + base;
    uint32_t *lvl = A.levels + (uint64_t)blockIdx.x * (A.n + 2);
    double *part = A.partial + base;
    for (uint32_t s = blockIdx.x; s < A.n; s += gridDim.x) {
        if (threadIdx.x == 0) {
            dist[s] = 0;
            sigma[s] = 1.0;
            queue[0] = s;
            s_tail = 1;
            lvl[0] = 0;
            lvl[1] = 1;
            s_nlev = 1;
        }
        __syncthreads();
        // forward BFS, one level at a time (a level is a queue segment)
        for (uint32_t lev = 0;; lev++) {
            const uint32_t lo = __ldcg(&lvl[lev]), hi = __ldcg(&lvl[lev + 1]);
            if (lo == hi) break;
            for (uint32_t i = lo + (threadIdx.x >> 5); i < hi; i += kBlock / 32) {
                const uint32_t x = queue[i];
                const double sx = sigma[x];
                const uint32_t rb = A.out_off[x], re = A.out_off[x + 1];
                for (uint32_t k = rb + (threadIdx.x & 31); k < re; k += 32) {
                    const uint32_t y = A.out_adj[k];
                    int32_t dy = __ldcg(&dist[y]);
                    if (dy < 0) {
                        const int32_t prev = atomicCAS(&dist[y], -1, (int32_t)lev + 1);
                        if (prev < 0) {
                            queue[atomicAdd(&s_tail, 1u)] = y;
                            dy = (int32_t)lev + 1;
                        } else {
                            dy = prev;
                        }
                    }
                    if (dy == (int32_t)lev + 1) atomicAdd(&sigma[y], sx);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                lvl[lev + 2] = s_tail;
                s_nlev = lev + 2;
            }
            __syncthreads();
        }
        // backward: delta(v) = sum over successors w of sigma(v)/sigma(w) (1 + delta(w)),
        // summed in row order
        const uint32_t nlev = s_nlev;
        for (int32_t lev = (int32_t)nlev - 1; lev >= 0; lev--) {
            const uint32_t lo = __ldcg(&lvl[lev]), hi = __ldcg(&lvl[lev + 1]);
            for (uint32_t i = lo + threadIdx.x; i < hi; i += kBlock) {
                const uint32_t v = queue[i];
                const double sv = sigma[v];
                double acc = 0.0;
                for (uint32_t k = A.out_off[v]; k < A.out_off[v + 1]; k++) {
                    const uint32_t w = A.out_adj[k];
                    if (__ldcg(&dist[w]) == lev + 1) acc += sv / sigma[w] * (1.0 + delta[w]);
                }
                delta[v] = acc;
                if (v != s) part[v] += acc;
            }
            __syncthreads();
        }
        // restore the visited nodes
        const uint32_t tail = s_tail;
        for (uint32_t i = threadIdx.x; i < tail; i += kBlock) {
            const uint32_t v = queue[i];
            dist[v] = -1;
            sigma[v] = 0.0;
            delta[v] = 0.0;
        }
        __syncthreads();
    }
}

__global__ void brandes_init_kernel(int32_t *dist, double *sigma, double *delta, double *partial,
                                    uint64_t total) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        dist[i] = -1;
        sigma[i] = 0.0;
        delta[i] = 0.0;
        partial[i] = 0.0;
    }
}

__global__ void brandes_sum_kernel(const double *partial, uint32_t n, uint32_t slots,
                                   double norm, double *out) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (uint32_t s = 0; s < slots; s++) acc += partial[(uint64_t)s * n + v];
        out[v] = acc / norm;
    }
}

}  // namespace

int exact_betweenness(const DeviceGraph &G, double *out_host) {
    const uint32_t n = G.n;
    int dev = 0, sms = 0;
    BK(cudaGetDevice(&dev));
    BK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // slots: a few per SM, bounded by a quarter of the free memory
    size_t fr = 0, tot = 0;
    BK(cudaMemGetInfo(&fr, &tot));
    const uint64_t per_slot = (uint64_t)n * (4 + 8 + 8 + 4 + 4 + 8) + 8;
    uint64_t slots = std::min<uint64_t>((uint64_t)sms * 2, std::max<uint64_t>(1, fr / 4 / per_slot));
    slots = std::min<uint64_t>(slots, n);
    BrandesArgs A{};
    A.out_off = G.d_out_off;
    A.out_adj = G.d_out_adj;
    A.n = n;
    void *p = nullptr;
    struct Bufs {
        std::vector<void *> v;
        ~Bufs() {
            for (void *b : v) device_free(b);
        }
    } bufs;
    auto get = [&](void **q, size_t bytes) -> int {
        int rc = device_alloc(q, bytes);
        if (rc == SILVAN_OK) bufs.v.push_back(*q);
        return rc;
    };
    const uint64_t tot_nodes = slots * n;
    BR(get(&p, 4 * tot_nodes));
    A.dist = (int32_t *)p;
    BR(get(&p, 8 * tot_nodes));
    A.sigma = (double *)p;
    BR(get(&p, 8 * tot_nodes));
    A.delta = (double *)p;
    BR(get(&p, 4 * tot_nodes));
    A.queue = (uint32_t *)p;
    BR(get(&p, 4 * slots * ((uint64_t)n + 2)));
    A.levels = (uint32_t *)p;
    BR(get(&p, 8 * tot_nodes));
    A.partial = (double *)p;
    double *d_out = nullptr;
    BR(get(&p, 8 * (uint64_t)n));
    d_out = (double *)p;
    brandes_init_kernel<<<1184, 256>>>(A.dist, A.sigma, A.delta, A.partial, tot_nodes);
    BK(cudaGetLastError());
    brandes_kernel<<<(uint32_t)slots, kBlock>>>(A);
    BK(cudaGetLastError());
    brandes_sum_kernel<<<(n + 255) / 256, 256>>>(A.partial, n, (uint32_t)slots,
                                                 (double)n * (double)(n - 1), d_out);
    BK(cudaGetLastError());
    BK(cudaMemcpy(out_host, d_out, sizeof(double) * n, cudaMemcpyDeviceToHost));
    return SILVAN_OK;
}

}  // namespace silvan
