// Device-side CSR preparation (see graph_dev.cuh).
#include "graph_dev.cuh"

namespace silvan {

namespace {

// Offsets above the entry count are clamped to it and flagged, so that no
// later kernel reads past the adjacency array.
__global__ void narrow_offsets_kernel(const uint64_t *in, uint32_t *out, uint32_t count,
                                      uint64_t limit, uint32_t *bad) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += gridDim.x * blockDim.x) {
        const uint64_t v = in[i];
        if (v > limit) atomicOr(bad, 1u);
        out[i] = (uint32_t)(v > limit ? limit : v);
    }
}

// one warp per row
__global__ void validate_rows_kernel(const uint32_t *off, const uint32_t *adj, uint32_t n,
                                     uint32_t *bad) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += nw) {
        const uint32_t b = off[v], e = off[v + 1];
        bool ok = e >= b;
        for (uint32_t k = b + lane; ok && k < e; k += 32) {
            const uint32_t y = adj[k];
            if (y >= n || (k > b && adj[k - 1] >= y)) ok = false;
        }
        if (__any_sync(0xffffffffu, !ok) && lane == 0) atomicOr(bad, 1u);
    }
}

__global__ void make_rows_kernel(const uint32_t *off, uint2 *rows, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        rows[v] = make_uint2(off[v], off[v + 1]);
}

}  // namespace

cudaError_t make_rows(const uint32_t *off, uint2 *rows, uint32_t n, cudaStream_t s) {
    make_rows_kernel<<<592, 256, 0, s>>>(off, rows, n);
    return cudaGetLastError();
}

cudaError_t narrow_offsets(const uint64_t *in, uint32_t *out, uint32_t count, uint64_t limit,
                           uint32_t *bad, cudaStream_t s) {
    narrow_offsets_kernel<<<592, 256, 0, s>>>(in, out, count, limit, bad);
    return cudaGetLastError();
}

cudaError_t validate_rows(const uint32_t *off, const uint32_t *adj, uint32_t n, uint32_t *bad,
                          cudaStream_t s) {
    validate_rows_kernel<<<1184, 256, 0, s>>>(off, adj, n, bad);
    return cudaGetLastError();
}

}  // namespace silvan
