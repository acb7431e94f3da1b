// Device-side preparation of an uploaded CSR: 64-bit offsets narrowed to the
// 32-bit form the kernels read, and the row invariants the sampler relies on
// (ascending, unique, in range) checked without a host pass over the edges.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace silvan {

cudaError_t narrow_offsets(const uint64_t *in, uint32_t *out, uint32_t count, uint64_t limit,
                           uint32_t *bad, cudaStream_t s);
// rows[v] = (off[v], off[v + 1]) for v < n: a row's bounds in one 8-byte load
// (one memory transaction where two 4-byte loads take two).
cudaError_t make_rows(const uint32_t *off, uint2 *rows, uint32_t n, cudaStream_t s);
// *bad (device) becomes nonzero when a row is not ascending and unique, when
// an id is >= n, or when the offsets decrease.
cudaError_t validate_rows(const uint32_t *off, const uint32_t *adj, uint32_t n, uint32_t *bad,
                          cudaStream_t s);

}  // namespace silvan
