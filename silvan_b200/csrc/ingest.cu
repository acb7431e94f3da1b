// Device-side edge-list ingest: the text file is parsed and turned into the
// CSR on the GPU, with exactly the line semantics of the reference loader
// (silvan/src/Graph.cpp:37-90, restated on the host in graph_host.cpp):
//   * lines end at '\n'; a final line without '\n' counts, an empty remainder
//     after the last '\n' does not;
//   * a line whose first byte is '#' is skipped;
//   * every other line goes through sscanf("%u %u"): whatever the conversion
//     leaves in (u, v) is inserted, so a line that fails to parse re-inserts
//     the previous pair ((0, 0) before the first one), and a line with only
//     one number keeps the previous v;
//   * a negative id or one above kMaxNodeId is an error with its line number;
//   * self-loops are kept, duplicates removed, rows ascending, n = 1 + max id.
//
// Steps: newline positions (device select), one thread per line parses its
// two numbers, the values carried over from earlier lines come from a
// max-scan over "last line that set u / v", kept lines become 64-bit
// (row << 32 | column) keys, and a radix sort + unique + row-boundary pass
// gives the CSR.  The scans, the select, the sort and the unique are CUB's
// device primitives; the parsing and CSR kernels are this file's.
//
// The CSR stays on the device.  For an undirected graph the components and
// the diameter bound are computed there too (components.cu); for a directed
// graph a host copy is read back for the reference's Tarjan numbering and the
// bound (graph_host.cpp).
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include <cstdio>
#include <string>
#include <vector>

#include "engine.h"
#include "ingest.h"
#include "components.h"

namespace silvan {

namespace {

struct IsNewline {
    const unsigned char *text;
    __device__ bool operator()(const uint64_t i) const { return text[i] == '\n'; }
};

struct NewlineOne {
    __device__ uint64_t operator()(const unsigned char c) const { return c == '\n' ? 1u : 0u; }
};

struct Widen {
    __device__ uint64_t operator()(const uint8_t k) const { return k; }
};

struct MaxOp {
    __device__ uint64_t operator()(uint64_t a, uint64_t b) const { return a > b ? a : b; }
};

__device__ __forceinline__ bool is_space(unsigned char c) {
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// One "%u" conversion (graph_host.cpp: scan_u): 1 converted, 0 no conversion,
// -1 an id the reference cannot hold.
__device__ int scan_u(const unsigned char *text, uint64_t &p, uint64_t end, uint32_t &out) {
    while (p < end && is_space(text[p])) p++;
    uint64_t q = p;
    bool neg = false;
    if (q < end && (text[q] == '+' || text[q] == '-')) {
        neg = text[q] == '-';
        q++;
    }
    if (q >= end || text[q] < '0' || text[q] > '9') return 0;
    uint64_t v = 0;
    bool big = false;
    while (q < end && text[q] >= '0' && text[q] <= '9') {
        v = v * 10 + (uint64_t)(text[q] - '0');
        if (v > kMaxNodeId) big = true;
        if (v > (1ull << 40)) v = 1ull << 40;
        q++;
    }
    p = q;
    if (neg || big) return -1;
    out = (uint32_t)v;
    return 1;
}

// Per line: keep (inserted) or skipped ('#'), the ids it converted, and the
// 1-based index of the line as the "last setter" of u and of v (0 if not).
__global__ void parse_lines_kernel(const unsigned char *text, uint64_t size, const uint64_t *nl,
                                   uint64_t n_nl, uint64_t lines, uint8_t *keep, uint32_t *uval,
                                   uint32_t *vval, uint64_t *uset, uint64_t *vset,
                                   unsigned long long *first_error) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < lines;
         j += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t start = j == 0 ? 0 : nl[j - 1] + 1;
        const uint64_t end = j < n_nl ? nl[j] : size;
        uint8_t k = 0;
        uint64_t us = 0, vs = 0;
        uint32_t u = 0, v = 0;
        if (end == start || text[start] != '#') {
            k = 1;
            uint64_t p = start;
            int r = scan_u(text, p, end, u);
            if (r == 1) {
                us = j + 1;
                while (p < end && is_space(text[p])) p++;
                r = scan_u(text, p, end, v);
                if (r == 1) vs = j + 1;
            }
            if (r < 0) atomicMin(first_error, (unsigned long long)j);
        }
        keep[j] = k;
        uval[j] = u;
        vval[j] = v;
        uset[j] = us;
        vset[j] = vs;
    }
}

// Effective (u, v) of every kept line from the last setters, as keys, and
// the largest id.  pos = exclusive prefix of keep.
__global__ void emit_keys_kernel(uint64_t lines, const uint8_t *keep, const uint64_t *pos,
                                 const uint32_t *uval, const uint32_t *vval,
                                 const uint64_t *ulast, const uint64_t *vlast, int directed,
                                 uint64_t *out_keys, uint64_t *in_keys, uint64_t edges,
                                 unsigned int *max_id) {
    uint32_t mx = 0;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < lines;
         j += (uint64_t)gridDim.x * blockDim.x) {
        if (!keep[j]) continue;
        const uint32_t u = ulast[j] ? uval[ulast[j] - 1] : 0u;
        const uint32_t v = vlast[j] ? vval[vlast[j] - 1] : 0u;
        const uint64_t e = pos[j];
        out_keys[e] = ((uint64_t)u << 32) | v;
        if (directed) in_keys[e] = ((uint64_t)v << 32) | u;
        else out_keys[edges + e] = ((uint64_t)v << 32) | u;
        mx = max(mx, max(u, v));
    }
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(max_id, mx);
}

// Row offsets from sorted unique keys: off[r] = first key index with row >= r.
__global__ void csr_offsets_kernel(const uint64_t *keys, uint64_t m, uint32_t n, uint32_t *off,
                                   uint32_t *adj) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const int64_t row = i < m ? (int64_t)(keys[i] >> 32) : (int64_t)n;
        const int64_t prev = i == 0 ? -1 : (int64_t)(keys[i - 1] >> 32);
        for (int64_t r = prev + 1; r <= row && r <= (int64_t)n; r++) off[r] = (uint32_t)i;
        if (i < m) adj[i] = (uint32_t)keys[i];
    }
}

template <typename T>
int dalloc(T **p, uint64_t count) {
    return device_alloc((void **)p, sizeof(T) * (count ? count : 1));
}

// Frees every registered buffer when the ingest returns.
struct Scratch {
    std::vector<void *> bufs;
    template <typename T>
    int get(T **p, uint64_t count) {
        int rc = dalloc(p, count);
        if (rc == SILVAN_OK) bufs.push_back(*p);
        return rc;
    }
    ~Scratch() {
        for (void *b : bufs) device_free(b);
    }
};

#define CKI(x)                                                                      \
    do {                                                                            \
        cudaError_t e_ = (x);                                                       \
        if (e_ != cudaSuccess) return cuda_status(e_, "device ingest");             \
    } while (0)
#define RKI(x)                                                                      \
    do {                                                                            \
        int r_ = (x);                                                               \
        if (r_ != SILVAN_OK) return r_;                                             \
    } while (0)

// Sorted unique keys -> CSR (u32 offsets) on the device and the host copy.
int keys_to_device_csr(Scratch &S, uint64_t *keys, uint64_t count, uint32_t n, int end_bit,
                       cudaStream_t st, uint32_t **d_off, uint32_t **d_adj, uint64_t *m_out,
                       std::vector<uint64_t> &h_off, std::vector<uint32_t> &h_adj,
                       bool host_copy) {
    uint64_t *sorted = nullptr, *uniq = nullptr, *d_m = nullptr;
    RKI(S.get(&sorted, count));
    RKI(S.get(&uniq, count));
    RKI(S.get(&d_m, 1));
    size_t tb = 0, tb2 = 0;
    CKI(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys, sorted, count, 0, end_bit, st));
    CKI(cub::DeviceSelect::Unique(nullptr, tb2, sorted, uniq, d_m, count, st));
    void *tmp = nullptr;
    RKI(S.get((unsigned char **)&tmp, std::max(tb, tb2)));
    CKI(cub::DeviceRadixSort::SortKeys(tmp, tb, keys, sorted, count, 0, end_bit, st));
    CKI(cub::DeviceSelect::Unique(tmp, tb2, sorted, uniq, d_m, count, st));
    uint64_t m = 0;
    CKI(cudaMemcpyAsync(&m, d_m, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
    CKI(cudaStreamSynchronize(st));
    if (m >= 0xffffffffull) {
        set_error("graphs with 2^32 or more edge entries are not supported");
        return SILVAN_E_BADARG;
    }
    RKI(dalloc(d_off, (uint64_t)n + 1));
    RKI(dalloc(d_adj, m));
    csr_offsets_kernel<<<1184, 256, 0, st>>>(uniq, m, n, *d_off, *d_adj);
    CKI(cudaGetLastError());
    if (host_copy) {
        std::vector<uint32_t> off32((size_t)n + 1);
        h_adj.resize(m);
        CKI(cudaMemcpyAsync(off32.data(), *d_off, sizeof(uint32_t) * ((size_t)n + 1),
                            cudaMemcpyDeviceToHost, st));
        if (m)
            CKI(cudaMemcpyAsync(h_adj.data(), *d_adj, sizeof(uint32_t) * m,
                                cudaMemcpyDeviceToHost, st));
        CKI(cudaStreamSynchronize(st));
        h_off.assign(off32.begin(), off32.end());
    } else {
        CKI(cudaStreamSynchronize(st));
    }
    *m_out = m;
    return SILVAN_OK;
}

}  // namespace

int device_ingest(const char *path, bool directed, DeviceGraph &G, std::string &err) {
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        err = std::string("cannot open graph file: ") + path;
        return SILVAN_E_IO;
    }
    std::fseek(f, 0, SEEK_END);
    const long fsz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (fsz < 0) {
        std::fclose(f);
        err = std::string("cannot read graph file: ") + path;
        return SILVAN_E_IO;
    }
    const uint64_t size = (uint64_t)fsz;
    std::vector<unsigned char> text(size ? size : 1);
    const size_t got = size ? std::fread(text.data(), 1, size, f) : 0;
    std::fclose(f);
    if (got != size) {
        err = std::string("cannot read graph file: ") + path;
        return SILVAN_E_IO;
    }
    cudaStream_t st = nullptr;
    CKI(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } sg{st};
    Scratch S;
    unsigned char *d_text = nullptr;
    RKI(S.get(&d_text, size));
    if (size) CKI(cudaMemcpyAsync(d_text, text.data(), size, cudaMemcpyHostToDevice, st));

    // ---- newline positions ------------------------------------------------
    uint64_t *nl = nullptr, *d_cnt = nullptr;
    uint64_t n_nl = 0;
    RKI(S.get(&d_cnt, 1));
    if (size) {
        thrust::transform_iterator<NewlineOne, const unsigned char *> ones(d_text, NewlineOne());
        size_t tr = 0;
        CKI(cub::DeviceReduce::Sum(nullptr, tr, ones, d_cnt, size, st));
        void *tmp = nullptr;
        RKI(S.get((unsigned char **)&tmp, tr));
        CKI(cub::DeviceReduce::Sum(tmp, tr, ones, d_cnt, size, st));
        CKI(cudaMemcpyAsync(&n_nl, d_cnt, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        CKI(cudaStreamSynchronize(st));
        RKI(S.get(&nl, n_nl));
        thrust::counting_iterator<uint64_t> idx(0);
        size_t ts = 0;
        CKI(cub::DeviceSelect::If(nullptr, ts, idx, nl, d_cnt, size, IsNewline{d_text}, st));
        void *tmp2 = nullptr;
        RKI(S.get((unsigned char **)&tmp2, ts));
        CKI(cub::DeviceSelect::If(tmp2, ts, idx, nl, d_cnt, size, IsNewline{d_text}, st));
    }
    uint64_t tail_start = 0;
    if (n_nl)
        CKI(cudaMemcpyAsync(&tail_start, nl + n_nl - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                            st));
    CKI(cudaStreamSynchronize(st));
    if (n_nl) tail_start += 1;
    const uint64_t lines = n_nl + (size > tail_start ? 1 : 0);

    // ---- parse ------------------------------------------------------------
    uint8_t *keep = nullptr;
    uint32_t *uval = nullptr, *vval = nullptr;
    uint64_t *uset = nullptr, *vset = nullptr, *ulast = nullptr, *vlast = nullptr, *pos = nullptr;
    unsigned long long *d_err = nullptr;
    unsigned int *d_max = nullptr;
    RKI(S.get(&keep, lines + 1));
    RKI(S.get(&uval, lines));
    RKI(S.get(&vval, lines));
    RKI(S.get(&uset, lines));
    RKI(S.get(&vset, lines));
    RKI(S.get(&ulast, lines));
    RKI(S.get(&vlast, lines));
    RKI(S.get(&pos, lines + 1));
    RKI(S.get(&d_err, 1));
    RKI(S.get(&d_max, 1));
    CKI(cudaMemsetAsync(d_err, 0xff, sizeof(unsigned long long), st));
    CKI(cudaMemsetAsync(d_max, 0, sizeof(unsigned int), st));
    CKI(cudaMemsetAsync(keep + lines, 0, 1, st));
    uint64_t edges = 0;
    if (lines) {
        parse_lines_kernel<<<1184, 256, 0, st>>>(d_text, size, nl, n_nl, lines, keep, uval, vval,
                                                 uset, vset, d_err);
        CKI(cudaGetLastError());
        unsigned long long first_err = 0;
        CKI(cudaMemcpyAsync(&first_err, d_err, sizeof(first_err), cudaMemcpyDeviceToHost, st));
        CKI(cudaStreamSynchronize(st));
        if (first_err != ~0ull) {
            err = "graph file line " + std::to_string(first_err + 1) +
                  ": node id is negative or larger than " + std::to_string(kMaxNodeId);
            return SILVAN_E_PARSE;
        }
        // last setters of u and v up to each line; positions of kept lines
        thrust::transform_iterator<Widen, const uint8_t *> keep64(keep, Widen());
        size_t t1 = 0, t2 = 0;
        CKI(cub::DeviceScan::InclusiveScan(nullptr, t1, uset, ulast, MaxOp(), lines, st));
        CKI(cub::DeviceScan::ExclusiveSum(nullptr, t2, keep64, pos, lines + 1, st));
        void *tmp = nullptr;
        RKI(S.get((unsigned char **)&tmp, std::max(t1, t2)));
        CKI(cub::DeviceScan::InclusiveScan(tmp, t1, uset, ulast, MaxOp(), lines, st));
        CKI(cub::DeviceScan::InclusiveScan(tmp, t1, vset, vlast, MaxOp(), lines, st));
        CKI(cub::DeviceScan::ExclusiveSum(tmp, t2, keep64, pos, lines + 1, st));
        CKI(cudaMemcpyAsync(&edges, pos + lines, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        CKI(cudaStreamSynchronize(st));
    }

    // ---- keys -------------------------------------------------------------
    const uint64_t n_out = directed ? edges : 2 * edges;
    uint64_t *out_keys = nullptr, *in_keys = nullptr;
    RKI(S.get(&out_keys, n_out));
    if (directed) RKI(S.get(&in_keys, edges));
    uint32_t n = 0;
    if (edges) {
        emit_keys_kernel<<<1184, 256, 0, st>>>(lines, keep, pos, uval, vval, ulast, vlast,
                                               directed ? 1 : 0, out_keys, in_keys, edges, d_max);
        CKI(cudaGetLastError());
        unsigned int mx = 0;
        CKI(cudaMemcpyAsync(&mx, d_max, sizeof(mx), cudaMemcpyDeviceToHost, st));
        CKI(cudaStreamSynchronize(st));
        n = mx + 1;
    }

    // ---- CSR --------------------------------------------------------------
    G.n = n;
    G.directed = directed;
    G.host.n = n;
    G.host.directed = directed;
    if (n < 2) {
        // the host loader builds the same (empty or one-node) graph; the
        // upload rejects it
        set_error("graph needs at least two nodes");
        return SILVAN_E_BADARG;
    }
    int end_bit = 32;
    while (end_bit < 64 && ((uint64_t)(n - 1) >> (end_bit - 32)) != 0) end_bit++;
    // undirected graphs: components and diameter bound on the device too, no
    // host copy; directed graphs: the reference's Tarjan numbering on the host
    const bool host_copy = directed;
    uint64_t m = 0, m_in = 0;
    RKI(keys_to_device_csr(S, out_keys, n_out, n, end_bit, st, &G.d_out_off, &G.d_out_adj, &m,
                           G.host.out_off, G.host.out_adj, host_copy));
    if (directed) {
        RKI(keys_to_device_csr(S, in_keys, edges, n, end_bit, st, &G.d_in_off, &G.d_in_adj, &m_in,
                               G.host.in_off, G.host.in_adj, host_copy));
    } else {
        G.d_in_off = G.d_out_off;
        G.d_in_adj = G.d_out_adj;
        m_in = m;
        G.host.in_off.clear();
        G.host.in_adj.clear();
    }
    G.m = m;
    G.m_in = m_in;
    CKI(cudaGetDevice(&G.device));
    RKI(G.make_rows(st));
    if (directed) {
        G.has_host = true;
        return G.finish_from_host_copy();
    }
    G.has_host = false;
    const double t0 = now_seconds();
    RKI(device_undirected_components(G, st));
    G.diameter_seconds = now_seconds() - t0;
    return SILVAN_OK;
}

}  // namespace silvan
