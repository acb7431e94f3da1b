// silvan_replay_samples_noalloc: the per-sample sampler with its scratch in a
// fixed device array, for callers that must not allocate device memory.
//
// Who needs it.  Some callers cannot let a library allocate GPU memory: a
// process that shares the GPU under a strict quota and already holds all the
// memory it may use, or a runtime (a framework's memory pool, an embedding
// host) that hands its libraries only buffers it allocated itself and
// forbids allocation calls behind its back.  The regular entry points
// allocate the sampler slots (tens of MB per slot) and the round buffers on
// first use; this one uses only the array below plus the buffers the caller
// passes, and calls no allocating routine.
//
// The scratch is a file-scope static __device__ array of kScratchBytes
// (64 MiB), held by every GPU that loads the library until the process exits.
// Host code must not pass the array's name to a kernel: on the host it is a
// stand-in symbol, not a device address.  The device address is taken once per
// device, with that device current, by cudaGetSymbolAddress during the first
// call on that device, and cached; that first call should therefore come
// before any stream capture.  The cached address does not survive a
// cudaDeviceReset (a process that resets a device must not call this entry
// point on it again).  All calls share the array and it keeps the previous
// call's contents, so every call re-initialises the part it uses; calls that
// overlap on the GPU (different streams, or different host threads) race on
// it.
#include <mutex>
#include <string>

#include "engine.h"
#include "sampler.cuh"

namespace silvan {

namespace {

constexpr size_t kScratchBytes = 64ull << 20;
constexpr uint32_t kMaxSamples = 65536;  // samples per call
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_sampler_scratch[kScratchBytes];

std::mutex g_setup_mu;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch on the current device (set up once).
int scratch_address(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_error("no usable CUDA device");
        return SILVAN_E_NOGPU;
    }
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sampler_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error(std::string("cudaGetSymbolAddress of the sampler scratch failed: ") +
                      cudaGetErrorString(e));
            return SILVAN_E_CUDA;
        }
        g_scratch_ptr[dev] = (unsigned char *)p;
    }
    *out = g_scratch_ptr[dev];
    return SILVAN_OK;
}

// Writes the round header and the single segment into the scratch on the
// stream (kernel parameters, so no host staging buffer is needed).
__global__ void noalloc_setup_kernel(RoundHeader *hdr, SegDesc *seg, RoundHeader h, SegDesc s) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *hdr = h;
        *seg = s;
    }
}

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Scratch layout: header | segment | ball[kMaxSamples] | pred[kMaxSamples] |
// slots.  A slot takes a node record and three u32 words per node, the
// meeting-edge list and its prefix, and up to 256 bytes of alignment for
// each of its six arrays.
constexpr size_t kHeadBytes = align256(sizeof(RoundHeader)) + align256(sizeof(SegDesc)) +
                              2 * align256(sizeof(uint32_t) * kMaxSamples);
constexpr size_t kSlotBytesPerNode = sizeof(NodeRec) + 3 * sizeof(uint32_t);
constexpr size_t kSlotFixedBytes = (sizeof(uint2) + sizeof(uint64_t)) * kMeetCap + 6 * 256;
// largest graph for which one slot fits
constexpr uint64_t kMaxNodes = (kScratchBytes - kHeadBytes - kSlotFixedBytes) / kSlotBytesPerNode;

}  // namespace

int replay_samples_noalloc(const DeviceGraph &G, uint64_t seed, uint32_t first, uint32_t count,
                           double alpha, uint32_t np_cap, int32_t *d_path_length,
                           int32_t *d_num_paths, uint64_t *d_vis_edges, int32_t *d_status,
                           uint32_t *d_records, uint64_t record_cap,
                           unsigned long long *d_record_count, cudaStream_t stream) {
    if (!d_path_length || !d_num_paths || !d_vis_edges || !d_status || !d_record_count ||
        (!d_records && record_cap)) {
        set_error("null output buffer");
        return SILVAN_E_BADARG;
    }
    if (count == 0) return SILVAN_OK;
    if (count > kMaxSamples) {
        set_error("silvan_replay_samples_noalloc draws at most 65536 samples per call");
        return SILVAN_E_CAPACITY;
    }
    {
        int cur = -1;
        if (cudaGetDevice(&cur) != cudaSuccess || cur != G.device) {
            cudaGetLastError();
            set_error("silvan_replay_samples_noalloc must run with the graph's device current "
                      "(the scratch is per device)");
            return SILVAN_E_BADARG;
        }
    }
    unsigned char *base = nullptr;
    int rc = scratch_address(&base);
    if (rc != SILVAN_OK) return rc;
    // scratch layout (kHeadBytes, then the slots)
    const uint64_t n = G.n;
    size_t off = 0;
    RoundHeader *hdr = (RoundHeader *)(base + off);
    off += align256(sizeof(RoundHeader));
    SegDesc *seg = (SegDesc *)(base + off);
    off += align256(sizeof(SegDesc));
    uint32_t *ball = (uint32_t *)(base + off);
    off += align256(sizeof(uint32_t) * kMaxSamples);
    uint32_t *pred = (uint32_t *)(base + off);
    off += align256(sizeof(uint32_t) * kMaxSamples);
    const size_t per_slot = kSlotBytesPerNode * n + kSlotFixedBytes;
    const size_t avail = kScratchBytes - off;
    uint64_t slots = avail / per_slot;
    if (slots == 0) {
        set_error("graph of " + std::to_string(n) +
                  " nodes too large for the fixed sampler scratch of "
                  "silvan_replay_samples_noalloc (64 MiB: at most " +
                  std::to_string(kMaxNodes) + " nodes)");
        return SILVAN_E_CAPACITY;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    slots = std::min<uint64_t>(slots, (uint64_t)sms * std::max(1, sampler_max_ctas_per_sm()));
    slots = std::min<uint64_t>(slots, count);
    SlotArrays S{};
    S.stride = n;
    S.rec = (NodeRec *)(base + off);
    off += align256(sizeof(NodeRec) * n * slots);
    S.queue = (uint32_t *)(base + off);
    off += align256(sizeof(uint32_t) * n * slots);
    S.hits = (uint32_t *)(base + off);
    off += align256(sizeof(uint32_t) * n * slots);
    S.touched = (uint32_t *)(base + off);
    off += align256(sizeof(uint32_t) * n * slots);
    S.meet = (uint2 *)(base + off);
    off += align256(sizeof(uint2) * kMeetCap * slots);
    S.meet_pre = (uint64_t *)(base + off);
    off += align256(sizeof(uint64_t) * kMeetCap * slots);
    if (off > kScratchBytes) {
        set_error("internal scratch layout overflow");
        return SILVAN_E_STATE;
    }
    SegDesc sd{};
    sd.out_off = G.d_out_off;
    sd.out_rows = G.d_out_rows;
    sd.in_rows = G.d_in_rows;
    sd.out_adj = G.d_out_adj;
    sd.in_off = G.d_in_off;
    sd.in_adj = G.d_in_adj;
    sd.cc = G.d_cc;
    sd.n = G.n;
    sd.directed = G.directed ? 1 : 0;
    sd.seed = seed;
    sd.alpha = alpha;
    sd.np_cap = np_cap ? np_cap : (1u << 24);
    sd.first_sample = first;
    sd.count = count;
    sd.base = 0;
    sd.out_pl = d_path_length;
    sd.out_np = d_num_paths;
    sd.out_vis = d_vis_edges;
    sd.out_status = d_status;
    sd.out_ball = ball;
    sd.out_pred = pred;
    sd.recs = reinterpret_cast<PathRec *>(d_records);
    sd.rec_cursor = d_record_count;
    sd.rec_cap = record_cap;
    RoundHeader h{};
    h.nsegs = 1u;
    h.total = count;
    h.wait_polls = kDefaultWaitPolls;
    SamplerLaunch L{};
    L.slots = S;
    L.hdr = hdr;
    L.segs = seg;
    // the array keeps the previous call's contents: restore neutral records
    cudaError_t e = sampler_init_slots(S.rec, S.hits, n * slots, stream);
    if (e == cudaSuccess) {
        noalloc_setup_kernel<<<1, 32, 0, stream>>>(hdr, seg, h, sd);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = sampler_round_begin(L, 1, stream);
    if (e == cudaSuccess) e = sampler_launch(L, (uint32_t)slots, stream);
    return cuda_status(e, "silvan_replay_samples_noalloc launch");
}

}  // namespace silvan
