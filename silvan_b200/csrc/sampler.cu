// Device s-t shortest-path sampler (see sampler.cuh).
//
// One CTA slot processes one sample at a time and takes the next round-local
// sample index from a device counter, so a round of many samples runs as one
// persistent launch (the batched form) and a round of 11 samples as a small
// one (the plain form); both execute the same per-sample code.
//
// Exactness.  The reference expands a BFS level by scanning the frontier in
// queue order and each adjacency row in ascending order
// (silvan/src/Sp_sampler.cpp:116-140).  Its results depend on that order:
// the first scan item that reaches a node fixes the node's queue position,
// predecessor lists are appended in scan order, and meeting edges are
// collected in scan order.  Here the items of a level are numbered
// g = 0, 1, ... in exactly that order and processed in tiles of ascending g:
//   phase 1  every item reads the state of its neighbour y; every item that
//            reaches a node of the new level (unvisited, or joined earlier in
//            this level) records itself with atomicMin/atomicMax of
//            (g << 32 | x) (the first and the last predecessor), a count and
//            sigma += sigma(x) (a wrapping sum, order-free);
//   phase 2  after a barrier the items whose g equals their node's minimum are
//            the joining hits; they mark their node as visited and, with the
//            meeting items, are compacted in g order (warp ballots plus one
//            block scan), which appends new nodes to the queue and meeting
//            edges to the list in the reference order.
// A later tile can never lower a node's minimum below an earlier tile's g, so
// each tile is final once its own phase 1 is done.
//
// The backtrack needs pred(y)[t] with t = min(r mod sigma(y), |pred(y)| - 1)
// (Sp_sampler.cpp:241-265: the walk adds n_paths[v] == 1 per entry).  t == 0
// is the first hit, t == |pred|-1 the last hit; any other t is resolved by
// ranking the predecessors (reverse neighbours on the previous level of the
// same side) by their own queue order.
#include "sampler.cuh"

namespace silvan {

namespace {

constexpr int kItems = 4;        // scan items per lane per tile
constexpr int kMaxLevels = 256;  // levels per side with recorded bounds

// Per-CTA-size constants: BLOCK threads serve one sample.  Smaller CTAs put
// more samples in flight per SM (throughput on many short searches), larger
// ones put more threads on one wide level (the slowest sample of a round).
template <int BLOCK>
struct Shape {
    static constexpr int kWarps = BLOCK / 32;
    static constexpr int kTile = BLOCK * kItems;                    // scan items per tile
    static constexpr int kChunk = BLOCK * 4 < 2048 ? BLOCK * 4 : 2048;  // frontier nodes staged
    static constexpr int kPerThread = kChunk / BLOCK;
    static constexpr int kMinBlocks = 1024 / BLOCK;                 // 64 registers per thread
};

template <int BLOCK>
struct SamplerSmem {
    static constexpr int kWarps = Shape<BLOCK>::kWarps;
    static constexpr int kChunk = Shape<BLOCK>::kChunk;
    uint32_t f_node[kChunk];
    uint32_t f_off[kChunk];
    uint32_t f_pre[kChunk + 1];
    unsigned long long f_sig[kChunk];
    uint32_t warp_a[kItems * kWarps];  // per (item slot, warp): joins, then their offsets
    uint32_t warp_b[kItems * kWarps];  // per (item slot, warp): meeting edges, offsets
    uint32_t scan_tmp[kWarps + 1];
    unsigned long long wsum[kWarps];
    unsigned long long rec_base;
    uint32_t sum_new;
    uint32_t pred_hits;
    // sample state
    uint32_t sample;  // round-local index, or >= count when done
    uint32_t u, v, draw_base;
    uint32_t end_q;
    uint32_t start_u, end_u, start_v, end_v;
    uint32_t sum_u, sum_v, depth_u, depth_v;
    uint32_t nmeet, ntouched;
    unsigned long long vis;
    int32_t status;
    int32_t nonmono;
    unsigned long long W;
    uint32_t work;
    // queue segment of every BFS level: side (U = 0, V = 1), depth
    uint32_t lvl_lo[2][kMaxLevels];
    uint32_t lvl_hi[2][kMaxLevels];
    SegDesc seg;  // the segment of the sample in flight
};

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t draw32(uint64_t seed, uint32_t sample, uint32_t d) {
    return philox_lo32(seed, sample, kStreamSampler, d);
}

// x mod m for a 32-bit x and a non-zero 64-bit m: x itself when m >= 2^32.
__device__ __forceinline__ uint32_t mod_u64(uint32_t x, unsigned long long m) {
    return (m >> 32) ? x : x % (uint32_t)m;
}

// Exclusive block scan of one value per thread; returns the block total.
// tmp needs kWarps + 1 entries.
template <int BLOCK>
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t &excl, uint32_t *tmp) {
    constexpr int kWarps = Shape<BLOCK>::kWarps;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) tmp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < kWarps ? tmp[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kWarps) tmp[lane] = wi - w;
        if (lane == kWarps - 1) tmp[kWarps] = wi;
    }
    __syncthreads();
    excl = tmp[warp] + incl - v;
    const uint32_t total = tmp[kWarps];
    __syncthreads();
    return total;
}

__device__ __forceinline__ void rec_reset(NodeRec *r) {
    uint4 *p = reinterpret_cast<uint4 *>(r);
    p[0] = make_uint4(0u, 0u, 0u, 0u);                  // st, cnt, sigma
    p[1] = make_uint4(0xffffffffu, 0xffffffffu, 0u, 0u);  // first = ~0, last = 0
}

// Predecessor of rank t (queue order) of node a, 0 < t < cnt - 1.  The
// predecessors of a node at depth d are the nodes of level d-1 of its side
// whose row (in the expansion direction) contains it, in queue order.  Two
// equivalent searches, whichever reads less:
//   level scan: walk the level's queue segment, binary-search a in each row;
//   reverse scan: walk a's reverse row, keep the candidates on level d-1 and
//                 rank them by their own queue position (their first hit).
template <class Smem>
__device__ uint32_t middle_pred(const SegDesc &A, const Smem &s, const NodeRec *rec,
                                const uint32_t *queue, uint32_t a, uint32_t st_a, uint32_t t,
                                int32_t &status) {
    const uint32_t side = st_side(st_a);
    const uint32_t dprev = st_dist(st_a) - 1u;
    const uint32_t want = st_make(side, dprev);
    const uint32_t *roff = side == kSideU ? A.in_off : A.out_off;
    const uint32_t *radj = side == kSideU ? A.in_adj : A.out_adj;
    const uint32_t *foff = side == kSideU ? A.out_off : A.in_off;
    const uint32_t *fadj = side == kSideU ? A.out_adj : A.in_adj;
    const uint32_t rb = roff[a], re = roff[a + 1];
    if (dprev < (uint32_t)kMaxLevels) {
        const uint32_t lo = s.lvl_lo[side - 1][dprev], hi = s.lvl_hi[side - 1][dprev];
        if ((uint64_t)(hi - lo) * 24u < (uint64_t)(re - rb)) {
            uint32_t seen = 0;
            for (uint32_t i = lo; i < hi; i++) {
                const uint32_t x = __ldcg(&queue[i]);
                uint32_t l = foff[x], h = foff[x + 1];
                while (l < h) {  // first entry >= a
                    const uint32_t mid = (l + h) >> 1;
                    if (fadj[mid] < a) l = mid + 1;
                    else h = mid;
                }
                if (l < foff[x + 1] && fadj[l] == a) {
                    if (seen == t) return x;
                    seen++;
                }
            }
            status = SILVAN_E_STATE;
            return a;
        }
    }
    // reverse scan with a bounded buffer of the t+1 smallest keys
    constexpr uint32_t kBuf = 16;
    if (t < kBuf) {
        unsigned long long key[kBuf];
        uint32_t node[kBuf];
        uint32_t nb = 0;
        for (uint32_t k = rb; k < re; k++) {
            const uint32_t x = radj[k];
            if (__ldcg(&rec[x].st) != want) continue;
            const unsigned long long kx = __ldcg(&rec[x].first) >> 32;
            if (nb == t + 1 && kx >= key[t]) continue;
            uint32_t p = nb < t + 1 ? nb++ : t;
            while (p > 0 && key[p - 1] > kx) {
                key[p] = key[p - 1];
                node[p] = node[p - 1];
                p--;
            }
            key[p] = kx;
            node[p] = x;
        }
        if (nb == t + 1) return node[t];
        status = SILVAN_E_STATE;
        return a;
    }
    unsigned long long prev = 0;
    bool have_prev = false;
    uint32_t bx = a;
    for (uint32_t r = 0; r <= t; r++) {
        unsigned long long best = ~0ull;
        for (uint32_t k = rb; k < re; k++) {
            const uint32_t x = radj[k];
            if (__ldcg(&rec[x].st) != want) continue;
            const unsigned long long kx = __ldcg(&rec[x].first) >> 32;
            if ((!have_prev || kx > prev) && kx < best) {
                best = kx;
                bx = x;
            }
        }
        prev = best;
        have_prev = true;
    }
    return bx;
}

// Sigma-weighted predecessor of node a (cnt >= 2): the first predecessor in
// queue order whose running sum of sigma exceeds r, r = draw mod sigma(a).
// The predecessors are the reverse-direction neighbours on the previous level
// of a's side; their queue order is the order of their own first-hit keys, so
// they are taken one at a time by increasing key.
__device__ uint32_t weighted_pred(const SegDesc &A, const NodeRec *rec, uint32_t a,
                                  uint32_t st_a, uint32_t cnt, uint32_t r, int32_t &status) {
    const uint32_t side = st_side(st_a);
    const uint32_t want = st_make(side, st_dist(st_a) - 1u);
    const uint32_t *roff = side == kSideU ? A.in_off : A.out_off;
    const uint32_t *radj = side == kSideU ? A.in_adj : A.out_adj;
    const uint32_t rb = roff[a], re = roff[a + 1];
    unsigned long long acc = 0, prev = 0;
    bool have_prev = false;
    uint32_t last = a;
    for (uint32_t i = 0; i < cnt; i++) {
        unsigned long long best = ~0ull, bs = 0;
        uint32_t bx = a;
        for (uint32_t k = rb; k < re; k++) {
            const uint32_t x = radj[k];
            if (__ldcg(&rec[x].st) != want) continue;
            const unsigned long long kx = __ldcg(&rec[x].first) >> 32;
            if ((!have_prev || kx > prev) && kx < best) {
                best = kx;
                bx = x;
                bs = __ldcg(&rec[x].sigma);
            }
        }
        if (bx == a) {
            status = SILVAN_E_STATE;
            return a;
        }
        acc += bs;
        last = bx;
        if (acc > (unsigned long long)r) return bx;
        prev = best;
        have_prev = true;
    }
    return last;
}

// Expands one BFS level of `side` (silvan/src/Sp_sampler.cpp:89-143).
//
// The level is latency-bound on deep, narrow searches (a grid's ~200 levels
// of a few hundred nodes), so every phase first issues all of its
// independent global loads (read-only CSR through the non-coherent path, slot
// state through L2) and only then stores or issues atomics: a store between
// two loads would serialise them, because the compiler cannot prove that they
// do not alias.
template <int BLOCK>
__device__ void expand_level(const SegDesc &A, SamplerSmem<BLOCK> &s, NodeRec *rec,
                             uint32_t *queue, uint2 *meet, uint32_t side, uint32_t lo,
                             uint32_t hi, uint32_t depth) {
    constexpr int kWarps = Shape<BLOCK>::kWarps;
    constexpr int kTile = Shape<BLOCK>::kTile;
    constexpr int kChunk = Shape<BLOCK>::kChunk;
    constexpr int kPer = Shape<BLOCK>::kPerThread;
    const uint32_t *off = side == kSideU ? A.out_off : A.in_off;
    const uint32_t *adj = side == kSideU ? A.out_adj : A.in_adj;
    const uint32_t new_st = st_make(side, depth + 1u);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t gbase = 0;  // item number of the chunk's first item within the level
    uint32_t sum_local = 0;
    uint32_t hits_local = 0;
    for (uint32_t c0 = lo; c0 < hi; c0 += kChunk) {
        const uint32_t nc = min((uint32_t)kChunk, hi - c0);
        // stage the chunk: row starts, degrees (prefix), sigma
        uint32_t xq[kPer], o0[kPer], o1[kPer];
        unsigned long long sg[kPer];
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            xq[i] = p < nc ? __ldcg(&queue[c0 + p]) : 0u;
        }
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            o0[i] = o1[i] = 0;
            sg[i] = 0;
            if (p < nc) {
                o0[i] = __ldg(&off[xq[i]]);
                o1[i] = __ldg(&off[xq[i] + 1]);
                sg[i] = __ldcg(&rec[xq[i]].sigma);
            }
        }
        uint32_t tsum = 0;
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            if (p < nc) {
                s.f_node[p] = xq[i];
                s.f_off[p] = o0[i];
                s.f_sig[p] = sg[i];
            }
            tsum += o1[i] - o0[i];
        }
        uint32_t excl;
        uint32_t total = block_exclusive_scan<BLOCK>(tsum, excl, s.scan_tmp);
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            if (p < nc) s.f_pre[p] = excl;
            excl += o1[i] - o0[i];
        }
        if (threadIdx.x == 0) s.f_pre[nc] = total;
        __syncthreads();
        const uint32_t G = total;
        for (uint32_t t0 = 0; t0 < G; t0 += kTile) {
            // ---- phase 1 ------------------------------------------------------
            // item slot k of thread tid is item t0 + k * BLOCK + tid: a narrow
            // level spreads over every warp, and the item order is (k, warp, lane)
            uint32_t ys[kItems], xs[kItems], code[kItems], li[kItems];
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                const uint32_t it = t0 + (uint32_t)(k * BLOCK) + threadIdx.x;
                code[k] = 0;
                ys[k] = 0;
                xs[k] = 0;
                li[k] = 0;
                if (it < G) {
                    uint32_t l = 0, h = nc;
                    while (h - l > 1) {
                        const uint32_t mid = (l + h) >> 1;
                        if (s.f_pre[mid] <= it) l = mid;
                        else h = mid;
                    }
                    li[k] = l;
                    xs[k] = s.f_node[l];
                    ys[k] = __ldg(&adj[s.f_off[l] + (it - s.f_pre[l])]);
                    code[k] = 3;  // valid, state not read yet
                }
            }
            // the neighbour's state, and its row (needed only if it joins; loaded
            // now so that the join does not wait for it)
            uint32_t sty[kItems], dg[kItems];
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                sty[k] = code[k] ? __ldcg(&rec[ys[k]].st) : 0u;
                dg[k] = code[k] ? __ldg(&off[ys[k] + 1]) - __ldg(&off[ys[k]]) : 0u;
            }
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                if (!code[k]) continue;
                // unvisited, or joined earlier in this level: a new-level hit
                // (the joining hit marks the node in phase 2)
                if (sty[k] == 0u || sty[k] == new_st) code[k] = 1;
                else if (st_side(sty[k]) != side) code[k] = 2;
                else code[k] = 0;
            }
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                if (code[k] != 1) continue;
                const uint32_t it = t0 + (uint32_t)(k * BLOCK) + threadIdx.x;
                const unsigned long long key = ((unsigned long long)(gbase + it) << 32) | xs[k];
                NodeRec *r = &rec[ys[k]];
                atomicMin(reinterpret_cast<unsigned long long *>(&r->first), key);
                atomicMax(reinterpret_cast<unsigned long long *>(&r->last), key);
                atomicAdd(&r->cnt, 1u);
                atomicAdd(reinterpret_cast<unsigned long long *>(&r->sigma), s.f_sig[li[k]]);
            }
            __syncthreads();
            // ---- phase 2: ordered compaction of joins and meeting edges -------
            unsigned long long fv[kItems];
#pragma unroll
            for (int k = 0; k < kItems; k++)
                fv[k] = code[k] == 1
                            ? __ldcg(reinterpret_cast<const unsigned long long *>(&rec[ys[k]].first))
                            : 0ull;
            uint32_t rn[kItems], rm[kItems];
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                const uint32_t it = t0 + (uint32_t)(k * BLOCK) + threadIdx.x;
                if (code[k] == 1) {
                    hits_local++;
                    if ((uint32_t)(fv[k] >> 32) != gbase + it) code[k] = 0;
                }
            }
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                const uint32_t bn = __ballot_sync(0xffffffffu, code[k] == 1);
                const uint32_t bm = __ballot_sync(0xffffffffu, code[k] == 2);
                rn[k] = __popc(bn & lanemask_lt());
                rm[k] = __popc(bm & lanemask_lt());
                if (lane == 0) {
                    s.warp_a[k * kWarps + warp] = __popc(bn);
                    s.warp_b[k * kWarps + warp] = __popc(bm);
                }
            }
            __syncthreads();
            if (warp == 0) {
                // exclusive offsets over (k, warp) in item order; the tile's
                // bases; the queue and meeting-list ends advance here (the
                // next tile reads them only after its own phase-1 barrier)
                constexpr int kE = kItems * kWarps;
                constexpr int kPerLane = (kE + 31) / 32;
                uint32_t va[kPerLane], vb[kPerLane];
                uint32_t sa = 0, sb = 0;
#pragma unroll
                for (int i = 0; i < kPerLane; i++) {
                    const int e = lane * kPerLane + i;
                    va[i] = e < kE ? s.warp_a[e] : 0u;
                    vb[i] = e < kE ? s.warp_b[e] : 0u;
                    sa += va[i];
                    sb += vb[i];
                }
                uint32_t ia = sa, ib = sb;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t ta = __shfl_up_sync(0xffffffffu, ia, o);
                    const uint32_t tb = __shfl_up_sync(0xffffffffu, ib, o);
                    if (lane >= o) {
                        ia += ta;
                        ib += tb;
                    }
                }
                const uint32_t an = __shfl_sync(0xffffffffu, ia, 31);
                const uint32_t am = __shfl_sync(0xffffffffu, ib, 31);
                const uint32_t qb = s.end_q, mb0 = s.nmeet;
                __syncwarp();
                uint32_t ea = qb + ia - sa, eb = mb0 + ib - sb;
#pragma unroll
                for (int i = 0; i < kPerLane; i++) {
                    const int e = lane * kPerLane + i;
                    if (e < kE) {
                        s.warp_a[e] = ea;
                        s.warp_b[e] = eb;
                    }
                    ea += va[i];
                    eb += vb[i];
                }
                if (lane == 0) {
                    s.end_q = qb + an;
                    s.nmeet = min(mb0 + am, kMeetCap);
                    if (mb0 + am > kMeetCap && s.status == 0) s.status = SILVAN_E_CAPACITY;
                }
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                if (code[k] == 1) {
                    const uint32_t y = ys[k];
                    queue[s.warp_a[k * kWarps + warp] + rn[k]] = y;
                    rec[y].st = new_st;
                    sum_local += dg[k];
                } else if (code[k] == 2) {
                    const uint32_t pos = s.warp_b[k * kWarps + warp] + rm[k];
                    if (pos < kMeetCap) meet[pos] = make_uint2(xs[k], ys[k]);
                }
            }
        }
        if (threadIdx.x == 0) s.vis += G;
        gbase += G;
        __syncthreads();
    }
    // degree sum of the new level (u32, wrapping like the reference's counter)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum_local += __shfl_xor_sync(0xffffffffu, sum_local, o);
        hits_local += __shfl_xor_sync(0xffffffffu, hits_local, o);
    }
    if (lane == 0) {
        s.warp_a[warp] = sum_local;
        s.warp_b[warp] = hits_local;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t sn = 0, ph = 0;
        for (int w = 0; w < kWarps; w++) {
            sn += s.warp_a[w];
            ph += s.warp_b[w];
        }
        s.sum_new = sn;
        s.pred_hits += ph;
    }
    // the caller's thread 0 consumes sum_new before its next barrier
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, Shape<BLOCK>::kMinBlocks) sampler_kernel(SamplerLaunch L) {
    constexpr int kWarps = Shape<BLOCK>::kWarps;
    __shared__ SamplerSmem<BLOCK> s;
    const uint32_t slot = blockIdx.x;
    const uint64_t base = (uint64_t)slot * L.slots.stride;
    NodeRec *rec = L.slots.rec + base;
    uint32_t *queue = L.slots.queue + base;
    uint32_t *hits = L.slots.hits + base;
    uint32_t *touched = L.slots.touched + base;
    uint2 *meet = L.slots.meet + (uint64_t)slot * kMeetCap;
    uint64_t *mpre = L.slots.meet_pre + (uint64_t)slot * kMeetCap;
    const uint32_t total = L.hdr->total;
    const uint32_t nsegs = L.hdr->nsegs;
    const SegDesc &A = s.seg;

    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t w = atomicAdd(&L.hdr->work, 1u);
            s.work = w;
            if (w < total) {
                // segment owning work index w: last segment with base <= w
                uint32_t l = 0, h = nsegs;
                while (h - l > 1) {
                    const uint32_t mid = (l + h) >> 1;
                    if (L.segs[mid].base <= w) l = mid;
                    else h = mid;
                }
                s.sample = l;
            }
        }
        __syncthreads();
        if (s.work >= total) break;
        {
            const uint32_t *src = reinterpret_cast<const uint32_t *>(&L.segs[s.sample]);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&s.seg);
            for (uint32_t i = threadIdx.x; i < sizeof(SegDesc) / 4; i += BLOCK)
                dst[i] = src[i];
        }
        __syncthreads();
        const uint32_t sl = s.work - A.base;
        const uint32_t gidx = A.first_sample + sl;
        const long long t_sample0 = clock64();

        // ---- endpoints (Sp_sampler.cpp:46,58-60) and void test (:62-74) -------
        if (threadIdx.x == 0) {
            uint32_t d = 0;
            uint32_t v = draw32(A.seed, gidx, d++) % A.n;
            uint32_t u = draw32(A.seed, gidx, d++) % A.n;
            while (u == v) v = draw32(A.seed, gidx, d++) % A.n;
            s.u = u;
            s.v = v;
            s.draw_base = d;
            s.status = 0;
            s.vis = 0;
            s.nmeet = 0;
            s.ntouched = 0;
            s.nonmono = 0;
            s.pred_hits = 0;
        }
        __syncthreads();
        const uint32_t u = s.u, v = s.v;
        const bool void_cc = A.directed ? (A.cc[u] < A.cc[v]) : (A.cc[u] != A.cc[v]);
        if (void_cc) {
            if (threadIdx.x == 0) {
                A.out_pl[sl] = 0;
                A.out_np[sl] = 0;
                A.out_vis[sl] = 0;
                A.out_status[sl] = 0;
                A.out_ball[sl] = 0;
                A.out_pred[sl] = 0;
                const unsigned long long dc = (unsigned long long)(clock64() - t_sample0);
                atomicAdd(&L.hdr->cycles, dc);
                atomicMax(&L.hdr->max_cycles, dc);
            }
            __syncthreads();
            continue;
        }
        if (threadIdx.x == 0) {
            rec[u].st = st_make(kSideU, 0);
            rec[u].sigma = 1;
            rec[v].st = st_make(kSideV, 0);
            rec[v].sigma = 1;
            queue[0] = u;
            queue[1] = v;
            s.lvl_lo[0][0] = 0;
            s.lvl_hi[0][0] = 1;
            s.lvl_lo[1][0] = 1;
            s.lvl_hi[1][0] = 2;
            s.end_q = 2;
            s.start_u = 0;
            s.end_u = 1;
            s.start_v = 1;
            s.end_v = 2;
            s.sum_u = 0;
            s.sum_v = 0;
            s.depth_u = 0;
            s.depth_v = 0;
        }
        __syncthreads();

        // ---- balanced bidirectional BFS (:89-144) ------------------------------
        uint32_t exp_side = kSideU;
        for (;;) {
            const bool side_u = s.sum_u <= s.sum_v;
            exp_side = side_u ? kSideU : kSideV;
            const uint32_t lo = side_u ? s.start_u : s.start_v;
            const uint32_t hi = side_u ? s.end_u : s.end_v;
            const uint32_t depth = side_u ? s.depth_u : s.depth_v;
            const uint32_t q0 = s.end_q;
            __syncthreads();
            expand_level(A, s, rec, queue, meet, exp_side, lo, hi, depth);
            if (threadIdx.x == 0) {
                if (depth + 1 < (uint32_t)kMaxLevels) {
                    s.lvl_lo[side_u ? 0 : 1][depth + 1] = q0;
                    s.lvl_hi[side_u ? 0 : 1][depth + 1] = s.end_q;
                }
                if (side_u) {
                    s.start_u = q0;
                    s.end_u = s.end_q;
                    s.sum_u = s.sum_new;
                    s.depth_u = depth + 1;
                } else {
                    s.start_v = q0;
                    s.end_v = s.end_q;
                    s.sum_v = s.sum_new;
                    s.depth_v = depth + 1;
                }
            }
            __syncthreads();
            if (s.nmeet > 0 || s.sum_new == 0 || s.status != 0) break;
        }

        // ---- meeting-edge weights and the number of paths (:159-170) ----------
        const uint32_t nm = s.nmeet;
        int32_t np = 0, pl = 0;
        if (nm > 0 && s.status == 0) {
            // inclusive prefix of sigma(x) * sigma(y), wrapping; non-decreasing
            // exactly when the 64-bit sum never wrapped
            unsigned long long carry = 0;
            for (uint32_t c0 = 0; c0 < nm; c0 += BLOCK) {
                uint32_t i = c0 + threadIdx.x;
                unsigned long long p = 0;
                if (i < nm) {
                    uint2 e = __ldcg(&meet[i]);
                    p = (unsigned long long)__ldcg(&rec[e.x].sigma) *
                        (unsigned long long)__ldcg(&rec[e.y].sigma);
                }
                // block inclusive scan of 64-bit values (wrapping)
                unsigned long long incl = p;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
                    if ((threadIdx.x & 31) >= o) incl += t;
                }
                if ((threadIdx.x & 31) == 31) s.wsum[threadIdx.x >> 5] = incl;
                __syncthreads();
                unsigned long long woff = 0;
                for (int w = 0; w < (int)(threadIdx.x >> 5); w++) woff += s.wsum[w];
                incl += woff + carry;
                if (i < nm) mpre[i] = incl;
                __syncthreads();
                unsigned long long tot = 0;
                for (int w = 0; w < kWarps; w++) tot += s.wsum[w];
                carry += tot;
                __syncthreads();
            }
            __syncthreads();
            for (uint32_t i = 1 + threadIdx.x; i < nm; i += BLOCK)
                if (__ldcg(&mpre[i]) < __ldcg(&mpre[i - 1])) s.nonmono = 1;
            if (threadIdx.x == 0) s.W = carry;
            __syncthreads();
            const unsigned long long W = s.W;
            const uint2 e0 = __ldcg(&meet[0]);
            const uint32_t L = st_dist(__ldcg(&rec[e0.x].st)) + st_dist(__ldcg(&rec[e0.y].st));
            if (W == 0ull) {
                if (threadIdx.x == 0) s.status = SILVAN_E_OVERFLOW;
            } else {
                np = 1;
                if (A.alpha > 0. && W > 1ull) {
                    double t = A.alpha * (double)W;
                    np = (t >= 2147483648.0) ? INT32_MIN : (int32_t)t;
                }
                pl = np >= 1 ? (int32_t)L : 0;
                if (pl > 0 && (uint32_t)np > A.np_cap) {
                    if (threadIdx.x == 0) s.status = SILVAN_E_NP_CAP;
                } else if (pl > 0 &&
                           (uint64_t)s.draw_base + (uint64_t)np * (1ull + L) > 0xffffffffull) {
                    if (threadIdx.x == 0) s.status = SILVAN_E_NP_CAP;
                }
            }
            __syncthreads();
            // ---- paths (:172-197) and backtracks (:241-265) ------------------
            if (s.status == 0 && pl > 0) {
                const bool mono = s.nonmono == 0;
                for (uint32_t j = threadIdx.x; j < (uint32_t)np; j += BLOCK) {
                    uint32_t d = s.draw_base + j * (1u + L);
                    const uint32_t r = mod_u64(draw32(A.seed, gidx, d++), W);
                    uint32_t ei;
                    if (mono) {  // first i with prefix > r
                        uint32_t l = 0, h = nm - 1;
                        while (l < h) {
                            uint32_t mid = (l + h) >> 1;
                            if (__ldcg(&mpre[mid]) > r) h = mid;
                            else l = mid + 1;
                        }
                        ei = l;
                    } else {
                        ei = 0;
                        while (ei < nm && !(__ldcg(&mpre[ei]) > (unsigned long long)r)) ei++;
                        if (ei >= nm) ei = nm - 1;
                    }
                    const uint2 e = __ldcg(&meet[ei]);
                    uint32_t starts[2] = {e.x, e.y};
                    for (int h2 = 0; h2 < 2; h2++) {
                        uint32_t a = starts[h2];
                        // the hit count of the previous node is checked after
                        // the next record load has been issued
                        uint32_t pend = 0xffffffffu, pend_old = 1u;
                        for (uint32_t steps = 0;; steps++) {
                            // every step moves one level closer to a root, so a
                            // walk longer than L or an id outside the graph is an
                            // internal inconsistency: report it, never follow it
                            if (a >= A.n || steps > L) {
                                s.status = SILVAN_E_STATE;
                                break;
                            }
                            // the whole record (one sector) in one load
                            const uint4 r0 = __ldcg(reinterpret_cast<const uint4 *>(&rec[a]));
                            const uint4 r1 = __ldcg(reinterpret_cast<const uint4 *>(&rec[a]) + 1);
                            if (pend != 0xffffffffu && pend_old == 0u) {
                                const uint32_t ti = atomicAdd(&s.ntouched, 1u);
                                touched[ti] = pend;
                            }
                            pend = 0xffffffffu;
                            const uint32_t sta = r0.x;
                            if (st_dist(sta) == 0) break;  // a is u or v
                            pend_old = atomicAdd(&hits[a], 1u);
                            pend = a;
                            const unsigned long long sg =
                                (unsigned long long)r0.z | ((unsigned long long)r0.w << 32);
                            uint32_t rr = draw32(A.seed, gidx, d++);
                            if (sg == 0ull) {
                                s.status = SILVAN_E_OVERFLOW;
                                break;
                            }
                            rr = mod_u64(rr, sg);
                            const uint32_t c = r0.y;
                            const uint32_t t = min(rr, c - 1u);
                            if (A.weighted && c > 1u) {
                                int32_t e = 0;
                                a = weighted_pred(A, rec, a, sta, c, rr, e);
                                if (e) {
                                    s.status = e;
                                    break;
                                }
                            } else if (t == 0) {
                                a = r1.x;  // low word of first: the joining predecessor
                            } else if (t == c - 1u) {
                                a = r1.z;  // low word of last
                            } else {
                                int32_t e = 0;
                                a = middle_pred(A, s, rec, queue, a, sta, t, e);
                                if (e) {
                                    s.status = e;
                                    break;
                                }
                            }
                        }
                        if (pend != 0xffffffffu && pend_old == 0u) {
                            const uint32_t ti = atomicAdd(&s.ntouched, 1u);
                            touched[ti] = pend;
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (s.status != 0) {
            np = 0;
            pl = 0;
        }

        // ---- emit the path map, restore the slot ---------------------------------
        const uint32_t nt = s.ntouched;
        if (threadIdx.x == 0) {
            unsigned long long b = 0;
            if (nt > 0 && s.status == 0) {
                b = atomicAdd(A.rec_cursor, (unsigned long long)nt);
                if (b + nt > A.rec_cap) s.status = SILVAN_E_CAPACITY;
            }
            s.rec_base = b;
        }
        __syncthreads();
        const unsigned long long rb = s.rec_base;
        const bool emit = s.status == 0;
        for (uint32_t i0 = threadIdx.x; i0 < nt; i0 += 4 * BLOCK) {
            uint32_t a4[4], c4[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t i = i0 + j * BLOCK;
                a4[j] = i < nt ? __ldcg(&touched[i]) : 0u;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) c4[j] = i0 + j * BLOCK < nt ? __ldcg(&hits[a4[j]]) : 0u;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t i = i0 + j * BLOCK;
                if (i >= nt) continue;
                if (emit) {
                    PathRec pr;
                    pr.node = a4[j];
                    pr.sample = sl;
                    pr.count = c4[j];
                    A.recs[rb + i] = pr;
                }
                hits[a4[j]] = 0;
            }
        }
        const uint32_t eq = s.end_q;
        for (uint32_t i0 = threadIdx.x; i0 < eq; i0 += 4 * BLOCK) {
            uint32_t q4[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t i = i0 + j * BLOCK;
                q4[j] = i < eq ? __ldcg(&queue[i]) : 0xffffffffu;
            }
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (q4[j] != 0xffffffffu) rec_reset(&rec[q4[j]]);
        }
        if (threadIdx.x == 0) {
            A.out_pl[sl] = s.status == 0 ? pl : 0;
            A.out_np[sl] = s.status == 0 ? np : 0;
            A.out_vis[sl] = s.vis;
            A.out_status[sl] = s.status;
            A.out_ball[sl] = s.end_q;
            A.out_pred[sl] = s.pred_hits;
            const unsigned long long dc = (unsigned long long)(clock64() - t_sample0);
            atomicAdd(&L.hdr->cycles, dc);
            atomicMax(&L.hdr->max_cycles, dc);
        }
        __syncthreads();
    }
}

__global__ void round_begin_kernel(SamplerLaunch L, uint32_t max_segs) {
    const uint32_t ns = min(L.hdr->nsegs, max_segs);
    for (uint32_t i = threadIdx.x; i < ns; i += blockDim.x) *L.segs[i].rec_cursor = 0ull;
    if (threadIdx.x == 0) {
        L.hdr->work = 0;
        L.hdr->cycles = 0;
        L.hdr->max_cycles = 0;
    }
}

__global__ void init_slots_kernel(NodeRec *rec, uint32_t *hits, uint64_t total) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        rec_reset(&rec[i]);
        hits[i] = 0;
    }
}

}  // namespace

cudaError_t sampler_init_slots(NodeRec *rec, uint32_t *hits, uint64_t total_nodes,
                               cudaStream_t stream) {
    init_slots_kernel<<<1184, 256, 0, stream>>>(rec, hits, total_nodes);
    return cudaGetLastError();
}

cudaError_t sampler_round_begin(const SamplerLaunch &L, uint32_t max_segs, cudaStream_t stream) {
    round_begin_kernel<<<1, 256, 0, stream>>>(L, max_segs);
    return cudaGetLastError();
}

cudaError_t sampler_launch(const SamplerLaunch &L, uint32_t grid, cudaStream_t stream, int block) {
    if (grid == 0) return cudaSuccess;
    switch (block) {
    case 128: sampler_kernel<128><<<grid, 128, 0, stream>>>(L); break;
    case 256: sampler_kernel<256><<<grid, 256, 0, stream>>>(L); break;
    case 512: sampler_kernel<512><<<grid, 512, 0, stream>>>(L); break;
    case 1024: sampler_kernel<1024><<<grid, 1024, 0, stream>>>(L); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int sampler_max_ctas_per_sm(int block) {
    int n = 0;
    switch (block) {
    case 128: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sampler_kernel<128>, 128, 0); break;
    case 256: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sampler_kernel<256>, 256, 0); break;
    case 512: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sampler_kernel<512>, 512, 0); break;
    case 1024: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sampler_kernel<1024>, 1024, 0); break;
    default: break;
    }
    return n;
}

}  // namespace silvan
