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
// each tile is final once its own phase 1 is done.  A wide level may instead
// be expanded by several CTAs, tile by tile with the same numbering (the help
// board, below).
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
// Samples a CTA takes from the round at once while many are left; one
// thread each draws the endpoints and runs the void test, so the void
// samples (most of them on sparse directed graphs) cost a fraction of a
// sample each.  Near the end of a round the CTAs take one at a time.
constexpr uint32_t kScreen = 8;
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
    // help board
    AssistLevel lvl;   // the level this CTA expands with others
    int32_t a_entry;   // entry owned or helped; -1 none, -2 leave, -3 a sample
    uint32_t a_state;  // state of the owned entry while it is set up
    uint32_t a_tile;   // the tile this CTA took
    uint32_t a_ok;     // the tile's waits ended
    uint32_t a_drained, a_polls, a_nap;  // no sample left; board polls since; next nap (ns)
    uint32_t a_spin;    // polls of a bounded wait (RoundHeader::wait_polls)
    uint32_t a_leave;   // a shared level of this CTA's sample failed: take no more samples
    // samples taken from the round in a chunk and screened in parallel: the
    // void ones are finished at once, the others wait here
    uint32_t pend_w[kScreen];
    uint32_t pend_n, pend_i, scr_w0, scr_v;
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

// The neutral record (st, cnt, sigma = 0; first = ~0; last = 0) in one
// 32-byte store: a node record is one sector, written by one transaction.
__device__ __forceinline__ void rec_reset(NodeRec *r) {
    asm volatile("st.global.v8.b32 [%0], {%1, %1, %1, %1, %2, %2, %1, %1};" ::"l"(r), "r"(0u),
                 "r"(0xffffffffu)
                 : "memory");
}

// A whole record in one 32-byte store.
__device__ __forceinline__ void rec_store(NodeRec *r, uint4 lo, uint4 hi) {
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(r), "r"(lo.x),
                 "r"(lo.y), "r"(lo.z), "r"(lo.w), "r"(hi.x), "r"(hi.y), "r"(hi.z), "r"(hi.w)
                 : "memory");
}

// A whole record in one 32-byte load through L2 (the slot is written by this
// CTA and, for shared levels, by others): words 0-3 and 4-7.
__device__ __forceinline__ void rec_load(const NodeRec *r, uint4 &lo, uint4 &hi) {
    asm volatile("ld.global.cg.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(lo.x), "=r"(lo.y), "=r"(lo.z), "=r"(lo.w), "=r"(hi.x), "=r"(hi.y),
                   "=r"(hi.z), "=r"(hi.w)
                 : "l"(r)
                 : "memory");
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
    const uint2 *rrows = side == kSideU ? A.in_rows : A.out_rows;
    const uint32_t *radj = side == kSideU ? A.in_adj : A.out_adj;
    const uint2 *frows = side == kSideU ? A.out_rows : A.in_rows;
    const uint32_t *fadj = side == kSideU ? A.out_adj : A.in_adj;
    const uint2 rr = rrows[a];
    const uint32_t rb = rr.x, re = rr.y;
    if (dprev < (uint32_t)kMaxLevels) {
        const uint32_t lo = s.lvl_lo[side - 1][dprev], hi = s.lvl_hi[side - 1][dprev];
        if ((uint64_t)(hi - lo) * 24u < (uint64_t)(re - rb)) {
            uint32_t seen = 0;
            for (uint32_t i = lo; i < hi; i++) {
                const uint32_t x = __ldcg(&queue[i]);
                const uint2 fr = frows[x];
                uint32_t l = fr.x, h = fr.y;
                while (l < h) {  // first entry >= a
                    const uint32_t mid = (l + h) >> 1;
                    if (fadj[mid] < a) l = mid + 1;
                    else h = mid;
                }
                if (l < fr.y && fadj[l] == a) {
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
    const uint2 rr = (side == kSideU ? A.in_rows : A.out_rows)[a];
    const uint32_t *radj = side == kSideU ? A.in_adj : A.out_adj;
    const uint32_t rb = rr.x, re = rr.y;
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
    const uint2 *rows = side == kSideU ? A.out_rows : A.in_rows;
    const uint32_t *adj = side == kSideU ? A.out_adj : A.in_adj;
    const uint32_t new_st = st_make(side, depth + 1u);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t gbase = 0;  // item number of the chunk's first item within the level
    uint32_t sum_local = 0;
    uint32_t hits_local = 0;
    // ends of the queue and of the meeting list, advanced tile by tile in
    // every thread alike (thread 0 stores them when the level is done)
    uint32_t qend = s.end_q, mend = s.nmeet;
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
                const uint2 r = __ldg(&rows[xq[i]]);
                o0[i] = r.x;
                o1[i] = r.y;
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
                const uint2 r = code[k] ? __ldg(&rows[ys[k]]) : make_uint2(0u, 0u);
                dg[k] = r.y - r.x;
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
            // Phase 1 records only the hit count and the smallest key.  Most
            // new nodes of a level have a single hit (about 1.2 hits per node
            // on R-MAT); their whole record is then written by the joining
            // hit with one store in phase 2, and only nodes with several hits
            // get the sigma and last-key atomics.  The tiles of a level run
            // one after another on this CTA, separated by a barrier after
            // each tile's stores, so a later tile's hits find the record
            // complete and add to it.
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                if (code[k] != 1) continue;
                const uint32_t it = t0 + (uint32_t)(k * BLOCK) + threadIdx.x;
                const unsigned long long key = ((unsigned long long)(gbase + it) << 32) | xs[k];
                NodeRec *r = &rec[ys[k]];
                atomicMin(reinterpret_cast<unsigned long long *>(&r->first), key);
                atomicAdd(&r->cnt, 1u);
            }
            __syncthreads();
            // ---- phase 2: ordered compaction of joins and meeting edges -------
            uint32_t single = 0;  // bit k: item k is the node's only hit so far
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                if (code[k] != 1) continue;
                uint4 lo4, hi4;
                rec_load(&rec[ys[k]], lo4, hi4);
                const uint32_t it = t0 + (uint32_t)(k * BLOCK) + threadIdx.x;
                const unsigned long long key = ((unsigned long long)(gbase + it) << 32) | xs[k];
                hits_local++;
                if (lo4.y > 1u) {  // several hits: sigma and the last key by atomics
                    NodeRec *r = &rec[ys[k]];
                    atomicMax(reinterpret_cast<unsigned long long *>(&r->last), key);
                    atomicAdd(reinterpret_cast<unsigned long long *>(&r->sigma), s.f_sig[li[k]]);
                } else {
                    single |= 1u << k;
                }
                if (hi4.y != gbase + it) code[k] = 0;  // not the joining hit
            }
            uint32_t rn[kItems], rm[kItems];
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
            // Every warp turns the counts into exclusive offsets over
            // (k, warp) in item order (the same sums in every warp) and picks
            // its own kItems of them by shuffles; no second barrier.  The next
            // tile writes the counts again only after its own phase-1
            // barrier, which every warp reaches after reading these.
            uint32_t oa[kItems], ob[kItems];
            {
                constexpr int kE = kItems * kWarps;
                constexpr int kPerLane = (kE + 31) / 32;
                uint32_t pa[kPerLane], pb[kPerLane];
                uint32_t sa = 0, sb = 0;
#pragma unroll
                for (int i = 0; i < kPerLane; i++) {
                    const int e = lane * kPerLane + i;
                    pa[i] = e < kE ? s.warp_a[e] : 0u;
                    pb[i] = e < kE ? s.warp_b[e] : 0u;
                    sa += pa[i];
                    sb += pb[i];
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
                // this lane's entries: counts -> exclusive offsets
                uint32_t ea = qend + ia - sa, eb = mend + ib - sb;
#pragma unroll
                for (int i = 0; i < kPerLane; i++) {
                    const uint32_t ca = pa[i], cb = pb[i];
                    pa[i] = ea;
                    pb[i] = eb;
                    ea += ca;
                    eb += cb;
                }
#pragma unroll
                for (int k = 0; k < kItems; k++) {
                    const int e = k * kWarps + warp;
                    const int owner = e / kPerLane, sub = e % kPerLane;
                    uint32_t va = pa[0], vb = pb[0];
#pragma unroll
                    for (int i = 1; i < kPerLane; i++)
                        if (sub == i) {
                            va = pa[i];
                            vb = pb[i];
                        }
                    oa[k] = __shfl_sync(0xffffffffu, va, owner);
                    ob[k] = __shfl_sync(0xffffffffu, vb, owner);
                }
                if (threadIdx.x == 0 && mend + am > kMeetCap && s.status == 0)
                    s.status = SILVAN_E_CAPACITY;
                qend += an;
                mend = min(mend + am, kMeetCap);
            }
#pragma unroll
            for (int k = 0; k < kItems; k++) {
                if (code[k] == 1) {
                    const uint32_t y = ys[k];
                    queue[oa[k] + rn[k]] = y;
                    if (single & (1u << k)) {
                        // the only hit: st, cnt = 1, sigma, first = last = key
                        const uint32_t it = t0 + (uint32_t)(k * BLOCK) + threadIdx.x;
                        const unsigned long long sg = s.f_sig[li[k]];
                        rec_store(&rec[y], make_uint4(new_st, 1u, (uint32_t)sg, (uint32_t)(sg >> 32)),
                                  make_uint4(xs[k], gbase + it, xs[k], gbase + it));
                    } else {
                        rec[y].st = new_st;
                    }
                    sum_local += dg[k];
                } else if (code[k] == 2) {
                    const uint32_t pos = ob[k] + rm[k];
                    if (pos < kMeetCap) meet[pos] = make_uint2(xs[k], ys[k]);
                }
            }
            // A single-hit record is written whole by its joining hit; a hit
            // of the next tile on the same node must find it written and add
            // to it, not be overwritten by it (the chunk's last tile has the
            // barrier below).
            if (t0 + (uint32_t)kTile < G) __syncthreads();
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
        s.end_q = qend;
        s.nmeet = mend;
    }
    // the caller's thread 0 consumes sum_new and the ends before its next barrier
}

// ---------------------------------------------------------------------------
// Wide levels expanded by several CTAs (the help board)
//
// A launch lasts about as long as its slowest sample, and the slowest samples
// spend most of their time in one or two wide levels (hub rows, ~10^5
// entries) on one CTA.  Such a level is posted on the board instead: its
// owner writes the frontier's item prefix and a table of tiles (at most kTile
// items inside one chunk of kChunk frontier nodes), and every CTA that joins,
// the owner included, takes the next tile in order and runs expand_level's
// two phases on it.  Two decoupled look-backs over the tiles stand in for the
// one-CTA tile order:
//   * after its phase 1 a tile waits until the phase 1 of every earlier tile
//     is done (a later tile cannot lower a minimum below its own items, so
//     its joining hits are then final);
//   * its joins and meeting edges go to the offsets summed over the earlier
//     tiles, in item order within the tile.
// The items, keys, joins and append order are those of expand_level, so the
// level's result is bit-identical.  Tiles are taken in order and no tile
// waits for a later one, so every wait ends; each is bounded all the same
// (RoundHeader::wait_polls polls): a wait that gives up marks the level
// failed (the sample reports SILVAN_E_TIMEOUT) and the tile skips its
// writes.  Records that the failed level touched may then be left
// non-neutral, and helpers may still be writing to them, so the owner's CTA
// takes no further sample in the launch and the host re-initialises the
// slots before the next one.
// ---------------------------------------------------------------------------
constexpr uint32_t kAssistPolls = 1u << 18;  // board polls of a CTA without samples
constexpr unsigned long long kCntMask = (1ull << 31) - 1u;

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Look-back word of a tile's append counts: state (1 own counts, 2 inclusive
// prefix), joins, meeting edges (each saturated to 31 bits).
__device__ __forceinline__ unsigned long long cnt_word(uint32_t state, unsigned long long j,
                                                       unsigned long long m) {
    return ((unsigned long long)state << 62) | (min(j, kCntMask) << 31) | min(m, kCntMask);
}

// Thread 0: waits until *p == 0 (false: gave up).
__device__ bool wait_zero(const uint32_t *p, uint32_t limit) {
    for (uint32_t i = 0; i < limit; i++) {
        if (ld_acquire_u32(p) == 0u) return true;
        __nanosleep(128);
    }
    return false;
}

// Thread 0: waits until *p >= v (false: gave up).
__device__ bool wait_at_least(const uint32_t *p, uint32_t v, uint32_t limit) {
    for (uint32_t i = 0; i < limit; i++) {
        if (ld_acquire_u32(p) >= v) return true;
        __nanosleep(128);
    }
    return false;
}

// Warp 0: waits until the phase 1 of every tile before t is done.  hit_flag
// of a tile is 1 once its own hits are recorded and 2 once those of every
// tile up to it are; the warp reads 32 predecessors at a time.
__device__ bool lookback_hits(const uint32_t *hit_flag, uint32_t t, uint32_t limit) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t j = t;
    if (j == 0) return true;
    for (uint32_t spin = 0; spin < limit;) {
        if (j == 0) return true;
        const uint32_t f = lane < j ? ld_acquire_u32(&hit_flag[j - 1 - lane]) : 2u;
        const uint32_t m2 = __ballot_sync(0xffffffffu, f == 2u);
        const uint32_t m0 = __ballot_sync(0xffffffffu, f == 0u);
        if (m2) {
            if ((m0 & ((m2 & (0u - m2)) - 1u)) == 0u) return true;
        } else if (m0 == 0u) {
            j -= 32u;  // j > 32 here: lanes at or past j read as 2
            continue;
        }
        __nanosleep(64);
        spin++;
    }
    return false;
}

// Warp 0: sums of the joins and meeting edges of the tiles before t (the
// decoupled look-back of a single-pass scan).  The same in every lane.
__device__ bool lookback_counts(const unsigned long long *cnt_flag, uint32_t t,
                                unsigned long long &ej, unsigned long long &em, uint32_t limit) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t j = t;
    ej = em = 0;
    if (j == 0) return true;
    for (uint32_t spin = 0; spin < limit;) {
        if (j == 0) return true;
        const unsigned long long w =
            lane < j ? ld_acquire_u64(&cnt_flag[j - 1 - lane]) : cnt_word(2u, 0, 0);
        const uint32_t st = (uint32_t)(w >> 62);
        const uint32_t m2 = __ballot_sync(0xffffffffu, st == 2u);
        const uint32_t m0 = __ballot_sync(0xffffffffu, st == 0u);
        uint32_t take = 0xffffffffu;
        if (m2) {
            const uint32_t first = m2 & (0u - m2);
            take = first | (first - 1u);
        }
        if (m0 & take) {  // a tile on the way has not counted yet
            __nanosleep(64);
            spin++;
            continue;
        }
        unsigned long long vj = ((take >> lane) & 1u) ? (w >> 31) & kCntMask : 0ull;
        unsigned long long vm = ((take >> lane) & 1u) ? w & kCntMask : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            vj += __shfl_xor_sync(0xffffffffu, vj, o);
            vm += __shfl_xor_sync(0xffffffffu, vm, o);
        }
        ej += vj;
        em += vm;
        if (m2) return true;
        j -= 32u;
    }
    return false;
}

// Thread 0: copies an open entry's level description (through L2: another
// SM wrote it).
__device__ void load_level(AssistLevel &dst, const AssistLevel *src) {
    const uint32_t *a = reinterpret_cast<const uint32_t *>(src);
    uint32_t *b = reinterpret_cast<uint32_t *>(&dst);
    for (uint32_t i = 0; i < sizeof(AssistLevel) / 4; i++) b[i] = __ldcg(a + i);
}

// Thread 0: takes a free entry for this CTA's level (-1: none free).
__device__ int32_t acquire_entry(const AssistBoard &B, uint32_t from, uint32_t &st_out) {
    for (uint32_t i = 0; i < kAssistEntries; i++) {
        const uint32_t e = (from + i) % kAssistEntries;
        const uint32_t st = ld_acquire_u32(&B.entries[e].state);
        if ((st & 3u) != 0u) continue;
        if (atomicCAS(&B.entries[e].state, st, st | 1u) == st) {
            st_out = st | 1u;
            return (int32_t)e;
        }
    }
    return -1;
}

// Thread 0: enters an open entry with tiles left, copying its level into
// s.lvl (-1: none).  The entry count `inside` is raised before the state is
// read again, so the owner either sees this helper or the helper sees the
// entry closing and leaves.
template <int BLOCK>
__device__ __noinline__ int32_t join_entry(const SamplerLaunch &L, SamplerSmem<BLOCK> &s,
                                           uint32_t from) {
    const uint32_t mask = ld_acquire_u32(&L.hdr->open_mask);
    if (!mask) return -1;
    for (uint32_t i = 0; i < kAssistEntries; i++) {
        const uint32_t e = (from + i) % kAssistEntries;
        if (!(mask & (1u << e))) continue;
        AssistEntry *E = L.assist.entries + e;
        const uint32_t st = ld_acquire_u32(&E->state);
        if ((st & 3u) != 2u) continue;
        if (ld_acquire_u32(&E->claim) >= ld_acquire_u32(&E->ntiles)) continue;
        atomicAdd(&E->inside, 1u);
        __threadfence();
        if (ld_acquire_u32(&E->state) != st) {
            atomicSub(&E->inside, 1u);
            continue;
        }
        load_level(s.lvl, &E->lvl);
        return (int32_t)e;
    }
    return -1;
}

// Thread 0, before a level of the sample in flight: takes a board entry for
// it when it is wide (-1: expand it alone).  The level's items are the degree
// sum of its frontier: the side's sum for depth >= 1, the root's degree at 0.
template <int BLOCK>
__device__ __forceinline__ int32_t post_level(const SamplerLaunch &L, SamplerSmem<BLOCK> &s,
                                           bool side_u, uint32_t lo, uint32_t hi,
                                           uint32_t depth) {
    const SegDesc &A = s.seg;
    const uint2 *drows = side_u ? A.out_rows : A.in_rows;
    const uint32_t x0 = side_u ? s.u : s.v;
    const uint2 r0 = drows[x0];
    const uint32_t items = depth == 0 ? r0.y - r0.x : (side_u ? s.sum_u : s.sum_v);
    const uint32_t F = hi - lo;
    // Default threshold: 32 tiles while the round still has samples to hand
    // out, 16 tiles once every sample is taken (on R-MAT scale 20, over 60
    // seeds: 16 and 24 tiles alike, 8 tiles 5 % longer, 4 tiles 7 %, 2 tiles
    // 10 %; eight tiles while samples remain 5 % longer).  While samples remain, every
    // CTA is busy with its own and helps only between samples, and a shared
    // tile costs more than one expanded alone (the look-backs and the tile
    // table), so only levels long enough to become the launch's tail are
    // shared; once the round is drained, the CTAs without samples are idle
    // and the last samples' levels are what the launch waits for.
    uint32_t thr = A.assist_items;
    if (thr == kAssistItemsAuto) {
        const bool draining = ld_acquire_u32(&L.hdr->work) >= L.hdr->total;
        thr = (draining ? 16u : 32u) * (uint32_t)Shape<BLOCK>::kTile;
    }
    if (items < thr || F > L.assist.node_cap ||
        (uint64_t)items / Shape<BLOCK>::kTile + F / Shape<BLOCK>::kChunk + 2u > L.assist.tile_cap)
        return -1;
    return acquire_entry(L.assist, blockIdx.x, s.a_state);
}

// Tile t of entry e's level: expand_level's two phases on the tile's items.
template <int BLOCK>
__device__ void assist_tile(SamplerSmem<BLOCK> &s, const AssistBoard &B, uint32_t e, uint32_t t) {
    constexpr int kWarps = Shape<BLOCK>::kWarps;
    constexpr int kPer = Shape<BLOCK>::kPerThread;
    const AssistLevel &V = s.lvl;
    AssistEntry *E = B.entries + e;
    const uint64_t tb = (uint64_t)e * B.tile_cap;
    const uint32_t *pre = B.pre + (uint64_t)e * (B.node_cap + 1u);
    const uint32_t *rs = B.rs + (uint64_t)e * B.node_cap;
    uint32_t *hit_flag = B.hit_flag + tb;
    unsigned long long *cnt_flag = B.cnt_flag + tb;
    const uint4 tl = __ldcg(&B.tiles[tb + t]);
    const uint32_t l0 = tl.x, ln = tl.y, g0 = tl.z, g1 = tl.w;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // stage the frontier nodes [l0, l0 + ln) that hold the tile's items
    {
        uint32_t xq[kPer];
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            xq[i] = 0u;
            if (p < ln) {
                xq[i] = __ldcg(&V.queue[V.lo + l0 + p]);
                s.f_off[p] = __ldcg(&rs[l0 + p]);
                s.f_pre[p] = __ldcg(&pre[l0 + p]);
            }
        }
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            if (p < ln) {
                s.f_node[p] = xq[i];
                s.f_sig[p] = __ldcg(&V.rec[xq[i]].sigma);
            }
        }
        if (threadIdx.x == 0) s.f_pre[ln] = __ldcg(&pre[l0 + ln]);
    }
    __syncthreads();
    // ---- phase 1 (as in expand_level) ----------------------------------------
    uint32_t ys[kItems], xs[kItems], code[kItems], li[kItems];
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        const uint32_t it = g0 + (uint32_t)(k * BLOCK) + threadIdx.x;
        code[k] = 0;
        ys[k] = 0;
        xs[k] = 0;
        li[k] = 0;
        if (it < g1) {
            uint32_t l = 0, h = ln;
            while (h - l > 1) {
                const uint32_t mid = (l + h) >> 1;
                if (s.f_pre[mid] <= it) l = mid;
                else h = mid;
            }
            li[k] = l;
            xs[k] = s.f_node[l];
            ys[k] = __ldg(&V.adj[s.f_off[l] + (it - s.f_pre[l])]);
            code[k] = 3;
        }
    }
    uint32_t sty[kItems];
#pragma unroll
    for (int k = 0; k < kItems; k++) sty[k] = code[k] ? __ldcg(&V.rec[ys[k]].st) : 0u;
    // joins of earlier tiles only turn a state 0 into new_st: the classes
    // are those of the level's start
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        if (!code[k]) continue;
        if (sty[k] == 0u || sty[k] == V.new_st) code[k] = 1;
        else if (st_side(sty[k]) != V.side) code[k] = 2;
        else code[k] = 0;
    }
    uint32_t nh = 0;
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        if (code[k] != 1) continue;
        const uint32_t it = g0 + (uint32_t)(k * BLOCK) + threadIdx.x;
        const unsigned long long key = ((unsigned long long)it << 32) | xs[k];
        NodeRec *r = &V.rec[ys[k]];
        atomicMin(reinterpret_cast<unsigned long long *>(&r->first), key);
        atomicMax(reinterpret_cast<unsigned long long *>(&r->last), key);
        atomicAdd(&r->cnt, 1u);
        atomicAdd(reinterpret_cast<unsigned long long *>(&r->sigma), s.f_sig[li[k]]);
        nh++;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nh += __shfl_xor_sync(0xffffffffu, nh, o);
    if (lane == 0 && nh) atomicAdd(&E->hits, nh);
    __syncthreads();
    if (warp == 0) {
        if (lane == 0) {
            __threadfence();
            st_release_u32(&hit_flag[t], 1u);
        }
        __syncwarp();
        const bool ok = lookback_hits(hit_flag, t, s.a_spin);
        if (lane == 0) {
            // published even after a failed wait, so that later tiles do not
            // wait as well (the level is reported failed)
            st_release_u32(&hit_flag[t], 2u);
            __threadfence();
            s.a_ok = ok ? 1u : 0u;
            if (!ok) atomicExch(&E->err, 1u);
        }
    }
    __syncthreads();
    // ---- phase 2: joining hits and meeting edges, in item order ---------------
    unsigned long long fv[kItems];
    uint32_t dg[kItems];
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        fv[k] = code[k] == 1
                    ? __ldcg(reinterpret_cast<const unsigned long long *>(&V.rec[ys[k]].first))
                    : 0ull;
        const uint2 r = code[k] == 1 ? __ldg(&V.rows[ys[k]]) : make_uint2(0u, 0u);
        dg[k] = r.y - r.x;
    }
    uint32_t rnm[kItems];  // rank among the warp's joins (low half) and meeting edges
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        const uint32_t it = g0 + (uint32_t)(k * BLOCK) + threadIdx.x;
        if (code[k] == 1 && (uint32_t)(fv[k] >> 32) != it) code[k] = 0;
        const uint32_t bn = __ballot_sync(0xffffffffu, code[k] == 1);
        const uint32_t bm = __ballot_sync(0xffffffffu, code[k] == 2);
        rnm[k] = __popc(bn & lanemask_lt()) | (__popc(bm & lanemask_lt()) << 16);
        if (lane == 0) {
            s.warp_a[k * kWarps + warp] = __popc(bn);
            s.warp_b[k * kWarps + warp] = __popc(bm);
        }
    }
    __syncthreads();
    if (warp == 0) {
        // offsets over (item slot, warp) as in expand_level, based on the
        // earlier tiles' sums
        constexpr int kE = kItems * kWarps;
        constexpr int kPerLane = (kE + 31) / 32;
        uint32_t va[kPerLane], vb[kPerLane];
        uint32_t sa = 0, sb = 0;
#pragma unroll
        for (int i = 0; i < kPerLane; i++) {
            const int x = lane * kPerLane + i;
            va[i] = x < kE ? s.warp_a[x] : 0u;
            vb[i] = x < kE ? s.warp_b[x] : 0u;
            sa += va[i];
            sb += vb[i];
        }
        uint32_t ia = sa, ib = sb;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t ta = __shfl_up_sync(0xffffffffu, ia, o);
            const uint32_t tb2 = __shfl_up_sync(0xffffffffu, ib, o);
            if (lane >= o) {
                ia += ta;
                ib += tb2;
            }
        }
        const uint32_t aj = __shfl_sync(0xffffffffu, ia, 31);
        const uint32_t am = __shfl_sync(0xffffffffu, ib, 31);
        if (lane == 0) st_release_u64(&cnt_flag[t], cnt_word(t == 0 ? 2u : 1u, aj, am));
        unsigned long long ej = 0, em = 0;
        bool ok = true;
        if (t > 0) {
            __syncwarp();
            ok = lookback_counts(cnt_flag, t, ej, em, s.a_spin);
            if (lane == 0) st_release_u64(&cnt_flag[t], cnt_word(2u, ej + aj, em + am));
        }
        ok = ok && s.a_ok != 0u;
        if (lane == 0) {
            atomicAdd(&E->joins, aj);
            atomicAdd(&E->meets, am);
            if (!ok) atomicExch(&E->err, 1u);
        }
        const unsigned long long qb = (unsigned long long)V.qbase + ej;
        const unsigned long long mb = (unsigned long long)V.mbase + em;
        uint32_t ea = (uint32_t)min(qb, 0xffffffffull) + ia - sa;
        uint32_t eb = (uint32_t)min(mb, (unsigned long long)kMeetCap) + ib - sb;
        __syncwarp();
#pragma unroll
        for (int i = 0; i < kPerLane; i++) {
            const int x = lane * kPerLane + i;
            if (x < kE) {
                s.warp_a[x] = ea;
                s.warp_b[x] = eb;
            }
            ea += va[i];
            eb += vb[i];
        }
        if (lane == 0) s.a_ok = ok ? 1u : 0u;
    }
    __syncthreads();
    uint32_t sum = 0;
    if (s.a_ok) {
#pragma unroll
        for (int k = 0; k < kItems; k++) {
            if (code[k] == 1) {
                const uint32_t y = ys[k];
                V.queue[s.warp_a[k * kWarps + warp] + (rnm[k] & 0xffffu)] = y;
                V.rec[y].st = V.new_st;
                sum += dg[k];
            } else if (code[k] == 2) {
                const uint32_t pos = s.warp_b[k * kWarps + warp] + (rnm[k] >> 16);
                if (pos < kMeetCap) V.meet[pos] = make_uint2(xs[k], ys[k]);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0 && sum) atomicAdd(&E->sum_new, sum);
    __syncthreads();
}

// Takes tiles of entry e's level until none is left (owner and helpers).
template <int BLOCK>
__device__ void assist_work(SamplerSmem<BLOCK> &s, const SamplerLaunch &L, uint32_t e,
                            bool owner) {
    AssistEntry *E = L.assist.entries + e;
    const uint32_t nt = s.lvl.ntiles;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t t = atomicAdd(&E->claim, 1u);
            if (t + 1u == nt) atomicAnd(&L.hdr->open_mask, ~(1u << e));  // the last tile is taken
            s.a_tile = t;
        }
        __syncthreads();
        const uint32_t t = s.a_tile;
        if (t >= nt) break;
        assist_tile<BLOCK>(s, L.assist, e, t);
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(&E->done, 1u);
            if (!owner) atomicAdd(&L.hdr->helper_tiles, 1u);
        }
    }
    __syncthreads();
}

// The owner's side of a posted level (entry e, taken by acquire_entry):
// the frontier's item prefix and tile table, its share of the tiles, the
// results into the sample state, and the entry handed back.  Returns false,
// with the entry freed and nothing changed, when the tile table would not
// fit; the caller then runs expand_level.
template <int BLOCK>
__device__ bool expand_level_assisted(const SamplerLaunch &L, const SegDesc &A,
                                      SamplerSmem<BLOCK> &s, NodeRec *rec, uint32_t *queue,
                                      uint2 *meet, uint32_t side, uint32_t lo, uint32_t hi,
                                      uint32_t depth, uint32_t e) {
    constexpr int kTile = Shape<BLOCK>::kTile;
    constexpr int kChunk = Shape<BLOCK>::kChunk;
    constexpr int kPer = Shape<BLOCK>::kPerThread;
    const AssistBoard &B = L.assist;
    AssistEntry *E = B.entries + e;
    const uint2 *rows = side == kSideU ? A.out_rows : A.in_rows;
    const uint32_t *adj = side == kSideU ? A.out_adj : A.in_adj;
    const uint32_t F = hi - lo;
    const uint64_t tb = (uint64_t)e * B.tile_cap;
    uint32_t *pre = B.pre + (uint64_t)e * (B.node_cap + 1u);
    uint32_t *rs = B.rs + (uint64_t)e * B.node_cap;
    uint4 *tiles = B.tiles + tb;
    // item prefix, row starts, and the tiles, each starting in the node that
    // holds its first item
    uint32_t carry = 0, tcarry = 0;
    for (uint32_t c0 = 0; c0 < F; c0 += kChunk) {
        const uint32_t nc = min((uint32_t)kChunk, F - c0);
        uint32_t xq[kPer], o0[kPer], o1[kPer];
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            xq[i] = p < nc ? __ldcg(&queue[lo + c0 + p]) : 0u;
        }
        uint32_t tsum = 0;
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            o0[i] = o1[i] = 0u;
            if (p < nc) {
                const uint2 r = __ldg(&rows[xq[i]]);
                o0[i] = r.x;
                o1[i] = r.y;
            }
            tsum += o1[i] - o0[i];
        }
        uint32_t excl;
        const uint32_t total = block_exclusive_scan<BLOCK>(tsum, excl, s.scan_tmp);
#pragma unroll
        for (int i = 0; i < kPer; i++) {
            const uint32_t p = threadIdx.x * kPer + i;
            const uint32_t d = o1[i] - o0[i];
            if (p < nc) {
                pre[c0 + p] = carry + excl;
                rs[c0 + p] = o0[i];
                for (uint64_t j = ((uint64_t)excl + kTile - 1) / kTile;
                     j * kTile < (uint64_t)excl + d; j++) {
                    const uint64_t ti = (uint64_t)tcarry + j;
                    if (ti < B.tile_cap)
                        tiles[ti] = make_uint4(c0 + p, 0u, carry + (uint32_t)(j * kTile),
                                               carry + (uint32_t)min((j + 1) * kTile,
                                                                     (uint64_t)total));
                }
            }
            excl += d;
        }
        carry += total;
        tcarry += (total + kTile - 1) / kTile;
    }
    if (threadIdx.x == 0) pre[F] = carry;
    __syncthreads();
    const bool fits = tcarry >= 1u && tcarry <= B.tile_cap;
    if (fits) {
        // nodes to stage per tile: up to the node of the next tile's first
        // item in the same chunk, else to the chunk's end; look-back words
        // cleared
        for (uint32_t t = threadIdx.x; t < tcarry; t += BLOCK) {
            const uint32_t l0 = __ldcg(reinterpret_cast<const uint32_t *>(&tiles[t]));
            const uint32_t c = l0 / (uint32_t)kChunk;
            const uint32_t cend = (uint32_t)min((uint64_t)(c + 1u) * kChunk, (uint64_t)F);
            uint32_t endn = cend;
            if (t + 1u < tcarry) {
                const uint32_t nx = __ldcg(reinterpret_cast<const uint32_t *>(&tiles[t + 1u]));
                if (nx / (uint32_t)kChunk == c) endn = min(nx + 1u, cend);
            }
            reinterpret_cast<uint32_t *>(&tiles[t])[1] = endn - l0;
            B.hit_flag[tb + t] = 0u;
            B.cnt_flag[tb + t] = 0ull;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (fits) {
            AssistLevel &V = s.lvl;
            V.ntiles = tcarry;
            V.items = carry;
            V.nodes = F;
            V.lo = lo;
            V.new_st = st_make(side, depth + 1u);
            V.side = side;
            V.qbase = s.end_q;
            V.mbase = s.nmeet;
            V.rows = rows;
            V.adj = adj;
            V.rec = rec;
            V.queue = queue;
            V.meet = meet;
            E->lvl = V;
            E->claim = 0u;
            E->done = 0u;
            E->ntiles = tcarry;
            E->hits = 0u;
            E->sum_new = 0u;
            E->joins = 0u;
            E->meets = 0u;
            E->err = 0u;
            __threadfence();
            st_release_u32(&E->state, (s.a_state & ~3u) | 2u);
            atomicOr(&L.hdr->open_mask, 1u << e);
        } else {
            st_release_u32(&E->state, ((s.a_state >> 2) + 1u) << 2);
        }
    }
    __syncthreads();
    if (!fits) return false;
    assist_work<BLOCK>(s, L, e, true);
    if (threadIdx.x == 0) {
        const bool ok = wait_at_least(&E->done, tcarry, s.a_spin);
        __threadfence();
        if (ok && __ldcg(&E->err) == 0u) {
            const AssistLevel &V = s.lvl;
            s.end_q = V.qbase + __ldcg(&E->joins);
            const uint64_t mt = (uint64_t)V.mbase + __ldcg(&E->meets);
            if (mt > kMeetCap && s.status == 0) s.status = SILVAN_E_CAPACITY;
            s.nmeet = (uint32_t)min(mt, (uint64_t)kMeetCap);
            s.vis += V.items;
            s.sum_new = __ldcg(&E->sum_new);
            s.pred_hits += __ldcg(&E->hits);
            atomicAdd(&L.hdr->assisted, 1u);
        } else {
            s.status = SILVAN_E_TIMEOUT;
            s.sum_new = 0u;
            s.a_leave = 1u;
        }
        // hand the entry on only when no helper is inside any more: a helper
        // either shows in `inside` here or sees the closed state and leaves
        atomicAnd(&L.hdr->open_mask, ~(1u << e));
        atomicExch(&E->state, (s.a_state & ~3u) | 3u);
        __threadfence();
        if (wait_zero(&E->inside, s.a_spin)) {
            st_release_u32(&E->state, ((s.a_state >> 2) + 1u) << 2);
        } else {
            // the entry stays closed until the next launch reopens it
            if (s.status == 0) s.status = SILVAN_E_TIMEOUT;
            s.a_leave = 1u;
        }
    }
    return true;
}

// Helps the posted level thread 0 entered (s.a_entry), then leaves it.
template <int BLOCK>
__device__ void help_entry(const SamplerLaunch &L, SamplerSmem<BLOCK> &s, uint32_t e) {
    assist_work<BLOCK>(s, L, e, false);
    if (threadIdx.x == 0) {
        __threadfence();
        atomicSub(&L.assist.entries[e].inside, 1u);
    }
}

// Segment owning work index w: the last segment whose base is <= w.
__device__ __forceinline__ uint32_t segment_of(const SegDesc *segs, uint32_t nsegs, uint32_t w) {
    uint32_t l = 0, h = nsegs;
    while (h - l > 1) {
        const uint32_t mid = (l + h) >> 1;
        if (segs[mid].base <= w) l = mid;
        else h = mid;
    }
    return l;
}

// Takes the next kScreen work indices of the round (one while few are left)
// and screens them, one thread each: endpoints (Sp_sampler.cpp:46,58-60)
// and the void test (:62-74).  A void sample's outputs are written here; the
// others are queued in s.pend_w for the full sampler.  Sets s.a_drained when
// the round has no sample left.
template <int BLOCK>
__device__ __noinline__ void screen_chunk(const SamplerLaunch &L, SamplerSmem<BLOCK> &s,
                                          uint32_t total, uint32_t nsegs) {
    if (threadIdx.x == 0) {
        const uint32_t taken = ld_acquire_u32(&L.hdr->work);
        const uint32_t left = taken < total ? total - taken : 0u;
        const uint32_t v = left > 2u * kScreen * gridDim.x ? kScreen : 1u;
        const uint32_t w0 = atomicAdd(&L.hdr->work, v);
        s.scr_w0 = w0;
        s.scr_v = v;
        s.pend_n = 0;
        s.pend_i = 0;
        if (w0 >= total) s.a_drained = 1;
    }
    __syncthreads();
    const uint32_t w = s.scr_w0 + threadIdx.x;
    bool is_void = false;
    if (threadIdx.x < s.scr_v && w < total) {
        const long long t0 = clock64();
        const SegDesc &A = L.segs[segment_of(L.segs, nsegs, w)];
        const uint32_t gidx = A.first_sample + (w - A.base);
        uint32_t d = 0;
        uint32_t v = draw32(A.seed, gidx, d++) % A.n;
        const uint32_t u = draw32(A.seed, gidx, d++) % A.n;
        while (u == v) v = draw32(A.seed, gidx, d++) % A.n;
        is_void = A.directed ? (A.cc[u] < A.cc[v]) : (A.cc[u] != A.cc[v]);
        if (is_void) {
            const uint32_t sl = w - A.base;
            A.out_pl[sl] = 0;
            A.out_np[sl] = 0;
            A.out_vis[sl] = 0;
            A.out_status[sl] = 0;
            A.out_ball[sl] = 0;
            A.out_pred[sl] = 0;
            atomicAdd(&L.hdr->cycles, (unsigned long long)(clock64() - t0));
        } else {
            s.pend_w[atomicAdd(&s.pend_n, 1u)] = w;
        }
    }
    const uint32_t nv = __syncthreads_count(is_void);
    if (threadIdx.x == 0 && nv) {
        __threadfence();
        atomicAdd(&L.hdr->finished, nv);
    }
    __syncthreads();
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

    // Between two samples, a posted level that has tiles left comes first.
    // Once the round has no sample left, the CTA keeps helping posted levels
    // until every sample is done (or it has polled kAssistPolls times).  The
    // loop's own state lives in shared memory, out of the registers of the
    // sample code.
    if (threadIdx.x == 0) {
        s.a_drained = 0;
        s.a_polls = 0;
        s.a_nap = 256;
        s.a_spin = L.hdr->wait_polls;
        s.a_leave = 0;
    }
    if (threadIdx.x == 0) s.pend_n = s.pend_i = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            int32_t pick = L.assist.entries != nullptr && !s.a_leave
                               ? join_entry<BLOCK>(L, s, blockIdx.x)
                               : -1;
            if (pick < 0 && !s.a_leave && s.pend_i < s.pend_n) {
                const uint32_t w = s.pend_w[s.pend_i++];
                s.work = w;
                s.sample = segment_of(L.segs, nsegs, w);
                pick = -3;  // a sample
            } else if (pick < 0 && !s.a_drained && !s.a_leave) {
                pick = -4;  // take the next chunk of the round
            }
            if (pick == -1 && s.a_leave) {
                // this CTA leaves the launch (its slot may be inconsistent):
                // the samples it screened but has not run are reported failed
                for (; s.pend_i < s.pend_n; s.pend_i++) {
                    const uint32_t w = s.pend_w[s.pend_i];
                    const SegDesc &B = L.segs[segment_of(L.segs, nsegs, w)];
                    const uint32_t sl = w - B.base;
                    B.out_pl[sl] = 0;
                    B.out_np[sl] = 0;
                    B.out_vis[sl] = 0;
                    B.out_status[sl] = SILVAN_E_TIMEOUT;
                    B.out_ball[sl] = 0;
                    B.out_pred[sl] = 0;
                    __threadfence();
                    atomicAdd(&L.hdr->finished, 1u);
                }
            }
            if (pick == -1) {
                // no sample left: wait for posted levels, or leave
                s.a_drained = 1;
                if (L.assist.entries == nullptr || s.a_leave || ++s.a_polls > kAssistPolls ||
                    ld_acquire_u32(&L.hdr->finished) >= total) {
                    pick = -2;
                } else {
                    __nanosleep(s.a_nap);
                    s.a_nap = min(s.a_nap * 2u, 4096u);
                }
            } else {
                s.a_nap = 256;
            }
            s.a_entry = pick;
        }
        __syncthreads();
        const int32_t pick = s.a_entry;
        if (pick >= 0) {
            help_entry<BLOCK>(L, s, (uint32_t)pick);
            __syncthreads();
            continue;
        }
        if (pick == -2) break;
        if (pick == -1) {
            __syncthreads();
            continue;
        }
        if (pick == -4) {
            screen_chunk<BLOCK>(L, s, total, nsegs);
            continue;
        }
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
                atomicAdd(&L.hdr->finished, 1u);
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
            if (threadIdx.x == 0)
                s.a_entry = (L.assist.entries != nullptr && A.assist_items != 0u)
                                ? post_level<BLOCK>(L, s, side_u, lo, hi, depth)
                                : -1;
            __syncthreads();
            if (s.a_entry < 0 ||
                !expand_level_assisted<BLOCK>(L, A, s, rec, queue, meet, exp_side, lo, hi, depth,
                                              (uint32_t)s.a_entry))
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
                            uint4 r0, r1;
                            rec_load(&rec[a], r0, r1);
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
            unsigned long long b = ~0ull;
            if (nt > 0 && s.status == 0) {
                b = atomicAdd(A.rec_cursor, (unsigned long long)nt);
                if (b + nt > A.rec_cap) s.status = SILVAN_E_CAPACITY;
            }
            s.rec_base = b;
        }
        __syncthreads();
        const unsigned long long rb = s.rec_base;
        const bool emit = s.status == 0;
        // A sample whose path map did not fit may have reserved slots below
        // the buffer's end: they get placeholders (count 0, node ~0) of this
        // sample, so that every slot below the end holds a defined record.
        const bool fill = !emit && rb < A.rec_cap;
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
                } else if (fill && rb + i < A.rec_cap) {
                    PathRec pr;
                    pr.node = 0xffffffffu;
                    pr.sample = sl;
                    pr.count = 0;
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
            if (s.a_leave) atomicAdd(&L.hdr->failed, 1u);
            __threadfence();
            atomicAdd(&L.hdr->finished, 1u);
        }
        __syncthreads();
    }
}

__global__ void round_begin_kernel(SamplerLaunch L, uint32_t max_segs) {
    const uint32_t ns = min(L.hdr->nsegs, max_segs);
    for (uint32_t i = threadIdx.x; i < ns; i += blockDim.x) *L.segs[i].rec_cursor = 0ull;
    if (threadIdx.x == 0) {
        L.hdr->work = 0;
        L.hdr->finished = 0;
        L.hdr->open_mask = 0;
        L.hdr->assisted = 0;
        L.hdr->helper_tiles = 0;
        L.hdr->failed = 0;
        L.hdr->cycles = 0;
        L.hdr->max_cycles = 0;
    }
    // No sampler CTA runs between two launches: a board entry that a failed
    // wait left closed (or any entry not free) is handed back here, with its
    // generation advanced and nobody inside.
    if (L.assist.entries != nullptr && threadIdx.x < kAssistEntries) {
        AssistEntry *E = L.assist.entries + threadIdx.x;
        const uint32_t st = E->state;
        if ((st & 3u) != 0u) {
            E->state = ((st >> 2) + 1u) << 2;
            E->inside = 0u;
        }
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

namespace {
constexpr uint32_t kAssistTileCap = 1u << 16;
uint64_t align256(uint64_t b) { return (b + 255u) & ~255ull; }
}  // namespace

uint64_t assist_board_bytes(uint64_t n) {
    return align256(sizeof(AssistEntry) * kAssistEntries) +
           align256(4ull * (n + 1) * kAssistEntries) + align256(4ull * n * kAssistEntries) +
           align256(16ull * kAssistTileCap * kAssistEntries) +
           align256(4ull * kAssistTileCap * kAssistEntries) +
           align256(8ull * kAssistTileCap * kAssistEntries);
}

cudaError_t assist_board_init(AssistBoard *b, void *mem, uint64_t n, cudaStream_t stream) {
    if (n >= 0x7fffffffull) return cudaErrorInvalidValue;  // joins fit the look-back words
    char *p = static_cast<char *>(mem);
    b->entries = reinterpret_cast<AssistEntry *>(p);
    p += align256(sizeof(AssistEntry) * kAssistEntries);
    b->pre = reinterpret_cast<uint32_t *>(p);
    p += align256(4ull * (n + 1) * kAssistEntries);
    b->rs = reinterpret_cast<uint32_t *>(p);
    p += align256(4ull * n * kAssistEntries);
    b->tiles = reinterpret_cast<uint4 *>(p);
    p += align256(16ull * kAssistTileCap * kAssistEntries);
    b->hit_flag = reinterpret_cast<uint32_t *>(p);
    p += align256(4ull * kAssistTileCap * kAssistEntries);
    b->cnt_flag = reinterpret_cast<unsigned long long *>(p);
    b->node_cap = (uint32_t)n;
    b->tile_cap = kAssistTileCap;
    return cudaMemsetAsync(b->entries, 0, sizeof(AssistEntry) * kAssistEntries, stream);
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
