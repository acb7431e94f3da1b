// Ordered commit of sample contributions (see counters.cuh).
//
// The reference adds every sample's path map to the per-node counters inside
// one critical section, in sample order (silvan/src/Probabilistic.cpp:479-544):
//   x = count * (1 / num_paths)
//   approx[u] += x;  emp_wimpy_vars[u] += x * x;
//   mcrade[u][j] = (int64)((double)mcrade[u][j] + sign_j * x)   (truncation)
// With num_paths > 1 the additions are not associative, so a node's updates
// must be applied in sample order.  A round's records are grouped by node
// (count, bucket space, scatter), each node's group is put in sample order
// (by rank: compares for groups of <= 32, a bitmap of the sub-round's samples
// otherwise) and the group is folded sequentially by one warp: lanes 0..24
// each carry one Monte Carlo trial, lane 25 approx, lane 26 the wimpy
// variance.  Different nodes are independent, so the only serial work is per
// node.
#include <algorithm>
#include <cstddef>
#include <cfloat>
#include <climits>
#include <cstring>
#include <vector>

#include "counters.cuh"

namespace silvan {

namespace {

// ---------------------------------------------------------------------------
// One commit round as a single cooperative kernel.  Its phases are separated
// by grid-wide barriers (every CTA is resident: cooperative launch):
//   A  per sample the Rademacher signs (pass 2) and 1 / num_paths; records
//      counted per node and the touched nodes listed
//   B  bucket space of every touched node taken from a cursor (warp
//      aggregated), the scatter cursors, the list of buckets of more than
//      32 entries
//   C  records scattered into their nodes' buckets
//   D  the sub-round's 1 / num_paths and signs staged in shared memory;
//      the large buckets on warp 0 of each CTA (claimed from a cursor), the
//      small ones on the other warps (fixed assignment); the round's scalar
//      sums; cursors zeroed
// Each barrier is bounded: a CTA that waits longer than kBarrierPolls polls
// records SILVAN_E_TIMEOUT in the job's error word and leaves the kernel.
// ---------------------------------------------------------------------------
constexpr int kCommitThreads = 1024;
constexpr uint32_t kBarrierPolls = 1u << 22;  // far above any real wait (microseconds)

__device__ __forceinline__ uint32_t round_records(const RoundBuffers &rb, const ApplyArgs &a) {
    return (uint32_t)min((uint64_t)a.n_records, rb.rec_cap);
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier over bar[0] (arrivals) and bar[1] (generation); false
// when this CTA gave up waiting.
__device__ bool grid_barrier(uint32_t *bar) {
    __syncthreads();
    int ok = 1;
    if (threadIdx.x == 0) {
        const uint32_t gen = ld_acquire(&bar[1]);
        __threadfence();
        if (atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
            bar[0] = 0u;
            __threadfence();
            st_release(&bar[1], gen + 1u);
        } else {
            uint32_t i = 0;
            while (ld_acquire(&bar[1]) == gen) {
                if (++i > kBarrierPolls) {
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
    }
    return __syncthreads_and(ok) != 0;
}

__device__ void bucket_count(const RoundBuffers &rb, const ApplyArgs &a) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31;
    // per sample, one warp: the Rademacher signs (pass 2; lane j draws trial
    // j, as rademacher_mask does) and 1 / num_paths, the factor every record
    // of the sample is multiplied by (Probabilistic.cpp:502)
    for (uint32_t s = a.lo + (tid >> 5); s < a.hi; s += nth >> 5) {
        if (a.pass == 2) {
            bool plus = false;
            if (lane < (uint32_t)kTrials)
                plus = philox_lo32(a.seed, a.first_sample + s, kStreamRademacher, lane) %
                           100000000u >= 50000000u;
            const uint32_t m = __ballot_sync(0xffffffffu, plus);
            if (lane == 0) rb.signs[s] = m;
        }
        if (lane == 31) rb.inv_np[s] = __ddiv_rn(1.0, (double)rb.np[s]);
    }
    const uint32_t R = round_records(rb, a);
    // warp-uniform loop: the first record of a node is appended to the
    // touched list with one counter increment per warp (a single counter
    // that every warp hits would serialise the whole phase)
    for (uint32_t i0 = tid - lane; i0 < R; i0 += nth) {
        const uint32_t i = i0 + lane;
        bool first = false;
        uint32_t node = 0;
        if (i < R) {
            const PathRec r = rb.recs[i];
            node = r.node;
            if (r.sample >= a.lo && r.sample < a.hi)
                first = atomicAdd(&rb.node_cnt[r.node], 1u) == 0u;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, first);
        if (m) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(rb.n_touched, (uint32_t)__popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (first) rb.touched[base + __popc(m & ((1u << lane) - 1u))] = node;
        }
    }
}

// Bucket space of every touched node, taken from a cursor (the buckets need
// no order among themselves): one atomic per warp for the warp's nodes, the
// lanes' offsets by a warp scan.  The node's count becomes its scatter
// cursor; buckets of more than 32 entries are listed for the CTA-wide fold.
__device__ void bucket_alloc(const RoundBuffers &rb, uint32_t T) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t t0 = tid - lane; t0 < T; t0 += nth) {
        const uint32_t t = t0 + lane;
        uint32_t node = 0, b = 0;
        if (t < T) {
            node = rb.touched[t];
            b = rb.node_cnt[node];
        }
        uint32_t incl = b;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        uint32_t base = 0;
        if (lane == 31 && incl) base = atomicAdd(rb.n_touched + 4, incl);
        base = __shfl_sync(0xffffffffu, base, 31);
        const bool large = b > 32;
        const uint32_t lm = __ballot_sync(0xffffffffu, large);
        uint32_t lbase = 0;
        if (lm && lane == 0) lbase = atomicAdd(rb.n_large, (uint32_t)__popc(lm));
        lbase = __shfl_sync(0xffffffffu, lbase, 0);
        if (t < T) {
            const uint32_t off = base + incl - b;
            rb.bucket_off[t] = off;
            rb.bucket_len[t] = b;
            rb.node_cnt[node] = off;  // becomes the scatter cursor
            if (large) rb.large[lbase + __popc(lm & ((1u << lane) - 1u))] = t;
        }
    }
}

__device__ void bucket_scatter(const RoundBuffers &rb, const ApplyArgs &a) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const uint32_t R = round_records(rb, a);
    for (uint32_t i = tid; i < R; i += nth) {
        PathRec r = rb.recs[i];
        if (r.sample < a.lo || r.sample >= a.hi) continue;
        uint32_t pos = atomicAdd(&rb.node_cnt[r.node], 1u);
        rb.entries[pos] = ((unsigned long long)r.sample << 32) | r.count;
    }
}
// Sequential fold of one node's contributions in sample order.  Every lane
// runs the same instruction stream and carries one chain: lane j < 25 trial j
// of mcrade, lane 25 approx (and the top-k crossing), lane 26 the wimpy
// variance; lanes 27..31 repeat lane 25's chain and store nothing.  The chains
// advance together, one entry per step.  The entries are staged 32 at a time
// in the warp's scratch: x = count * (1 / num_paths), the sample's signs and
// its round-local index.
struct FoldScratch {
    double x[32];
    uint32_t signs[32];
    uint32_t sample[32];
    uint32_t upd[32];  // nodes updated for the first time, not yet on upd_list
    uint32_t nupd;
    double sup_a, sup_w;  // the warp's maxima of approx and emp_wimpy_vars
};

// Per-warp folding state: reset before a warp's first fold, flushed after its
// last (fold_flush), so that the job-wide maxima and the update list take one
// global atomic per warp rather than one per node.
__device__ __forceinline__ void fold_begin(FoldScratch &fs) {
    if ((threadIdx.x & 31) == 0) {
        fs.nupd = 0;
        fs.sup_a = 0.0;
        fs.sup_w = 0.0;
    }
    __syncwarp();
}

__device__ __forceinline__ void upd_flush(const JobCounters &jc, FoldScratch &fs) {
    const uint32_t lane = threadIdx.x & 31;
    __syncwarp();
    const uint32_t k = fs.nupd;
    if (k) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&jc.sc->n_upd, k);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (lane < k) jc.upd_list[base + lane] = fs.upd[lane];
        __syncwarp();
        if (lane == 0) fs.nupd = 0;
    }
    __syncwarp();
}

__device__ __forceinline__ void atomic_max_nonneg_double(unsigned long long *p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ void fold_flush(const JobCounters &jc, FoldScratch &fs) {
    upd_flush(jc, fs);
    if ((threadIdx.x & 31) == 0) {
        if (fs.sup_a > 0.) atomic_max_nonneg_double(&jc.sc->sup_approx_bits, fs.sup_a);
        if (fs.sup_w > 0.) atomic_max_nonneg_double(&jc.sc->sup_wimpy_bits, fs.sup_w);
    }
    __syncwarp();
}

// A node's counters as its fold starts, loaded before its entries are put in
// order so that the loads overlap that work.
struct NodeState {
    double v;         // this lane's chain
    uint32_t lu0;     // last_upd before the round
    bool crossed;     // lane 25: approx reached 3 in an earlier round (top-k pass 1)
};

// A journaled round also saves them at the node's touched position t.
__device__ __forceinline__ NodeState fold_load(const JobCounters &jc, const RoundJournal &jr,
                                               const ApplyArgs &a, uint32_t node, uint32_t t) {
    const int lane = threadIdx.x & 31;
    NodeState s{0.0, 0u, true};
    if (lane < kTrials) {
        if (a.pass == 2) {
            const long long m = jc.mcrade[(uint64_t)node * kTrials + lane];
            if (a.journal) jr.mcrade[(uint64_t)t * kTrials + lane] = m;
            s.v = (double)m;
        }
    } else if (lane == 26) {
        s.v = jc.wimpy[node];
        if (a.journal) jr.wimpy[t] = s.v;
    } else {
        s.v = jc.approx[node];
        if (lane == 25) {
            s.lu0 = jc.last_upd[node];
            if (a.track_cross) s.crossed = jc.cross_flag[node] != 0;
            if (a.journal) {
                jr.approx[t] = s.v;
                jr.last_upd[t] = s.lu0;
            }
        }
    }
    return s;
}

// Folds the node's b entries; fill(r0) has lane i stage entry r0 + i (when
// below b) in the scratch.
template <typename Fill>
__device__ void fold_node(const JobCounters &jc, const ApplyArgs &a, uint32_t node, uint32_t b,
                          NodeState st, Fill fill, FoldScratch &fs) {
    const int lane = threadIdx.x & 31;
    const bool mc = lane < kTrials, wv = lane == 26;
    double v = st.v;
    uint32_t lu = 0;
    for (uint32_t r0 = 0; r0 < b; r0 += 32) {
        fill(r0);
        __syncwarp();
        const bool pos = r0 + lane < b && fs.x[lane] > 0.;
        const uint32_t pm = __ballot_sync(0xffffffffu, pos);
        // 1 + global index of the last sample that adds to approx
        if (pm) lu = a.first_sample + fs.sample[31 - __clz(pm)] + 1u;
        const uint32_t kmax = min(32u, b - r0);
        int kc = -1;
#pragma unroll 4
        for (uint32_t k = 0; k < kmax; k++) {
            const double x = fs.x[k];
            const bool plus = (fs.signs[k] >> lane) & 1u;
            // mcrade: (int64)((double)m + s x), m kept as an integer-valued
            // double (|m| is at most the sample count, far below 2^53, so the
            // conversions are exact and truncating in double is the same);
            // approx and the wimpy variance add x and x * x when x > 0
            const double add = x > 0. ? (wv ? __dmul_rn(x, x) : x) : 0.0;
            const double y = mc ? (plus ? x : -x) : add;
            const double t = __dadd_rn(v, y);
            if (!st.crossed && kc < 0 && t >= 3.0) kc = (int)k;
            v = mc ? trunc(t) : t;
        }
        if (kc >= 0) {  // lane 25 only: approx reached 3 at entry kc
            st.crossed = true;
            jc.cross_flag[node] = 1;
            const uint32_t q = atomicAdd(&jc.sc->n_cross, 1u);
            jc.cross_sample[q] = a.first_sample + fs.sample[kc];
        }
        __syncwarp();
    }
    if (mc) {
        if (a.pass == 2) jc.mcrade[(uint64_t)node * kTrials + lane] = (long long)v;
    } else if (lane == 25) {
        jc.approx[node] = v;
        if (lu) {
            if (st.lu0 == 0) fs.upd[fs.nupd++] = node;
            jc.last_upd[node] = lu;
        }
        fs.sup_a = fmax(fs.sup_a, v);
    } else if (wv) {
        jc.wimpy[node] = v;
        fs.sup_w = fmax(fs.sup_w, v);
    }
    __syncwarp();
    if (fs.nupd == 32) upd_flush(jc, fs);
}

// Shared memory of phase D: the sub-round's per-sample factors (read by every
// fold in place of global gathers), warp 0's large bucket in sample order, and
// one fold scratch per warp.  s_inv holds samples from lo & ~1 on, s_sgn
// from lo & ~3 on (inv_base / sgn_base).
struct CommitSmem {
    double s_inv[kLargeBucket + 2];         // 1 / num_paths of the sub-round's samples
    uint32_t s_sgn[kLargeBucket + 4];       // their Rademacher signs (pass 2)
    unsigned long long sbuf[kLargeBucket];  // warp 0's bucket, in sample order
    uint32_t bits[kLargeBucket / 32];       // samples of that bucket
    uint32_t wpre[kLargeBucket / 32];       // set bits before each word
    FoldScratch fsc[kCommitThreads / 32];
};
constexpr size_t kCommitSmem = sizeof(CommitSmem);
__device__ __forceinline__ uint32_t inv_base(const ApplyArgs &a) { return a.lo & ~1u; }
__device__ __forceinline__ uint32_t sgn_base(const ApplyArgs &a) { return a.lo & ~3u; }

// The sub-round's 1 / num_paths and signs into shared memory, read with
// L2-coherent loads: phase A wrote them from other CTAs, ordered before this
// read by the grid barrier.
__device__ void stage_factors(const RoundBuffers &rb, const ApplyArgs &a, CommitSmem &sm) {
    const uint32_t i0 = inv_base(a), i1 = min((a.hi + 1u) & ~1u, rb.max_samples);
    const uint32_t s0 = sgn_base(a), s1 = min((a.hi + 3u) & ~3u, rb.max_samples);
    for (uint32_t i = threadIdx.x; i < i1 - i0; i += blockDim.x)
        sm.s_inv[i] = __ldcg(&rb.inv_np[i0 + i]);
    for (uint32_t i = threadIdx.x; i < s1 - s0; i += blockDim.x)
        sm.s_sgn[i] = a.pass == 2 ? __ldcg(&rb.signs[s0 + i]) : 0u;
    __syncthreads();
}
constexpr int kLoads = 8;  // bucket entries a lane of warp 0 loads at once
constexpr uint32_t kSmallWarps = kCommitThreads / 32 - 1;  // warps 1.. of each CTA

// Buckets of at most 32 entries, on warps 1.. of every CTA: touched node t
// goes to warp t mod (CTAs x kSmallWarps), no cursor.  A bucket holds
// distinct samples, so each entry's position in sample order is the number
// of entries with a smaller sample (32 compares per lane, no sort).
__device__ void apply_small(const RoundBuffers &rb, const JobCounters &jc, const RoundJournal &jr,
                            const ApplyArgs &a, uint32_t T, CommitSmem &sm) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    FoldScratch &fs = sm.fsc[wib];
    fold_begin(fs);
    const uint32_t stride = gridDim.x * kSmallWarps;
    for (uint32_t t = blockIdx.x * kSmallWarps + (uint32_t)(wib - 1); t < T; t += stride) {
        const uint32_t b = __ldcg(&rb.bucket_len[t]);
        if (b > 32) continue;
        const uint32_t node = __ldcg(&rb.touched[t]);
        const NodeState st = fold_load(jc, jr, a, node, t);
        const unsigned long long key =
            (uint32_t)lane < b ? __ldcg(&rb.entries[__ldcg(&rb.bucket_off[t]) + lane]) : ~0ull;
        uint32_t rank = 0;
        for (uint32_t j = 0; j < b; j++) rank += __shfl_sync(0xffffffffu, key, (int)j) < key;
        fold_node(jc, a, node, b, st,
                  [&](uint32_t) {
                      if ((uint32_t)lane < b) {
                          const uint32_t sl = (uint32_t)(key >> 32);
                          fs.x[rank] = __dmul_rn((double)(uint32_t)key, sm.s_inv[sl - inv_base(a)]);
                          fs.signs[rank] = sm.s_sgn[sl - sgn_base(a)];
                          fs.sample[rank] = sl;
                      }
                  },
                  fs);
    }
    fold_flush(jc, fs);
}

// Buckets of more than 32 entries, on warp 0 of every CTA, claimed from a
// cursor.  The entries of a bucket are distinct samples of the sub-round (a
// node is on a sample's path map once), so their order is the rank of each
// sample in a bitmap of the sub-round: set one bit per entry, prefix-count
// the bits per word, and each entry goes to its rank (linear in the bucket;
// no comparison sort).
__device__ void apply_large(const RoundBuffers &rb, const JobCounters &jc, const RoundJournal &jr,
                            const ApplyArgs &a, CommitSmem &sm) {
    const int lane = threadIdx.x & 31;
    FoldScratch &fs = sm.fsc[0];
    fold_begin(fs);
    const uint32_t NL = __ldcg(rb.n_large);
    const uint32_t S = a.hi - a.lo;
    const uint32_t nwords = (S + 31) / 32, per = (nwords + 31) / 32;
    const uint32_t w0 = min(nwords, lane * per), w1 = min(nwords, w0 + per);
    for (;;) {
        uint32_t li = 0;
        if (lane == 0) li = atomicAdd(rb.n_touched + 5, 1u);
        li = __shfl_sync(0xffffffffu, li, 0);
        if (li >= NL) break;
        const uint32_t t = __ldcg(&rb.large[li]);
        const uint32_t b0 = __ldcg(&rb.bucket_off[t]), b = __ldcg(&rb.bucket_len[t]);
        if (b > S) {  // more entries than samples: not a bucket of distinct samples
            if (lane == 0) atomicCAS(&jc.sc->error, 0, SILVAN_E_STATE);
            continue;
        }
        const uint32_t node = __ldcg(&rb.touched[t]);
        const NodeState st = fold_load(jc, jr, a, node, t);
        for (uint32_t w = w0; w < w1; w++) sm.bits[w] = 0u;
        __syncwarp();
        // the bucket's entries kLoads at a time per lane, all loads in
        // flight before their uses
        for (uint32_t i0 = 0; i0 < b; i0 += 32 * kLoads) {
            unsigned long long e[kLoads];
#pragma unroll
            for (int j = 0; j < kLoads; j++) {
                const uint32_t i = i0 + (uint32_t)j * 32 + lane;
                e[j] = i < b ? __ldcg(&rb.entries[b0 + i]) : 0ull;
            }
#pragma unroll
            for (int j = 0; j < kLoads; j++) {
                if (i0 + (uint32_t)j * 32 + lane >= b) continue;
                const uint32_t sidx = (uint32_t)(e[j] >> 32) - a.lo;
                if (sidx < S) atomicOr(&sm.bits[sidx >> 5], 1u << (sidx & 31));
                else atomicCAS(&jc.sc->error, 0, SILVAN_E_STATE);
            }
        }
        __syncwarp();
        // exclusive prefix of the words' bit counts (lane L owns words
        // [L per, (L + 1) per))
        uint32_t c = 0;
        for (uint32_t w = w0; w < w1; w++) c += __popc(sm.bits[w]);
        uint32_t incl = c;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        uint32_t run = incl - c;
        for (uint32_t w = w0; w < w1; w++) {
            sm.wpre[w] = run;
            run += __popc(sm.bits[w]);
        }
        __syncwarp();
        for (uint32_t i0 = 0; i0 < b; i0 += 32 * kLoads) {
            unsigned long long e[kLoads];
#pragma unroll
            for (int j = 0; j < kLoads; j++) {
                const uint32_t i = i0 + (uint32_t)j * 32 + lane;
                e[j] = i < b ? __ldcg(&rb.entries[b0 + i]) : 0ull;
            }
#pragma unroll
            for (int j = 0; j < kLoads; j++) {
                if (i0 + (uint32_t)j * 32 + lane >= b) continue;
                const uint32_t sidx = (uint32_t)(e[j] >> 32) - a.lo;
                if (sidx < S) {
                    const uint32_t w = sidx >> 5;
                    sm.sbuf[sm.wpre[w] + __popc(sm.bits[w] & ((1u << (sidx & 31)) - 1u))] = e[j];
                }
            }
        }
        __syncwarp();
        fold_node(jc, a, node, b, st,
                  [&](uint32_t r0) {
                      const uint32_t r = r0 + lane;
                      if (r < b) {
                          const unsigned long long e = sm.sbuf[r];
                          const uint32_t sl = (uint32_t)(e >> 32);
                          fs.x[lane] = __dmul_rn((double)(uint32_t)e, sm.s_inv[sl - inv_base(a)]);
                          fs.signs[lane] = sm.s_sgn[sl - sgn_base(a)];
                          fs.sample[lane] = sl;
                      }
                  },
                  fs);
    }
    fold_flush(jc, fs);
}

__device__ void commit_sums(const RoundBuffers &rb, const JobCounters &jc, const ApplyArgs &a) {
    unsigned long long vis = 0, cnt = 0, vd = 0, paths = 0, ball = 0, pred = 0;
    for (uint32_t s = a.lo + blockIdx.x * blockDim.x + threadIdx.x; s < a.hi;
         s += gridDim.x * blockDim.x) {
        const int32_t st = rb.status[s];
        if (st != 0) atomicCAS(&jc.sc->error, 0, st);
        vis += rb.vis[s];
        ball += rb.ball[s];
        pred += rb.pred[s];
        const int32_t pl = rb.pl[s];
        if (pl > 0) {
            if ((uint32_t)pl <= a.D) atomicAdd((unsigned long long *)&jc.sp_lengths[pl], 1ull);
            else atomicCAS(&jc.sc->error, 0, SILVAN_E_STATE);
            cnt++;
            paths += (unsigned long long)rb.np[s];
        } else {
            vd++;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        vis += __shfl_xor_sync(0xffffffffu, vis, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        vd += __shfl_xor_sync(0xffffffffu, vd, o);
        paths += __shfl_xor_sync(0xffffffffu, paths, o);
        ball += __shfl_xor_sync(0xffffffffu, ball, o);
        pred += __shfl_xor_sync(0xffffffffu, pred, o);
    }
    // per CTA in shared memory, then one global add per CTA and sum
    __shared__ unsigned long long cs[6];
    if (threadIdx.x < 6) cs[threadIdx.x] = 0ull;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        if (vis) atomicAdd(&cs[0], vis);
        if (cnt) atomicAdd(&cs[1], cnt);
        if (vd) atomicAdd(&cs[2], vd);
        if (paths) atomicAdd(&cs[3], paths);
        if (ball) atomicAdd(&cs[4], ball);
        if (pred) atomicAdd(&cs[5], pred);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (cs[0]) atomicAdd(&jc.sc->vis_edges, cs[0]);
        if (cs[1]) atomicAdd(&jc.sc->counted_samples, cs[1]);
        if (cs[2]) atomicAdd(&jc.sc->void_samples, cs[2]);
        if (cs[3]) atomicAdd(&jc.sc->paths, cs[3]);
        if (cs[4]) atomicAdd(&jc.sc->ball_nodes, cs[4]);
        if (cs[5]) atomicAdd(&jc.sc->pred_entries, cs[5]);
    }
}


// The last CTA out zeroes the round's control words for the next round
// (word 7, the touched count, stays for undo_round).
__device__ void commit_exit(const RoundBuffers &rb) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(rb.n_touched + 6, 1u) == gridDim.x - 1) {
            rb.n_touched[0] = 0u;
            rb.n_touched[1] = 0u;
            rb.n_touched[4] = 0u;
            rb.n_touched[5] = 0u;
            rb.n_touched[6] = 0u;
            __threadfence();
        }
    }
}

__global__ void __launch_bounds__(kCommitThreads, 1) commit_round_kernel(const ApplyState st) {
    extern __shared__ __align__(16) unsigned char commit_smem[];
    const RoundBuffers &rb = st.rb;
    const JobCounters &jc = st.jc;
    const RoundJournal &jr = st.jr;
    const ApplyArgs &a = st.a;
    uint32_t *bar = rb.n_touched + 2;
    if (a.journal && blockIdx.x == 0) {
        // the scalars and path-length counts as the round starts (phase D
        // is the first to change them)
        const unsigned long long *src = reinterpret_cast<const unsigned long long *>(jc.sc);
        unsigned long long *dst = reinterpret_cast<unsigned long long *>(jr.sc);
        for (uint32_t i = threadIdx.x; i < sizeof(JobScalars) / 8; i += blockDim.x) dst[i] = src[i];
        for (uint32_t i = threadIdx.x; i <= a.D; i += blockDim.x) jr.sp_lengths[i] = jc.sp_lengths[i];
    }
    bucket_count(rb, a);
    if (!grid_barrier(bar)) goto timeout;
    {
        const uint32_t T = __ldcg(rb.n_touched);
        if (blockIdx.x == 0 && threadIdx.x == 0) rb.n_touched[7] = T;
        bucket_alloc(rb, T);
        if (!grid_barrier(bar)) goto timeout;
        bucket_scatter(rb, a);
        if (!grid_barrier(bar)) goto timeout;
        CommitSmem &sm = *reinterpret_cast<CommitSmem *>(commit_smem);
        // the sub-round's factors into shared memory, then warp 0 folds the
        // large buckets while the other warps fold the small ones
        stage_factors(rb, a, sm);
        if (threadIdx.x < 32) apply_large(rb, jc, jr, a, sm);
        else apply_small(rb, jc, jr, a, T, sm);
        __syncthreads();
        commit_sums(rb, jc, a);
        // the scatter cursors back to zero for the next round
        for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T;
             t += gridDim.x * blockDim.x)
            rb.node_cnt[rb.touched[t]] = 0;
    }
    commit_exit(rb);
    return;
timeout:
    if (threadIdx.x == 0) atomicCAS(&jc.sc->error, 0, SILVAN_E_TIMEOUT);
    commit_exit(rb);
}

int g_commit_grid = 0;  // resident CTAs of commit_round_kernel (apply_init)

}  // namespace

cudaError_t apply_init() {
    cudaError_t e = cudaFuncSetAttribute(commit_round_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kCommitSmem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, commit_round_kernel,
                                                      kCommitThreads, kCommitSmem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorLaunchOutOfResources;
    g_commit_grid = sms * per_sm;
    return cudaSuccess;
}

// One warp per node of the round's touched list, lanes as in the fold.
__global__ void undo_round_kernel(RoundBuffers rb, JobCounters jc, RoundJournal jr, int pass,
                                  uint32_t D) {
    const uint32_t T = __ldcg(rb.n_touched + 7);
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < T; t += nw) {
        const uint32_t node = rb.touched[t];
        if (lane < kTrials) {
            if (pass == 2)
                jc.mcrade[(uint64_t)node * kTrials + lane] = jr.mcrade[(uint64_t)t * kTrials + lane];
        } else if (lane == 25) {
            jc.approx[node] = jr.approx[t];
            jc.last_upd[node] = jr.last_upd[t];
        } else if (lane == 26) {
            jc.wimpy[node] = jr.wimpy[t];
        }
    }
    if (blockIdx.x == 0) {
        const unsigned long long *src = reinterpret_cast<const unsigned long long *>(jr.sc);
        unsigned long long *dst = reinterpret_cast<unsigned long long *>(jc.sc);
        for (uint32_t i = threadIdx.x; i < sizeof(JobScalars) / 8; i += blockDim.x) dst[i] = src[i];
        for (uint32_t i = threadIdx.x; i <= D; i += blockDim.x) jc.sp_lengths[i] = jr.sp_lengths[i];
    }
}

cudaError_t apply_round(const ApplyState &st, cudaStream_t stream) {
    if (g_commit_grid <= 0) return cudaErrorNotReady;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)g_commit_grid);
    cfg.blockDim = dim3(kCommitThreads);
    cfg.dynamicSmemBytes = kCommitSmem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, commit_round_kernel, st);
}

namespace {

// Neutral accumulator: every maximum at its identity.
__global__ void stop_init_kernel(StopReduction *acc) {
    for (int i = threadIdx.x; i < kMaxPartitions * kTrials; i += blockDim.x)
        acc->mc_max[i] = LLONG_MIN;
    for (int i = threadIdx.x; i < kMaxPartitions; i += blockDim.x) {
        acc->wimpy_max[i] = 0.0;
        acc->touched[i] = 0;
    }
    if (threadIdx.x == 0) {
        acc->approx_max = 0.0;
        acc->wimpy_all_max = 0.0;
    }
}

// One warp per updated node: lanes 0..24 read the node's 25 trials (one
// 200-byte row), lane 25 approx and wimpy.  Each CTA folds its nodes in
// shared memory and into the device accumulator; the last CTA out writes the
// result, the job's scalars and the path-length counts to the (host-mapped)
// readback and leaves the accumulator neutral for the next check.
__global__ void __launch_bounds__(512) stop_reduce_kernel(JobCounters jc, int nparts, uint32_t D,
                                                          StopReduction *acc, uint32_t *ticket,
                                                          StopReadback rb) {
    __shared__ long long smc[kMaxPartitions * kTrials];
    __shared__ unsigned long long sw[kMaxPartitions];
    __shared__ uint32_t st[kMaxPartitions];
    __shared__ bool last;
    for (int i = threadIdx.x; i < nparts * kTrials; i += blockDim.x) smc[i] = LLONG_MIN;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        sw[i] = 0ull;
        st[i] = 0;
    }
    __syncthreads();
    const uint32_t T = jc.sc->n_upd;
    const int lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long amax = 0, wmax = 0;
    // kNodes nodes per warp at a time, their loads in flight together
    constexpr int kNodes = 4;
    for (uint32_t t0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t0 < T; t0 += kNodes * nw) {
        uint32_t v[kNodes];
        int p[kNodes];
        long long m[kNodes];
        unsigned long long wb[kNodes], ab[kNodes];
#pragma unroll
        for (int i = 0; i < kNodes; i++) {
            const uint32_t t = t0 + (uint32_t)i * nw;
            v[i] = t < T ? jc.upd_list[t] : 0xffffffffu;
        }
#pragma unroll
        for (int i = 0; i < kNodes; i++) {
            p[i] = 0;
            m[i] = LLONG_MIN;
            wb[i] = ab[i] = 0ull;
            if (v[i] == 0xffffffffu) continue;
            p[i] = jc.partition[v[i]];
            if (lane < kTrials) {
                m[i] = jc.mcrade[(uint64_t)v[i] * kTrials + lane];
            } else if (lane == kTrials) {
                wb[i] = (unsigned long long)__double_as_longlong(jc.wimpy[v[i]]);
                ab[i] = (unsigned long long)__double_as_longlong(jc.approx[v[i]]);
            }
        }
#pragma unroll
        for (int i = 0; i < kNodes; i++) {
            if (v[i] == 0xffffffffu) continue;
            if (lane < kTrials) {
                if (m[i] > smc[p[i] * kTrials + lane]) atomicMax(&smc[p[i] * kTrials + lane], m[i]);
            } else if (lane == kTrials) {
                if (wb[i] > sw[p[i]]) atomicMax(&sw[p[i]], wb[i]);
                atomicAdd(&st[p[i]], 1u);
                amax = ab[i] > amax ? ab[i] : amax;
                wmax = wb[i] > wmax ? wb[i] : wmax;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long x = __shfl_xor_sync(0xffffffffu, amax, o);
        unsigned long long y = __shfl_xor_sync(0xffffffffu, wmax, o);
        amax = x > amax ? x : amax;
        wmax = y > wmax ? y : wmax;
    }
    if (lane == 0) {
        if (amax) atomicMax(reinterpret_cast<unsigned long long *>(&acc->approx_max), amax);
        if (wmax) atomicMax(reinterpret_cast<unsigned long long *>(&acc->wimpy_all_max), wmax);
    }
    __syncthreads();
    // every CTA folds the same few hundred words: an atomic only where this
    // CTA's value is above the accumulator's (most are not), so that the
    // CTAs do not queue on the same addresses
    for (int i = threadIdx.x; i < nparts * kTrials; i += blockDim.x)
        if (smc[i] != LLONG_MIN && smc[i] > __ldcg(&acc->mc_max[i]))
            atomicMax(&acc->mc_max[i], smc[i]);
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        unsigned long long *wm = reinterpret_cast<unsigned long long *>(&acc->wimpy_max[i]);
        if (sw[i] && sw[i] > __ldcg(wm)) atomicMax(wm, sw[i]);
        if (st[i]) atomicAdd(&acc->touched[i], st[i]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int i = threadIdx.x; i < nparts * kTrials; i += blockDim.x) {
        rb.red->mc_max[i] = __ldcg(&acc->mc_max[i]);
        acc->mc_max[i] = LLONG_MIN;
    }
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        rb.red->wimpy_max[i] = __ldcg(&acc->wimpy_max[i]);
        rb.red->touched[i] = __ldcg(&acc->touched[i]);
        acc->wimpy_max[i] = 0.0;
        acc->touched[i] = 0;
    }
    if (threadIdx.x == 0) {
        rb.red->approx_max = __ldcg(&acc->approx_max);
        rb.red->wimpy_all_max = __ldcg(&acc->wimpy_all_max);
        acc->approx_max = 0.0;
        acc->wimpy_all_max = 0.0;
        *ticket = 0u;
    }
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(jc.sc);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(rb.sc);
    for (uint32_t i = threadIdx.x; i < sizeof(JobScalars) / 8; i += blockDim.x) dst[i] = __ldcg(&src[i]);
    if (rb.sp)
        for (uint32_t i = threadIdx.x; i <= D; i += blockDim.x) rb.sp[i] = __ldcg(&jc.sp_lengths[i]);
}

// Peeling index of node v (Probabilistic.cpp:855-862), stored in peel_idx.
// The C library's log may differ from the device's by an ulp; the nodes
// where that could move (int)t are listed so that the host recomputes them.
__device__ __forceinline__ int32_t peel_index_of(const JobCounters &jc, uint32_t v, double m,
                                                 double la, uint32_t *unc, uint32_t *n_unc,
                                                 uint32_t cap) {
    const double ew = jc.wimpy[v] / m;
    const double mi = fmin(1. / ew, m);
    const double t = log(mi) / la + 1;
    const int32_t idx = (int)t;
    jc.peel_idx[v] = idx;
    const double fr = t - floor(t);
    if (fr < 1e-9 || fr > 1.0 - 1e-9) {
        uint32_t k = atomicAdd(n_unc, 1u);
        if (k < cap) unc[k] = v;
    }
    return idx;
}

// The end of pass 1 in one kernel: with peeling (nbins > 0) every node's
// index, the uncertain list and the histogram of the indices over
// [idx_min, idx_min + nbins) (hist and n_unc zeroed before); the last CTA
// out copies the histogram, the uncertain count, the scalars and the
// path-length counts to `out` (host-mapped).
__global__ void __launch_bounds__(512) pass1_readback_kernel(
    JobCounters jc, uint32_t n, double m, double a, int32_t idx_min, int32_t nbins,
    uint32_t *hist, uint32_t *unc, uint32_t *n_unc, uint32_t cap, uint32_t D, uint32_t *ticket,
    Pass1Readback out) {
    extern __shared__ uint32_t sh[];
    __shared__ bool last;
    const bool local = nbins > 0 && nbins <= kPeelLocalBins;
    if (local)
        for (int i = threadIdx.x; i < nbins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    if (nbins > 0) {
        const double la = log(a);
        for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n;
             v += gridDim.x * blockDim.x) {
            int32_t b = peel_index_of(jc, v, m, la, unc, n_unc, cap) - idx_min;
            b = b < 0 ? 0 : (b >= nbins ? nbins - 1 : b);
            atomicAdd(local ? &sh[b] : &hist[b], 1u);
        }
    }
    __syncthreads();
    if (local)
        for (int i = threadIdx.x; i < nbins; i += blockDim.x)
            if (sh[i]) atomicAdd(&hist[i], sh[i]);
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) out.hist[i] = __ldcg(&hist[i]);
    if (threadIdx.x == 0) {
        *out.n_unc = __ldcg(n_unc);
        *ticket = 0u;
    }
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(jc.sc);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(out.sc);
    for (uint32_t i = threadIdx.x; i < sizeof(JobScalars) / 8; i += blockDim.x) dst[i] = __ldcg(&src[i]);
    for (uint32_t i = threadIdx.x; i <= D; i += blockDim.x) out.sp[i] = __ldcg(&jc.sp_lengths[i]);
}

// Zeroes approx, wimpy and last_upd of the nodes on upd_list (every node
// with a non-zero one): the counters of pass 2 start from zero.
__global__ void reset_updated_kernel(JobCounters jc) {
    const uint32_t T = jc.sc->n_upd;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        const uint32_t v = jc.upd_list[t];
        jc.approx[v] = 0.0;
        jc.wimpy[v] = 0.0;
        jc.last_upd[v] = 0u;
    }
}

// Shared-memory histogram per block (the bins are few: about log(m)/log(a)).
__global__ void peel_hist_kernel(JobCounters jc, uint32_t n, int32_t idx_min, int32_t nbins,
                                 uint32_t *hist) {
    extern __shared__ uint32_t sh[];
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        int32_t b = jc.peel_idx[v] - idx_min;
        b = b < 0 ? 0 : (b >= nbins ? nbins - 1 : b);
        atomicAdd(&sh[b], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nbins; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

__global__ void peel_hist_global_kernel(JobCounters jc, uint32_t n, int32_t idx_min,
                                        int32_t nbins, uint32_t *hist) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        int32_t b = jc.peel_idx[v] - idx_min;
        b = b < 0 ? 0 : (b >= nbins ? nbins - 1 : b);
        atomicAdd(&hist[b], 1u);
    }
}

__global__ void peel_map_kernel(JobCounters jc, uint32_t n, const int32_t *lut, int32_t idx_min,
                                int32_t lut_size) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        int32_t b = jc.peel_idx[v] - idx_min;
        b = b < 0 ? 0 : (b >= lut_size ? lut_size - 1 : b);
        jc.partition[v] = lut[b];
    }
}

}  // namespace

__global__ void divide_kernel(const double *approx, double m, double *out, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        out[v] = __ddiv_rn(approx[v], m);
}

cudaError_t undo_round(const RoundBuffers &rb, const JobCounters &jc, const RoundJournal &jr,
                       int pass, uint32_t D, cudaStream_t stream) {
    undo_round_kernel<<<296, 512, 0, stream>>>(rb, jc, jr, pass, D);
    return cudaGetLastError();
}

cudaError_t divide_estimates(const double *approx, double num_samples, double *out, uint32_t n,
                             cudaStream_t stream) {
    divide_kernel<<<592, 256, 0, stream>>>(approx, num_samples, out, n);
    return cudaGetLastError();
}

cudaError_t stop_reduce_init(StopReduction *acc, uint32_t *ticket, cudaStream_t stream) {
    stop_init_kernel<<<1, 256, 0, stream>>>(acc);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(ticket, 0, sizeof(uint32_t), stream);
}

cudaError_t stop_reduce(const JobCounters &jc, int nparts, uint32_t D, StopReduction *acc,
                        uint32_t *ticket, const StopReadback &out, cudaStream_t stream) {
    stop_reduce_kernel<<<296, 512, 0, stream>>>(jc, nparts, D, acc, ticket, out);
    return cudaGetLastError();
}

cudaError_t pass1_readback(const JobCounters &jc, uint32_t n, double num_samples, double a,
                           int32_t idx_min, int32_t nbins, uint32_t *hist, uint32_t *uncertain,
                           uint32_t *n_uncertain, uint32_t cap, uint32_t D, uint32_t *ticket,
                           const Pass1Readback &out, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(n_uncertain, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess && nbins > 0)
        e = cudaMemsetAsync(hist, 0, sizeof(uint32_t) * nbins, stream);
    if (e != cudaSuccess) return e;
    const size_t smem = nbins > 0 && nbins <= kPeelLocalBins ? sizeof(uint32_t) * nbins : 0;
    pass1_readback_kernel<<<296, 512, smem, stream>>>(jc, n, num_samples, a, idx_min, nbins, hist,
                                                      uncertain, n_uncertain, cap, D, ticket, out);
    return cudaGetLastError();
}

cudaError_t reset_updated(const JobCounters &jc, cudaStream_t stream) {
    reset_updated_kernel<<<296, 512, 0, stream>>>(jc);
    return cudaGetLastError();
}

cudaError_t peel_hist(const JobCounters &jc, uint32_t n, int32_t idx_min, int32_t nbins,
                      uint32_t *hist, cudaStream_t stream) {
    cudaMemsetAsync(hist, 0, sizeof(uint32_t) * nbins, stream);
    if (nbins <= kPeelLocalBins)
        peel_hist_kernel<<<296, 512, sizeof(uint32_t) * nbins, stream>>>(jc, n, idx_min, nbins,
                                                                          hist);
    else
        peel_hist_global_kernel<<<592, 256, 0, stream>>>(jc, n, idx_min, nbins, hist);
    return cudaGetLastError();
}

cudaError_t peel_map(const JobCounters &jc, uint32_t n, const int32_t *lut, int32_t idx_min,
                     int32_t lut_size, uint32_t *hist, cudaStream_t stream) {
    (void)hist;
    peel_map_kernel<<<592, 256, 0, stream>>>(jc, n, lut, idx_min, lut_size);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Top-K selection of the ranking (see counters.cuh).  A node's key is the
// 128-bit (approx bits, last update << 32 | node), compared as an unsigned
// number: approx is non-negative, so its bit pattern orders like its value,
// and node ids make every key distinct.  Digit i (i = 0 the most
// significant) is 16 bits of it.
// ---------------------------------------------------------------------------
namespace {

constexpr uint32_t kTopkSortCap = 8192;  // candidates one CTA sorts in shared memory

struct Key128 {
    unsigned long long hi, lo;
};

__device__ __forceinline__ Key128 node_key(const JobCounters &jc, uint32_t v) {
    Key128 k;
    k.hi = (unsigned long long)__double_as_longlong(jc.approx[v]);
    k.lo = ((unsigned long long)jc.last_upd[v] << 32) | v;
    return k;
}

// word w (0 most significant) of the key
__device__ __forceinline__ uint32_t key_word(const Key128 &k, int w) {
    const unsigned long long x = w < 2 ? k.hi : k.lo;
    return (w & 1) ? (uint32_t)x : (uint32_t)(x >> 32);
}

__device__ __forceinline__ uint32_t key_digit(const Key128 &k, uint32_t i) {
    return (key_word(k, (int)(i >> 1)) >> ((i & 1) ? 0 : 16)) & 0xffffu;
}

// -1, 0, 1: the key's first L digits against the prefix's (4 words).
__device__ __forceinline__ int cmp_prefix(const Key128 &k, const uint32_t *pre, uint32_t L) {
    for (uint32_t w = 0; w < 4 && 2 * w < L; w++) {
        const uint32_t mask = (2 * w + 1 < L) ? 0xffffffffu : 0xffff0000u;
        const uint32_t a = key_word(k, (int)w) & mask, b = pre[w] & mask;
        if (a != b) return a < b ? -1 : 1;
    }
    return 0;
}

// state: [0] digits fixed (L), [1..4] prefix words, [5] nodes known to be
// above the prefix's group, [6] size of the group, [7] candidates
__global__ void topk_hist_kernel(JobCounters jc, uint32_t n_upd, const uint32_t *state,
                                 uint32_t *hist) {
    const uint32_t L = state[0];
    uint32_t pre[4] = {state[1], state[2], state[3], state[4]};
    const int lane = threadIdx.x & 31;
    for (uint32_t t0 = blockIdx.x * blockDim.x; t0 < n_upd; t0 += gridDim.x * blockDim.x) {
        const uint32_t t = t0 + threadIdx.x;
        bool in = false;
        uint32_t d = 0;
        if (t < n_upd) {
            const Key128 k = node_key(jc, jc.upd_list[t]);
            in = cmp_prefix(k, pre, L) == 0;
            d = key_digit(k, L);
        }
        // one atomic per distinct digit of the warp
        const uint32_t act = __ballot_sync(0xffffffffu, in);
        if (in) {
            const uint32_t peers = __match_any_sync(act, d);
            if ((peers & ((1u << lane) - 1u)) == 0u) atomicAdd(&hist[d], (uint32_t)__popc(peers));
        }
    }
}

// One CTA of 1024 threads: the digit d of level L at which the K-th key lies
// (counting from the largest), the count above it, and the state of the
// next level (its prefix extended by d).
__global__ void __launch_bounds__(1024) topk_pick_kernel(const uint32_t *hist, uint32_t *state,
                                                         uint32_t K) {
    __shared__ uint32_t ws[32];
    __shared__ uint32_t found;
    const uint32_t L = state[0], above = state[5];
    const uint32_t t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    // thread t owns digits [hi - 63, hi], hi = 65535 - 64 t (descending)
    const uint32_t top = 65535u - 64u * t;
    uint32_t sum = 0;
    for (int j = 0; j < 64; j++) sum += hist[top - j];
    uint32_t incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
    }
    if (lane == 31) ws[warp] = incl;
    if (t == 0) found = 0;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = ws[lane];
        uint32_t wi = w;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += x;
        }
        ws[lane] = wi - w;
    }
    __syncthreads();
    uint32_t before = above + ws[warp] + incl - sum;  // keys above this thread's digits
    if (before < K && before + sum >= K) {
        for (int j = 0; j < 64; j++) {
            const uint32_t h = hist[top - j];
            if (before + h >= K) {
                const uint32_t d = top - j;
                const uint32_t w = L >> 1;
                state[1 + w] |= (L & 1) ? d : (d << 16);
                state[0] = L + 1;
                state[5] = before;
                state[6] = h;
                found = 1;
                break;
            }
            before += h;
        }
    }
    __syncthreads();
    if (t == 0 && !found) state[0] = 0xffffffffu;  // fewer than K keys: cannot happen
}

// Every updated node whose first L digits are at least the prefix's.
__global__ void topk_collect_kernel(JobCounters jc, uint32_t n_upd, uint32_t *state,
                                    unsigned long long *cand, uint32_t cap) {
    const uint32_t L = state[0];
    uint32_t pre[4] = {state[1], state[2], state[3], state[4]};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n_upd;
         t += gridDim.x * blockDim.x) {
        const Key128 k = node_key(jc, jc.upd_list[t]);
        if (cmp_prefix(k, pre, L) >= 0) {
            const uint32_t i = atomicAdd(&state[7], 1u);
            if (i < cap) {
                cand[2 * i] = k.hi;
                cand[2 * i + 1] = k.lo;
            }
        }
    }
}

// One CTA: bitonic sort of the n <= kTopkSortCap candidates, largest first,
// in shared memory; the sorted keys go back to cand.
__global__ void __launch_bounds__(1024) topk_sort_kernel(unsigned long long *cand,
                                                         const uint32_t *state) {
    extern __shared__ unsigned long long kv[];  // 2 x P words
    const uint32_t n = state[7];
    uint32_t P = 64;
    while (P < n) P <<= 1;
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
        kv[2 * i] = i < n ? cand[2 * i] : 0ull;
        kv[2 * i + 1] = i < n ? cand[2 * i + 1] : 0ull;
    }
    __syncthreads();
    for (uint32_t k = 2; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const unsigned long long ah = kv[2 * i], al = kv[2 * i + 1];
                    const unsigned long long bh = kv[2 * l], bl = kv[2 * l + 1];
                    const bool a_less = ah < bh || (ah == bh && al < bl);
                    const bool desc = (i & k) == 0;
                    if (desc ? a_less : !a_less) {
                        kv[2 * i] = bh;
                        kv[2 * i + 1] = bl;
                        kv[2 * l] = ah;
                        kv[2 * l + 1] = al;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        cand[2 * i] = kv[2 * i];
        cand[2 * i + 1] = kv[2 * i + 1];
    }
}

}  // namespace

uint32_t topk_capacity(uint32_t K) { return std::max<uint32_t>(kTopkSortCap, 2u * K); }

int topk_select(const JobCounters &jc, uint32_t n_upd, uint32_t K, const TopkBuffers &tb,
                cudaStream_t stream, uint32_t *nodes, double *values, uint32_t *count) {
    *count = 0;
    if (n_upd == 0 || K == 0) return SILVAN_OK;
    if (tb.cap < topk_capacity(K)) return SILVAN_E_BADARG;
    static bool attr_set = false;  // the sort kernel's shared memory (once per process)
    if (!attr_set) {
        if (cudaFuncSetAttribute(topk_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(2 * kTopkSortCap * sizeof(unsigned long long))) !=
            cudaSuccess)
            return SILVAN_E_CUDA;
        attr_set = true;
    }
    uint32_t *hs = tb.h_state;
    for (int i = 0; i < 8; i++) hs[i] = 0;
    if (cudaMemcpyAsync(tb.state, hs, 8 * sizeof(uint32_t), cudaMemcpyHostToDevice, stream) !=
        cudaSuccess)
        return SILVAN_E_CUDA;
    // refine while the candidates (keys at or above the prefix) would not fit
    uint32_t ncand = n_upd;
    while (ncand > tb.cap) {
        if (cudaMemsetAsync(tb.hist, 0, 65536 * sizeof(uint32_t), stream) != cudaSuccess)
            return SILVAN_E_CUDA;
        topk_hist_kernel<<<592, 256, 0, stream>>>(jc, n_upd, tb.state, tb.hist);
        topk_pick_kernel<<<1, 1024, 0, stream>>>(tb.hist, tb.state, K);
        if (cudaMemcpyAsync(hs, tb.state, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return SILVAN_E_CUDA;
        if (hs[0] > 8) return SILVAN_E_STATE;
        ncand = hs[5] + hs[6];
        if (hs[0] == 8 && ncand > tb.cap) return SILVAN_E_STATE;  // keys are distinct
    }
    topk_collect_kernel<<<592, 256, 0, stream>>>(jc, n_upd, tb.state, tb.cand, tb.cap);
    if (cudaMemcpyAsync(hs, tb.state, 8 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return SILVAN_E_CUDA;
    const uint32_t n = hs[7];
    if (n > tb.cap || n < std::min(K, n_upd)) return SILVAN_E_STATE;
    const uint32_t take = std::min(K, n);
    if (n <= kTopkSortCap) {
        topk_sort_kernel<<<1, 1024, 2 * kTopkSortCap * sizeof(unsigned long long), stream>>>(
            tb.cand, tb.state);
        if (cudaMemcpyAsync(tb.h_cand, tb.cand, 2 * sizeof(unsigned long long) * take,
                            cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return SILVAN_E_CUDA;
    } else {
        // more than one CTA sorts: the (at most 2K) candidates are ordered on
        // the host, still without any n-sized transfer
        if (cudaMemcpyAsync(tb.h_cand, tb.cand, 2 * sizeof(unsigned long long) * n,
                            cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return SILVAN_E_CUDA;
        std::vector<uint32_t> ord(n);
        for (uint32_t i = 0; i < n; i++) ord[i] = i;
        const unsigned long long *c = tb.h_cand;
        std::partial_sort(ord.begin(), ord.begin() + take, ord.end(), [&](uint32_t x, uint32_t y) {
            return c[2 * x] != c[2 * y] ? c[2 * x] > c[2 * y] : c[2 * x + 1] > c[2 * y + 1];
        });
        std::vector<unsigned long long> tmp(2 * (size_t)take);
        for (uint32_t i = 0; i < take; i++) {
            tmp[2 * i] = c[2 * ord[i]];
            tmp[2 * i + 1] = c[2 * ord[i] + 1];
        }
        std::copy(tmp.begin(), tmp.end(), tb.h_cand);
    }
    for (uint32_t i = 0; i < take; i++) {
        nodes[i] = (uint32_t)tb.h_cand[2 * i + 1];
        std::memcpy(&values[i], &tb.h_cand[2 * i], sizeof(double));
    }
    *count = take;
    return SILVAN_OK;
}

}  // namespace silvan
