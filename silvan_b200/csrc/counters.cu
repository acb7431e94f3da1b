// Ordered commit of sample contributions (see counters.cuh).
//
// The reference adds every sample's path map to the per-node counters inside
// one critical section, in sample order (silvan/src/Probabilistic.cpp:479-544):
//   x = count * (1 / num_paths)
//   approx[u] += x;  emp_wimpy_vars[u] += x * x;
//   mcrade[u][j] = (int64)((double)mcrade[u][j] + sign_j * x)   (truncation)
// With num_paths > 1 the additions are not associative, so a node's updates
// must be applied in sample order.  A round's records are grouped by node
// (count, scan, scatter), each node's group is sorted by sample index (a warp
// bitonic sort for groups of <= 32, a CTA sort in shared memory otherwise)
// and the group is folded sequentially: lanes 0..24 each carry one Monte
// Carlo trial, lane 25 approx, lane 26 the wimpy variance.  Different nodes
// are independent, so the only serial work is per node.
#include <cfloat>

#include "counters.cuh"

namespace silvan {

namespace {

constexpr int kScanBlocks = 296;
constexpr int kScanThreads = 256;

__device__ __forceinline__ uint32_t round_records(const RoundBuffers &rb, const ApplyArgs &a) {
    return (uint32_t)min((uint64_t)a.n_records, rb.rec_cap);
}

// The Rademacher signs of the round's samples (pass 2), and the records per
// node with the list of touched nodes.
__global__ void bucket_count_kernel(const ApplyState *st) {
    const RoundBuffers rb = st->rb;
    const ApplyArgs a = st->a;
    if (a.pass == 2)
        for (uint32_t s = a.lo + blockIdx.x * blockDim.x + threadIdx.x; s < a.hi;
             s += gridDim.x * blockDim.x)
            rb.signs[s] = rademacher_mask(a.seed, a.first_sample + s);
    const uint32_t R = round_records(rb, a);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x) {
        PathRec r = rb.recs[i];
        if (r.sample < a.lo || r.sample >= a.hi) continue;
        if (atomicAdd(&rb.node_cnt[r.node], 1u) == 0u) {
            uint32_t t = atomicAdd(rb.n_touched, 1u);
            rb.touched[t] = r.node;
        }
    }
}

// Three-step exclusive scan of node_cnt over the touched list; each block owns
// a contiguous range of the list.
__device__ __forceinline__ void range_of(uint32_t T, uint32_t &b, uint32_t &e) {
    uint32_t per = (T + gridDim.x - 1) / gridDim.x;
    b = min(T, blockIdx.x * per);
    e = min(T, b + per);
}

__device__ uint32_t block_sum(uint32_t v, uint32_t *tmp) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) tmp[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t t = 0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += tmp[w];
        tmp[0] = t;
    }
    __syncthreads();
    t = tmp[0];
    __syncthreads();
    return t;
}

__global__ void scan_reduce_kernel(const ApplyState *st) {
    __shared__ uint32_t tmp[32];
    const RoundBuffers rb = st->rb;
    const uint32_t T = *rb.n_touched;
    uint32_t b, e;
    range_of(T, b, e);
    uint32_t s = 0;
    for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x) s += rb.node_cnt[rb.touched[i]];
    s = block_sum(s, tmp);
    if (threadIdx.x == 0) rb.block_sums[blockIdx.x] = s;
}

// One warp: exclusive scan of the block sums, 32 at a time.
__global__ void scan_top_kernel(const ApplyState *st, int nblocks) {
    const RoundBuffers rb = st->rb;
    const int lane = threadIdx.x & 31;
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    uint32_t acc = 0;
    for (int i0 = 0; i0 < nblocks; i0 += 32) {
        const int i = i0 + lane;
        const uint32_t v = i < nblocks ? rb.block_sums[i] : 0u;
        uint32_t incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (i < nblocks) rb.block_sums[i] = acc + incl - v;
        acc += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) rb.block_sums[nblocks] = acc;
}

__global__ void scan_down_kernel(const ApplyState *st) {
    __shared__ uint32_t tmp[33];
    const RoundBuffers rb = st->rb;
    const uint32_t T = *rb.n_touched;
    uint32_t b, e;
    range_of(T, b, e);
    uint32_t carry = rb.block_sums[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t c0 = b; c0 < e; c0 += blockDim.x) {
        uint32_t i = c0 + threadIdx.x;
        uint32_t node = 0, v = 0;
        if (i < e) {
            node = rb.touched[i];
            v = rb.node_cnt[node];
        }
        uint32_t incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) tmp[warp] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (int w = 0; w < nw; w++) {
                uint32_t t = tmp[w];
                tmp[w] = acc;
                acc += t;
            }
            tmp[32] = acc;
        }
        __syncthreads();
        const uint32_t excl = carry + tmp[warp] + incl - v;
        if (i < e) {
            rb.bucket_off[i] = excl;
            rb.node_cnt[node] = excl;  // becomes the scatter cursor
        }
        carry += tmp[32];
        __syncthreads();
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) rb.bucket_off[T] = rb.block_sums[gridDim.x];
}

__global__ void bucket_scatter_kernel(const ApplyState *st) {
    const RoundBuffers rb = st->rb;
    const ApplyArgs a = st->a;
    const uint32_t R = round_records(rb, a);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x) {
        PathRec r = rb.recs[i];
        if (r.sample < a.lo || r.sample >= a.hi) continue;
        uint32_t pos = atomicAdd(&rb.node_cnt[r.node], 1u);
        rb.entries[pos] = ((unsigned long long)r.sample << 32) | r.count;
    }
}

__device__ __forceinline__ void atomic_max_nonneg_double(unsigned long long *p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// Sequential fold of one node's sorted contributions.  Lane j < 25 carries
// trial j of mcrade, lane 25 approx (and the top-k mark), lane 26 the wimpy
// variance.  get(r) returns the r-th (sample << 32 | count) entry.  Entries
// are prepared 32 at a time by all lanes (x = count * (1/num_paths) and the
// sample's signs, into the warp's shared scratch) so that the sequential
// chains only read shared memory.
struct FoldScratch {
    double x[32];
    uint32_t signs[32];
    uint32_t sample[32];
};

template <typename Get>
__device__ void fold_node(const RoundBuffers &rb, const JobCounters &jc, const ApplyArgs &a,
                          uint32_t node, uint32_t b, Get get, FoldScratch &fs) {
    const int lane = threadIdx.x & 31;
    const bool pass2 = a.pass == 2;
    long long m = 0;
    double acc = 0.0;
    uint32_t lu = 0;
    if (lane < kTrials) {
        if (pass2) m = jc.mcrade[(uint64_t)node * kTrials + lane];
    } else if (lane == 25) {
        acc = jc.approx[node];
        lu = jc.last_upd[node];
    } else if (lane == 26) {
        acc = jc.wimpy[node];
    }
    bool crossed = a.track_cross ? jc.cross_flag[node] != 0 : true;
    for (uint32_t r0 = 0; r0 < b; r0 += 32) {
        const uint32_t r = r0 + lane;
        if (r < b) {
            const unsigned long long e = get(r);
            const uint32_t sl = (uint32_t)(e >> 32);
            const uint32_t c = (uint32_t)e;
            fs.x[lane] = __dmul_rn((double)c, __ddiv_rn(1.0, (double)rb.np[sl]));
            fs.signs[lane] = pass2 ? rb.signs[sl] : 0u;
            fs.sample[lane] = sl;
        }
        __syncwarp();
        const uint32_t kmax = min(32u, b - r0);
        if (lane < kTrials) {
            if (pass2) {
                for (uint32_t k = 0; k < kmax; k++) {
                    const double x = fs.x[k];
                    const bool plus = (fs.signs[k] >> lane) & 1u;
                    m = (long long)__double2ll_rz(__dadd_rn(__ll2double_rn(m), plus ? x : -x));
                }
            }
        } else if (lane == 25) {
            for (uint32_t k = 0; k < kmax; k++) {
                const double x = fs.x[k];
                if (x > 0.) {
                    acc = __dadd_rn(acc, x);
                    lu = a.first_sample + fs.sample[k] + 1u;
                    if (!crossed && acc >= 3.0) {
                        crossed = true;
                        jc.cross_flag[node] = 1;
                        const uint32_t q = atomicAdd(&jc.sc->n_cross, 1u);
                        jc.cross_sample[q] = a.first_sample + fs.sample[k];
                    }
                }
            }
        } else if (lane == 26) {
            for (uint32_t k = 0; k < kmax; k++) {
                const double x = fs.x[k];
                if (x > 0.) acc = __dadd_rn(acc, __dmul_rn(x, x));
            }
        }
        __syncwarp();
    }
    if (lane < kTrials) {
        if (pass2) jc.mcrade[(uint64_t)node * kTrials + lane] = m;
    } else if (lane == 25) {
        jc.approx[node] = acc;
        if (lu) {
            if (jc.last_upd[node] == 0) jc.upd_list[atomicAdd(&jc.sc->n_upd, 1u)] = node;
            jc.last_upd[node] = lu;
        }
        atomic_max_nonneg_double(&jc.sc->sup_approx_bits, acc);
    } else if (lane == 26) {
        jc.wimpy[node] = acc;
        atomic_max_nonneg_double(&jc.sc->sup_wimpy_bits, acc);
    }
}

__device__ __forceinline__ void warp_bitonic_sort(unsigned long long &key) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, j);
            const bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
            key = take_min ? (key < o ? key : o) : (key > o ? key : o);
        }
    }
}

constexpr int kApplyThreads = 256;

// Groups of at most 32 entries: one warp per node.
__global__ void __launch_bounds__(kApplyThreads) apply_small_kernel(const ApplyState *st) {
    __shared__ unsigned long long buf[kApplyThreads / 32][32];
    __shared__ FoldScratch fsc[kApplyThreads / 32];
    const RoundBuffers rb = st->rb;
    const JobCounters jc = st->jc;
    const ApplyArgs a = st->a;
    const uint32_t T = *rb.n_touched;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + wib;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);
    for (uint32_t t = gw; t < T; t += nw) {
        const uint32_t b0 = rb.bucket_off[t];
        const uint32_t b = rb.bucket_off[t + 1] - b0;
        if (b > 32) {
            // for apply_large, which then visits only these
            if (lane == 0) rb.large[atomicAdd(rb.n_large, 1u)] = t;
            continue;
        }
        const uint32_t node = rb.touched[t];
        unsigned long long key = (uint32_t)lane < b ? rb.entries[b0 + lane] : ~0ull;
        warp_bitonic_sort(key);
        buf[wib][lane] = key;
        __syncwarp();
        fold_node(rb, jc, a, node, b, [&](uint32_t r) { return buf[wib][r]; }, fsc[wib]);
        __syncwarp();
    }
}

// Groups of more than 32 entries: one CTA per node, bitonic sort in shared
// memory (groups are bounded by kLargeBucket through the sub-round size).
__global__ void __launch_bounds__(1024) apply_large_kernel(const ApplyState *st) {
    extern __shared__ unsigned long long sbuf[];
    __shared__ FoldScratch fsc;
    const RoundBuffers rb = st->rb;
    const JobCounters jc = st->jc;
    const ApplyArgs a = st->a;
    const uint32_t NL = *rb.n_large;
    for (uint32_t li = blockIdx.x; li < NL; li += gridDim.x) {
        const uint32_t t = rb.large[li];
        const uint32_t b0 = rb.bucket_off[t];
        const uint32_t b = rb.bucket_off[t + 1] - b0;
        if (b > kLargeBucket) {
            if (threadIdx.x == 0) atomicCAS(&jc.sc->error, 0, SILVAN_E_CAPACITY);
            continue;
        }
        uint32_t P = 64;
        while (P < b) P <<= 1;
        for (uint32_t i = threadIdx.x; i < P; i += blockDim.x)
            sbuf[i] = i < b ? rb.entries[b0 + i] : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= P; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                    const uint32_t l = i ^ j;
                    if (l > i) {
                        const unsigned long long x = sbuf[i], y = sbuf[l];
                        const bool asc = (i & k) == 0;
                        if (asc ? (x > y) : (x < y)) {
                            sbuf[i] = y;
                            sbuf[l] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        if (threadIdx.x < 32) {
            const uint32_t node = rb.touched[t];
            fold_node(rb, jc, a, node, b, [&](uint32_t r) { return sbuf[r]; }, fsc);
        }
        __syncthreads();
    }
}

__device__ void commit_sums(const ApplyState *st) {
    const RoundBuffers rb = st->rb;
    const JobCounters jc = st->jc;
    const ApplyArgs a = st->a;
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
    if ((threadIdx.x & 31) == 0) {
        if (vis) atomicAdd(&jc.sc->vis_edges, vis);
        if (cnt) atomicAdd(&jc.sc->counted_samples, cnt);
        if (vd) atomicAdd(&jc.sc->void_samples, vd);
        if (paths) atomicAdd(&jc.sc->paths, paths);
        if (ball) atomicAdd(&jc.sc->ball_nodes, ball);
        if (pred) atomicAdd(&jc.sc->pred_entries, pred);
    }
}

// The round's scalar sums (commit_sums) and the per-node cursors zeroed for
// the next round; neither depends on the folds.
__global__ void commit_kernel(const ApplyState *st) {
    commit_sums(st);
    const RoundBuffers rb = st->rb;
    const uint32_t T = *rb.n_touched;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        rb.node_cnt[rb.touched[t]] = 0;
}

__global__ void stop_init_kernel(StopReduction *out, int nparts, long long init) {
    for (int i = threadIdx.x; i < nparts * kTrials; i += blockDim.x) out->mc_max[i] = init;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        out->wimpy_max[i] = 0.0;
        out->touched[i] = 0;
    }
    if (threadIdx.x == 0) {
        out->approx_max = 0.0;
        out->wimpy_all_max = 0.0;
    }
}

// One warp per updated node: lanes 0..24 read the node's 25 trials (one
// 200-byte row), lane 25 approx and wimpy.
__global__ void __launch_bounds__(512) stop_reduce_kernel(JobCounters jc, int nparts,
                                                          long long init, StopReduction *out) {
    __shared__ long long smc[kMaxPartitions * kTrials];
    __shared__ unsigned long long sw[kMaxPartitions];
    __shared__ uint32_t st[kMaxPartitions];
    for (int i = threadIdx.x; i < nparts * kTrials; i += blockDim.x) smc[i] = init;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        sw[i] = 0ull;
        st[i] = 0;
    }
    __syncthreads();
    const uint32_t T = jc.sc->n_upd;
    const int lane = threadIdx.x & 31;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    unsigned long long amax = 0, wmax = 0;
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < T; t += nw) {
        const uint32_t v = jc.upd_list[t];
        const int p = jc.partition[v];
        if (lane < kTrials) {
            const long long m = jc.mcrade[(uint64_t)v * kTrials + lane];
            if (m > smc[p * kTrials + lane]) atomicMax(&smc[p * kTrials + lane], m);
        } else if (lane == kTrials) {
            const unsigned long long wb = (unsigned long long)__double_as_longlong(jc.wimpy[v]);
            const unsigned long long ab = (unsigned long long)__double_as_longlong(jc.approx[v]);
            if (wb > sw[p]) atomicMax(&sw[p], wb);
            atomicAdd(&st[p], 1u);
            amax = ab > amax ? ab : amax;
            wmax = wb > wmax ? wb : wmax;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long x = __shfl_xor_sync(0xffffffffu, amax, o);
        unsigned long long y = __shfl_xor_sync(0xffffffffu, wmax, o);
        amax = x > amax ? x : amax;
        wmax = y > wmax ? y : wmax;
    }
    if (lane == 0) {
        if (amax) atomicMax(reinterpret_cast<unsigned long long *>(&out->approx_max), amax);
        if (wmax) atomicMax(reinterpret_cast<unsigned long long *>(&out->wimpy_all_max), wmax);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nparts * kTrials; i += blockDim.x)
        if (smc[i] != init) atomicMax(&out->mc_max[i], smc[i]);
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
        if (sw[i]) atomicMax(reinterpret_cast<unsigned long long *>(&out->wimpy_max[i]), sw[i]);
        if (st[i]) atomicAdd(&out->touched[i], st[i]);
    }
}

__global__ void peel_index_kernel(JobCounters jc, uint32_t n, double m, double a, uint32_t *unc,
                                  uint32_t *n_unc, uint32_t cap) {
    const double la = log(a);
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const double ew = jc.wimpy[v] / m;
        const double mi = fmin(1. / ew, m);
        const double t = log(mi) / la + 1;
        jc.peel_idx[v] = (int)t;
        // the C library's log may differ from the device's by an ulp; flag the
        // nodes where that could move (int)t so the host recomputes them
        const double fr = t - floor(t);
        if (fr < 1e-9 || fr > 1.0 - 1e-9) {
            uint32_t k = atomicAdd(n_unc, 1u);
            if (k < cap) unc[k] = v;
        }
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

cudaError_t apply_init() {
    return cudaFuncSetAttribute(apply_large_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(kLargeBucket * sizeof(unsigned long long)));
}

cudaError_t apply_round(const ApplyState *st, uint32_t *n_touched, cudaStream_t stream) {
    cudaMemsetAsync(n_touched, 0, 2 * sizeof(uint32_t), stream);  // n_touched, n_large
    bucket_count_kernel<<<592, 256, 0, stream>>>(st);
    scan_reduce_kernel<<<kScanBlocks, kScanThreads, 0, stream>>>(st);
    scan_top_kernel<<<1, 32, 0, stream>>>(st, kScanBlocks);
    scan_down_kernel<<<kScanBlocks, kScanThreads, 0, stream>>>(st);
    bucket_scatter_kernel<<<592, 256, 0, stream>>>(st);
    apply_small_kernel<<<592, kApplyThreads, 0, stream>>>(st);
    apply_large_kernel<<<148, 1024, kLargeBucket * sizeof(unsigned long long), stream>>>(st);
    commit_kernel<<<148, 256, 0, stream>>>(st);
    return cudaGetLastError();
}

__global__ void divide_kernel(const double *approx, double m, double *out, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        out[v] = __ddiv_rn(approx[v], m);
}

cudaError_t divide_estimates(const double *approx, double num_samples, double *out, uint32_t n,
                             cudaStream_t stream) {
    divide_kernel<<<592, 256, 0, stream>>>(approx, num_samples, out, n);
    return cudaGetLastError();
}

cudaError_t stop_reduce(const JobCounters &jc, int nparts, long long init,
                        StopReduction *out_dev, cudaStream_t stream) {
    stop_init_kernel<<<1, 256, 0, stream>>>(out_dev, nparts, init);
    stop_reduce_kernel<<<296, 512, 0, stream>>>(jc, nparts, init, out_dev);
    return cudaGetLastError();
}

cudaError_t peel_index(const JobCounters &jc, uint32_t n, double num_samples, double a,
                       uint32_t *uncertain, uint32_t *n_uncertain, uint32_t cap,
                       cudaStream_t stream) {
    cudaMemsetAsync(n_uncertain, 0, sizeof(uint32_t), stream);
    peel_index_kernel<<<592, 256, 0, stream>>>(jc, n, num_samples, a, uncertain, n_uncertain, cap);
    return cudaGetLastError();
}

cudaError_t peel_hist(const JobCounters &jc, uint32_t n, int32_t idx_min, int32_t nbins,
                      uint32_t *hist, cudaStream_t stream) {
    cudaMemsetAsync(hist, 0, sizeof(uint32_t) * nbins, stream);
    if (nbins <= 8192)
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

cudaError_t ranking_candidates(const JobCounters &, uint32_t, double, uint32_t *, uint32_t *,
                               uint32_t, cudaStream_t) {
    return cudaErrorNotSupported;
}

}  // namespace silvan
