// hj_partition.cu - radix-partitioned join (phj_radix_bc / phj_radix_lp) on sm_100a.
//
// Reference algorithm (src/algo/phj.c):
//   pass 1  parallel_radix_partition / _optimized (phj.c:147-215, 257-360): per-thread histogram of
//           digit (key & (F1-1)), cross-thread prefix, stable scatter into padded partitions through
//           software write-combining buffers.
//   pass 2  serial_radix_partition -> radix_cluster (phj.c:366-491): each pass-1 partition re-clustered
//           on (key >> b1) & (F2-1), again stable; a join task per non-empty (R_p, S_p) pair.
//   join    bc_join (phj.c:496-571): bucket[next_pow_2(|R_p|)] + next[|R_p|] chains, every equal key
//           counted; lp_join (phj.c:574-680): open addressing, the probe stops at the first equal key,
//           which is the first R tuple of the partition in input order.
//
// B200 pipeline (all on one stream, no host round trip):
//   hist_kernel     one read of R and S: joint histogram of the low B key bits in shared memory
//   plan_kernel     exclusive scans -> final partition starts, pass segment tables, join work items
//   scatter_kernel  per pass: persistent CTAs take 2048-tuple tiles in order, rank tuples per digit with
//                   warp match (stable), publish per-digit counts and resolve the tile's output offsets
//                   with a decoupled look-back over predecessor tiles, stage the tile in shared memory
//                   sorted by digit and write each digit run with coalesced 16-byte streaming stores
//                   (the shared-memory analogue of the reference's SWWCB + non-temporal flush)
//   join_small      persistent CTAs take (partition, S chunk) items; R_p arrives in shared memory by one
//                   TMA bulk copy; the bucket chains (u16 head/next) are built with shared-memory atomics;
//                   S is streamed with evict-first vector loads
//   join_large_*    partitions whose R side exceeds shared memory: chains in global memory
#include <cstdio>

#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {

// ------------------------------------------------------------------------------------------------
// Device-side plan structures
// ------------------------------------------------------------------------------------------------
struct Seg {
    const tuple_v *in;
    tuple_v *out;
    uint64_t count;
    uint64_t out_len;     // bound for output indices
    uint32_t first_tile;  // first global tile of this segment
    uint32_t pad;
};

struct JoinItem {
    uint64_t r_begin;  // index into the final R buffer
    uint64_t s_begin;  // index into the final S buffer
    uint32_t r_len;
    uint32_t s_len;
    uint32_t pad[2];
};

struct LargePart {
    uint64_t r_begin, s_begin;
    uint64_t r_len, s_len;
    uint64_t table_off;  // u32 words into the large table: head[nb] then next[r_len]
    uint64_t r_flat, s_flat;
    uint32_t nb_log;
    uint32_t pad;
};

// counters[] slots
enum : int {
    kCtrTile1 = 0,
    kCtrTile2 = 1,
    kCtrNTiles1 = 2,
    kCtrNTiles2 = 3,
    kCtrNSegs1 = 4,
    kCtrNSegs2 = 5,
    kCtrNItems = 6,
    kCtrNLarge = 7,
    kCtrItem = 8,
    kCtrLargeR = 9,      // total R tuples in large partitions (u32 pairs: lo, hi)
    kCtrLargeS = 11,     // total S tuples in large partitions (lo, hi)
    kCtrLargeWords = 13, // table words used (lo, hi)
    kCtrErr = 15,
    kNumCounters = 16
};

constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;
constexpr int kSpinLimit = 1 << 22;

__device__ __forceinline__ uint64_t ld_u64_pair(const uint32_t *p) {
    return (uint64_t)p[0] | ((uint64_t)p[1] << 32);
}
__device__ __forceinline__ void st_u64_pair(uint32_t *p, uint64_t v) {
    p[0] = (uint32_t)v;
    p[1] = (uint32_t)(v >> 32);
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t *p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__host__ __device__ __forceinline__ uint32_t ceil_div_u64(uint64_t a, uint64_t b) {
    return (uint32_t)((a + b - 1) / b);
}

__device__ __forceinline__ uint32_t next_pow2_u32(uint32_t x) {
    return x <= 1 ? 1u : 1u << (32 - __clz(x - 1));
}

// ------------------------------------------------------------------------------------------------
// 1. Histogram of the low `bits` key bits over R (blocks [0, gR)) and S (blocks [gR, grid)).
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) hist_kernel(const tuple_v *__restrict__ R, size_t nR,
                                                    const tuple_v *__restrict__ S, size_t nS, int bits,
                                                    uint32_t *__restrict__ hist, int gR) {
    extern __shared__ uint32_t sh_hist[];
    const int nbins = 1 << bits;
    const uint64_t mask = (uint64_t)nbins - 1;
    const int rel = (int)blockIdx.x < gR ? 0 : 1;
    const int b = rel ? (int)blockIdx.x - gR : (int)blockIdx.x;
    const int G = rel ? (int)gridDim.x - gR : gR;
    const tuple_v *in = rel ? S : R;
    const size_t n = rel ? nS : nR;
    for (int v = threadIdx.x; v < nbins; v += blockDim.x) sh_hist[v] = 0;
    __syncthreads();
    const size_t chunk = (n + G - 1) / G;
    const size_t lo = (size_t)b * chunk;
    const size_t hi = lo + chunk < n ? lo + chunk : n;
    const size_t step = (size_t)blockDim.x;
    size_t i = lo + threadIdx.x;
    for (; i + 3 * step < hi; i += 4 * step) {
        tuple_v t0 = ld_stream(in + i), t1 = ld_stream(in + i + step);
        tuple_v t2 = ld_stream(in + i + 2 * step), t3 = ld_stream(in + i + 3 * step);
        atomicAdd(&sh_hist[t0.x & mask], 1u);
        atomicAdd(&sh_hist[t1.x & mask], 1u);
        atomicAdd(&sh_hist[t2.x & mask], 1u);
        atomicAdd(&sh_hist[t3.x & mask], 1u);
    }
    for (; i < hi; i += step) atomicAdd(&sh_hist[ld_stream(in + i).x & mask], 1u);
    __syncthreads();
    uint32_t *out = hist + (size_t)rel * nbins;
    for (int v = threadIdx.x; v < nbins; v += blockDim.x) {
        uint32_t c = sh_hist[v];
        if (c) atomicAdd(&out[v], c);
    }
}

// ------------------------------------------------------------------------------------------------
// 2. Plan: partition starts, segment tables of both passes, join work items, large partitions.
//    One CTA of 1024 threads.
// ------------------------------------------------------------------------------------------------
struct PlanArgs {
    int bits, passes, b1, F1, F2;
    const tuple_v *R, *S;
    uint64_t nR, nS;
    const uint32_t *hist;
    uint64_t *start;
    Seg *segs;        // [2][kMaxPass2Segs + 1]
    uint64_t *obase;  // [2][kMaxPass2Segs][256]
    uint32_t *counters;
    tuple_v *tmp1, *tmp2;
    JoinItem *items;
    uint64_t max_items;
    LargePart *large;
    uint64_t max_large;
    uint64_t large_table_words;
};

__device__ __forceinline__ uint32_t part_to_value(int f, int passes, int b1, int F2) {
    if (passes == 1) return (uint32_t)f;
    const uint32_t d1 = (uint32_t)f / (uint32_t)F2, d2 = (uint32_t)f % (uint32_t)F2;
    return d1 | (d2 << b1);
}

__global__ void __launch_bounds__(1024, 1) plan_kernel(PlanArgs a) {
    __shared__ uint32_t tmp[32];
    const int tid = threadIdx.x;
    const int nparts = 1 << a.bits;
    const uint64_t nrel[2] = {a.nR, a.nS};

    // Final partition starts in (d1, d2) order.
    for (int rel = 0; rel < 2; rel++) {
        uint64_t *start = a.start + (size_t)rel * (nparts + 1);
        const uint32_t *hist = a.hist + (size_t)rel * nparts;
        uint64_t running = 0;
        for (int c = 0; c < nparts; c += 1024) {
            const int f = c + tid;
            const uint32_t cnt = f < nparts ? hist[part_to_value(f, a.passes, a.b1, a.F2)] : 0u;
            uint32_t tot;
            const uint32_t ex = block_excl_scan_u32(cnt, tmp, &tot);
            if (f < nparts) start[f] = running + ex;
            running += tot;
        }
        if (tid == 0) start[nparts] = running;
    }
    __syncthreads();

    tuple_v *fin = a.passes == 2 ? a.tmp2 : a.tmp1;
    const tuple_v *inrel[2] = {a.R, a.S};
    // Pass-1 segments: one per relation.
    if (tid == 0) {
        uint32_t ft = 0;
        for (int rel = 0; rel < 2; rel++) {
            Seg s;
            s.in = inrel[rel];
            s.out = a.tmp1 + (rel ? a.nR : 0);
            s.count = nrel[rel];
            s.out_len = nrel[rel];
            s.first_tile = ft;
            s.pad = 0;
            a.segs[rel] = s;
            ft += ceil_div_u64(nrel[rel], kTile);
        }
        Seg sentinel = {};
        sentinel.first_tile = ft;
        a.segs[2] = sentinel;
        a.counters[kCtrNTiles1] = ft;
        a.counters[kCtrNSegs1] = 2;
    }
    for (int idx = tid; idx < 2 * a.F1; idx += blockDim.x) {
        const int rel = idx / a.F1, d1 = idx % a.F1;
        a.obase[(size_t)rel * 256 + d1] = a.start[(size_t)rel * (nparts + 1) + (size_t)d1 * a.F2];
    }
    // Pass-2 segments: one per (relation, pass-1 partition).
    if (a.passes == 2) {
        Seg *segs2 = a.segs + (kMaxPass2Segs + 1);
        uint64_t *obase2 = a.obase + (size_t)kMaxPass2Segs * 256;
        const int nseg = 2 * a.F1;  // <= 512 <= blockDim
        uint32_t ntile = 0;
        uint64_t b0 = 0, b1e = 0;
        int rel = 0, d1 = 0;
        if (tid < nseg) {
            rel = tid / a.F1;
            d1 = tid % a.F1;
            const uint64_t *st = a.start + (size_t)rel * (nparts + 1);
            b0 = st[(size_t)d1 * a.F2];
            b1e = st[(size_t)(d1 + 1) * a.F2];
            ntile = ceil_div_u64(b1e - b0, kTile);
        }
        uint32_t tot;
        const uint32_t ft = block_excl_scan_u32(ntile, tmp, &tot);
        if (tid < nseg) {
            Seg s;
            s.in = a.tmp1 + (rel ? a.nR : 0) + b0;
            s.out = fin + (rel ? a.nR : 0);
            s.count = b1e - b0;
            s.out_len = nrel[rel];
            s.first_tile = ft;
            s.pad = 0;
            segs2[tid] = s;
        }
        if (tid == 0) {
            Seg sentinel = {};
            sentinel.first_tile = tot;
            segs2[nseg] = sentinel;
            a.counters[kCtrNTiles2] = tot;
            a.counters[kCtrNSegs2] = nseg;
        }
        for (int idx = tid; idx < nseg * a.F2; idx += blockDim.x) {
            const int s = idx / a.F2, d2 = idx % a.F2;
            const int r2 = s / a.F1, q1 = s % a.F1;
            obase2[(size_t)s * 256 + d2] =
                a.start[(size_t)r2 * (nparts + 1) + (size_t)q1 * a.F2 + d2];
        }
    }
    __syncthreads();

    // Join work items and large partitions.
    const uint64_t *stR = a.start, *stS = a.start + (nparts + 1);
    uint64_t item_run = 0, large_run = 0;
    __syncthreads();
    for (int c = 0; c < nparts; c += 1024) {
        const int f = c + tid;
        uint64_t nr = 0, ns = 0;
        if (f < nparts) {
            nr = stR[f + 1] - stR[f];
            ns = stS[f + 1] - stS[f];
        }
        const bool both = nr > 0 && ns > 0;
        const bool small = both && nr <= (uint64_t)kSmemCap;
        const bool large = both && !small;
        const uint32_t k = small ? ceil_div_u64(ns, kProbeChunk) : 0u;
        uint32_t ktot, ltot;
        const uint32_t kex = block_excl_scan_u32(k, tmp, &ktot);
        const uint32_t lex = block_excl_scan_u32(large ? 1u : 0u, tmp, &ltot);
        if (small) {
            for (uint32_t q = 0; q < k; q++) {
                const uint64_t idx = item_run + kex + q;
                if (idx < a.max_items) {
                    JoinItem it;
                    it.r_begin = stR[f];
                    it.s_begin = stS[f] + (uint64_t)q * kProbeChunk;
                    it.r_len = (uint32_t)nr;
                    const uint64_t rem = ns - (uint64_t)q * kProbeChunk;
                    it.s_len = (uint32_t)(rem < (uint64_t)kProbeChunk ? rem : (uint64_t)kProbeChunk);
                    it.pad[0] = it.pad[1] = 0;
                    a.items[idx] = it;
                } else {
                    atomicOr(&a.counters[kCtrErr], kErrCapacity);
                }
            }
        }
        if (large) {
            const uint64_t li = large_run + lex;
            if (li < a.max_large) {
                LargePart lp;
                lp.r_begin = stR[f];
                lp.s_begin = stS[f];
                lp.r_len = nr;
                lp.s_len = ns;
                uint32_t nb_log = 0;
                while ((1ull << nb_log) < nr) nb_log++;
                lp.nb_log = nb_log;
                lp.pad = 0;
                lp.table_off = 0;
                lp.r_flat = lp.s_flat = 0;
                a.large[li] = lp;
            } else {
                atomicOr(&a.counters[kCtrErr], kErrCapacity);
            }
        }
        item_run += ktot;
        large_run += ltot;
        __syncthreads();
    }
    // Offsets of the large partitions (sequential: there are few).
    __syncthreads();
    if (tid == 0) {
        const uint64_t nl = large_run < a.max_large ? large_run : a.max_large;
        uint64_t off = 0, rf = 0, sf = 0;
        for (uint64_t l = 0; l < nl; l++) {
            LargePart &lp = a.large[l];
            lp.table_off = off;
            lp.r_flat = rf;
            lp.s_flat = sf;
            off += (1ull << lp.nb_log) + lp.r_len;
            rf += lp.r_len;
            sf += lp.s_len;
        }
        if (off > a.large_table_words) atomicOr(&a.counters[kCtrErr], kErrCapacity);
        a.counters[kCtrNItems] = (uint32_t)(item_run < a.max_items ? item_run : a.max_items);
        a.counters[kCtrNLarge] = (uint32_t)nl;
        st_u64_pair(&a.counters[kCtrLargeR], off > a.large_table_words ? 0 : rf);
        st_u64_pair(&a.counters[kCtrLargeS], off > a.large_table_words ? 0 : sf);
        st_u64_pair(&a.counters[kCtrLargeWords], off > a.large_table_words ? 0 : off);
    }
}

// ------------------------------------------------------------------------------------------------
// 3. Stable scatter of one pass with decoupled look-back.
// ------------------------------------------------------------------------------------------------
struct ScatterArgs {
    const Seg *segs;
    const uint64_t *obase;  // [seg][256]
    uint32_t *counters;
    int ctr_tile, ctr_ntiles, ctr_nsegs;
    int F, shift;
    uint32_t *status;  // [tile][F]
    uint64_t status_words;
};

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS, 4) scatter_kernel(ScatterArgs a) {
    constexpr int T = THREADS * ITEMS;
    constexpr int NW = THREADS / 32;
    extern __shared__ __align__(16) unsigned char smem[];
    tuple_v *stage = reinterpret_cast<tuple_v *>(smem);
    long long *gbase = reinterpret_cast<long long *>(stage + T);  // [256]
    uint32_t *whist = reinterpret_cast<uint32_t *>(gbase + 256);  // [NW][F]
    uint32_t *tdstart = whist + NW * a.F;                         // [256]
    uint32_t *segft = tdstart + 256;                              // [nsegs + 1]
    __shared__ uint32_t scan_tmp[32];
    __shared__ uint32_t s_tile;

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int F = a.F;
    const uint64_t dmask = (uint64_t)F - 1;
    const uint32_t ntiles = a.counters[a.ctr_ntiles];
    const int nsegs = (int)a.counters[a.ctr_nsegs];
    unsigned int *err = &a.counters[kCtrErr];
    for (int s = tid; s <= nsegs; s += THREADS) segft[s] = a.segs[s].first_tile;
    const unsigned ltmask = lanemask_lt();

    for (;;) {
        if (tid == 0) s_tile = atomicAdd(&a.counters[a.ctr_tile], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= ntiles) break;
        // Segment of this tile: largest s with segft[s] <= tile.
        int lo = 0, hi = nsegs;  // invariant segft[lo] <= tile < segft[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (segft[mid] <= tile) lo = mid; else hi = mid;
        }
        const int seg = lo;
        const Seg sg = a.segs[seg];
        const uint32_t ltile = tile - segft[seg];
        const uint64_t begin = (uint64_t)ltile * T;
        const uint32_t cnt = (uint32_t)(sg.count - begin < (uint64_t)T ? sg.count - begin : (uint64_t)T);

        // Load: warp w owns tuples [w*32*ITEMS, (w+1)*32*ITEMS) of the tile, one coalesced 512-byte
        // row per item.
        tuple_v v[ITEMS];
        uint32_t d[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t idx = (uint32_t)(w * 32 * ITEMS + i * 32 + lane);
            if (idx < cnt) {
                v[i] = ld_stream(sg.in + begin + idx);
                d[i] = (uint32_t)((v[i].x >> a.shift) & dmask);
            } else {
                v[i] = make_ulonglong2(0, 0);
                d[i] = (uint32_t)F;
            }
        }
        uint32_t *wh = whist + w * F;
        for (int j = lane; j < F; j += 32) wh[j] = 0;
        __syncwarp();
        // Stable rank within the warp: items in order, lanes in order.
        uint32_t rk[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const unsigned peers = __match_any_sync(0xffffffffu, d[i]);
            const bool valid = d[i] < (uint32_t)F;
            uint32_t pre = 0;
            if (valid) pre = wh[d[i]];
            rk[i] = pre + __popc(peers & ltmask);
            __syncwarp();
            if (valid && (peers & ltmask) == 0) wh[d[i]] = pre + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // Tile histogram per digit and exclusive prefix over warps.
        uint32_t h = 0;
        if (tid < F) {
            for (int q = 0; q < NW; q++) {
                const uint32_t c = whist[q * F + tid];
                whist[q * F + tid] = h;
                h += c;
            }
        }
        const bool first = ltile == 0;
        uint32_t *my_status = a.status + (size_t)tile * F;
        if (tid < F && (uint64_t)tile * F + F <= a.status_words)
            st_relaxed_u32(&my_status[tid], (first ? kFlagPrefix : kFlagAgg) | h);
        const uint32_t ex = block_excl_scan_u32(tid < F ? h : 0u, scan_tmp, nullptr);
        if (tid < F) tdstart[tid] = ex;
        __syncthreads();
        // Stage the tile sorted by digit (stable).
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            if (d[i] < (uint32_t)F) {
                const uint32_t pos = tdstart[d[i]] + wh[d[i]] + rk[i];
                stage[pos] = v[i];
            }
        }
        // Look-back: exclusive prefix of this digit over the segment's earlier tiles.
        if (tid < F) {
            uint64_t excl = 0;
            if (!first) {
                int64_t t2 = (int64_t)tile - 1;
                int spins = 0;
                const int64_t tmin = (int64_t)segft[seg];
                while (t2 >= tmin) {
                    const uint32_t s = ld_relaxed_u32(&a.status[(size_t)t2 * F + tid]);
                    const uint32_t flag = s & ~kValueMask;
                    if (flag == 0) {
                        if (++spins > kSpinLimit) {
                            set_error(err, kErrSpinLimit);
                            break;
                        }
                        __nanosleep(32);
                        continue;
                    }
                    excl += s & kValueMask;
                    if (flag == kFlagPrefix) break;
                    t2--;
                }
                if ((uint64_t)tile * F + F <= a.status_words)
                    st_relaxed_u32(&my_status[tid], kFlagPrefix | (uint32_t)((excl + h) & kValueMask));
            }
            gbase[tid] = (long long)a.obase[(size_t)seg * 256 + tid] + (long long)excl - (long long)ex;
        }
        __syncthreads();
        // Write each digit run: consecutive threads write consecutive 16-byte tuples.
        for (uint32_t j = tid; j < cnt; j += THREADS) {
            const tuple_v t = stage[j];
            const uint32_t dd = (uint32_t)((t.x >> a.shift) & dmask);
            const long long dst = gbase[dd] + (long long)j;
            if (dst >= 0 && (uint64_t)dst < sg.out_len)
                st_stream(sg.out + dst, t);
            else
                set_error(err, kErrBounds);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------------
// 4. Partition join in shared memory.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// 16-bit exchange on a shared-memory halfword through a 32-bit CAS on its word (lock-free: every
// failed CAS means another thread's CAS succeeded).
__device__ __forceinline__ uint32_t atomic_exch_u16(uint16_t *addr, uint32_t val) {
    uint32_t *word = reinterpret_cast<uint32_t *>(reinterpret_cast<uintptr_t>(addr) & ~(uintptr_t)3);
    const uint32_t shift = (uint32_t)(reinterpret_cast<uintptr_t>(addr) & 2) * 8;
    uint32_t old = *reinterpret_cast<volatile uint32_t *>(word), assumed;
    do {
        assumed = old;
        const uint32_t nw = (assumed & ~(0xffffu << shift)) | (val << shift);
        old = atomicCAS(word, assumed, nw);
    } while (old != assumed);
    return (assumed >> shift) & 0xffffu;
}

struct JoinArgs {
    const JoinItem *items;
    const LargePart *large;
    uint32_t *counters;
    const tuple_v *finR, *finS;
    uint32_t *large_table;
    int bits;
    int lp;
    JoinAccum *acc;
};

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
    for (int it = 0; it < (1 << 24); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

constexpr int kHeadMax = 16384;  // next_pow_2(kSmemCap)
constexpr size_t kJoinSmem = (size_t)kSmemCap * 16 + kHeadMax * 2 + (size_t)kSmemCap * 2;

__global__ void __launch_bounds__(kJoinThreads, 1) join_small_kernel(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    tuple_v *rt = reinterpret_cast<tuple_v *>(smem);                      // [kSmemCap]
    uint16_t *head = reinterpret_cast<uint16_t *>(rt + kSmemCap);         // [kHeadMax]
    uint16_t *nxt = head + kHeadMax;                                       // [kSmemCap]
    __shared__ __align__(8) unsigned long long bar_storage;
    __shared__ unsigned long long red[64];
    __shared__ uint32_t s_item;
    const int tid = threadIdx.x;
    const uint32_t bar = smem_u32(&bar_storage);
    unsigned int *err = &a.counters[kCtrErr];
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t nitems = a.counters[kCtrNItems];
    const int B = a.bits;
    const bool lp = a.lp != 0;
    unsigned long long cnt = 0, sum = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(&a.counters[kCtrItem], 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= nitems) break;
        const JoinItem item = a.items[it];
        const uint32_t nr = item.r_len;
        const uint32_t nb = next_pow2_u32(nr);
        const uint64_t hmask = nb - 1;
        if (tid == 0) {
            // Order earlier generic-proxy accesses to rt before the async-proxy writes.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const uint32_t bytes = nr * 16u;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                         : "memory");
            const char *src = reinterpret_cast<const char *>(a.finR + item.r_begin);
            const uint32_t dst = smem_u32(rt);
            for (uint32_t off = 0; off < bytes; off += 32768u) {
                const uint32_t sz = bytes - off < 32768u ? bytes - off : 32768u;
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        dst + off),
                    "l"(src + off), "r"(sz), "r"(bar)
                    : "memory");
            }
        }
        uint32_t *head32 = reinterpret_cast<uint32_t *>(head);
        for (uint32_t q = tid; q < (nb + 1) / 2; q += kJoinThreads) head32[q] = 0;
        if (!mbar_wait(bar, phase)) {
            set_error(err, kErrSpinLimit);
            ok = false;
        }
        phase ^= 1u;
        __syncthreads();
        if (!ok) break;
        // Build: chain every R tuple (lp_join skips key 0, which reads as an empty slot there).
        for (uint32_t i = tid; i < nr; i += kJoinThreads) {
            const uint64_t k = rt[i].x;
            if (lp && k == 0) continue;
            const uint32_t h = (uint32_t)((k >> B) & hmask);
            nxt[i] = (uint16_t)atomic_exch_u16(&head[h], i + 1);
        }
        __syncthreads();
        // Probe.
        const tuple_v *S = a.finS + item.s_begin;
        const uint32_t ns = item.s_len;
        for (uint32_t j0 = tid; j0 < ns; j0 += 4 * kJoinThreads) {
            tuple_v s[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t j = j0 + u * kJoinThreads;
                s[u] = j < ns ? ld_stream(S + j) : make_ulonglong2(0, 0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t j = j0 + u * kJoinThreads;
                if (j >= ns) continue;
                const uint64_t k = s[u].x;
                uint32_t e = head[(k >> B) & hmask];
                uint32_t best = 0;
                uint32_t steps = 0;
                while (e) {
                    const tuple_v r = rt[e - 1];
                    if (r.x == k) {
                        if (lp) {
                            if (best == 0 || e < best) best = e;
                        } else {
                            cnt++;
                            sum += r.y + s[u].y;
                        }
                    }
                    e = nxt[e - 1];
                    if (++steps > nr) {
                        set_error(err, kErrProbeLimit);
                        break;
                    }
                }
                if (lp && best) {
                    cnt++;
                    sum += rt[best - 1].y + s[u].y;
                }
            }
        }
        __syncthreads();
    }
    block_sum2_to(cnt, sum, red, &a.acc->matched, &a.acc->checksum);
}

// Large partitions: chained tables in global memory, one flattened index space for all of them.
__device__ __forceinline__ int find_large(const LargePart *L, int nl, uint64_t g, bool by_r) {
    int lo = 0, hi = nl;  // largest l with flat[l] <= g
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        const uint64_t f = by_r ? L[mid].r_flat : L[mid].s_flat;
        if (f <= g) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void join_large_clear(JoinArgs a) {
    const uint64_t words = ld_u64_pair(&a.counters[kCtrLargeWords]);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < words;
         i += (uint64_t)gridDim.x * blockDim.x)
        a.large_table[i] = 0;
}

__global__ void join_large_build(JoinArgs a) {
    const int nl = (int)a.counters[kCtrNLarge];
    const uint64_t total = ld_u64_pair(&a.counters[kCtrLargeR]);
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const int l = find_large(a.large, nl, g, true);
        const LargePart &L = a.large[l];
        const uint64_t i = g - L.r_flat;
        const uint64_t k = a.finR[L.r_begin + i].x;
        if (a.lp && k == 0) continue;
        uint32_t *head = a.large_table + L.table_off;
        uint32_t *nxt = head + (1ull << L.nb_log);
        const uint64_t h = (k >> a.bits) & ((1ull << L.nb_log) - 1);
        nxt[i] = atomicExch(&head[h], (uint32_t)(i + 1));
    }
}

__global__ void join_large_probe(JoinArgs a) {
    __shared__ unsigned long long red[64];
    const int nl = (int)a.counters[kCtrNLarge];
    const uint64_t total = ld_u64_pair(&a.counters[kCtrLargeS]);
    unsigned long long cnt = 0, sum = 0;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const int l = find_large(a.large, nl, g, false);
        const LargePart &L = a.large[l];
        const tuple_v s = ld_stream(a.finS + L.s_begin + (g - L.s_flat));
        const uint32_t *head = a.large_table + L.table_off;
        const uint32_t *nxt = head + (1ull << L.nb_log);
        const tuple_v *rr = a.finR + L.r_begin;
        uint32_t e = head[(s.x >> a.bits) & ((1ull << L.nb_log) - 1)];
        uint32_t best = 0;
        uint64_t steps = 0;
        while (e) {
            const tuple_v r = rr[e - 1];
            if (r.x == s.x) {
                if (a.lp) {
                    if (best == 0 || e < best) best = e;
                } else {
                    cnt++;
                    sum += r.y + s.y;
                }
            }
            e = nxt[e - 1];
            if (++steps > L.r_len) {
                set_error(&a.counters[kCtrErr], kErrProbeLimit);
                break;
            }
        }
        if (a.lp && best) {
            cnt++;
            sum += rr[best - 1].y + s.y;
        }
    }
    block_sum2_to(cnt, sum, red, &a.acc->matched, &a.acc->checksum);
    if (blockIdx.x == 0 && threadIdx.x == 0 && nl) atomicAdd(&a.acc->large_parts, (unsigned long long)nl);
}

__global__ void copy_error(const uint32_t *counters, JoinAccum *acc) {
    if (threadIdx.x == 0 && counters[kCtrErr]) atomicOr(&acc->error, counters[kCtrErr]);
}

// ------------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------------
int radix_geom(int bits, int passes, RadixGeom *g) {
    if (bits < 1 || bits > 15) return HJ_E_INVAL;
    if (passes != 1 && passes != 2) return HJ_E_INVAL;
    // Partition results do not depend on how the bits are split across passes; a single pass is
    // run as one physical pass only while its fanout fits the shared-memory staging (<= 256).
    int P = passes;
    if (P == 1 && bits > 8) P = 2;
    if (P == 2 && bits < 2) P = 1;
    g->bits = bits;
    g->passes = P;
    g->b1 = P == 2 ? bits / 2 : bits;
    g->b2 = bits - g->b1;
    if (g->b1 > 8 || g->b2 > 8) return HJ_E_INVAL;
    g->F1 = 1 << g->b1;
    g->F2 = 1 << g->b2;
    return HJ_OK;
}

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct PhjSizes {
    size_t hist, start, segs, obase, counters, status, items, large, large_table, tmp1, tmp2;
    size_t max_items, max_large, status_words, large_table_words;
};

static PhjSizes phj_sizes(const RadixGeom &g, size_t nR, size_t nS) {
    PhjSizes z;
    const size_t np = (size_t)g.nparts();
    z.hist = align_up(2 * np * 4, 256);
    z.start = align_up(2 * (np + 1) * 8, 256);
    z.segs = align_up(2 * (kMaxPass2Segs + 1) * sizeof(Seg), 256);
    z.obase = align_up((size_t)2 * kMaxPass2Segs * 256 * 8, 256);
    z.counters = 256;
    const size_t max_tiles = (nR + nS) / kTile + 2 * (size_t)kMaxPass2Segs + 4;
    const size_t maxF = (size_t)(g.F1 > g.F2 ? g.F1 : g.F2);
    z.status_words = max_tiles * maxF;
    z.status = align_up(z.status_words * 4, 256);
    z.max_items = np + nS / kProbeChunk + 2;
    z.items = align_up(z.max_items * sizeof(JoinItem), 256);
    z.max_large = np < nR / kSmemCap + 1 ? np : nR / kSmemCap + 1;
    z.large = align_up(z.max_large * sizeof(LargePart), 256);
    z.tmp1 = align_up((nR + nS) * 16, 256);
    z.tmp2 = g.passes == 2 ? z.tmp1 : 0;
    // Large-partition chains: head <= 2*|R_p| words, next = |R_p| words. With two passes they reuse
    // the pass-1 buffer, which is dead once pass 2 has run.
    z.large_table_words = 3 * nR + 2;
    z.large_table = g.passes == 2 ? 0 : align_up(z.large_table_words * 4, 256);
    return z;
}

size_t phj_scratch_bytes(const RadixGeom &g, size_t nR, size_t nS) {
    PhjSizes z = phj_sizes(g, nR, nS);
    return z.hist + z.start + z.segs + z.obase + z.counters + z.status + z.items + z.large +
           z.large_table + z.tmp1 + z.tmp2;
}

void phj_carve(const RadixGeom &g, size_t nR, size_t nS, char *base, PhjScratch *s) {
    PhjSizes z = phj_sizes(g, nR, nS);
    char *p = base;
    s->hist = reinterpret_cast<uint32_t *>(p); p += z.hist;
    s->start = reinterpret_cast<uint64_t *>(p); p += z.start;
    s->segs = p; p += z.segs;
    s->obase = reinterpret_cast<uint64_t *>(p); p += z.obase;
    s->counters = reinterpret_cast<uint32_t *>(p); p += z.counters;
    s->status = reinterpret_cast<uint32_t *>(p); p += z.status;
    s->status_words = z.status_words;
    s->items = p; p += z.items;
    s->max_items = z.max_items;
    s->large = p; p += z.large;
    s->max_large = z.max_large;
    s->tmp1 = reinterpret_cast<ulonglong2 *>(p); p += z.tmp1;
    if (g.passes == 2) {
        s->tmp2 = reinterpret_cast<ulonglong2 *>(p); p += z.tmp2;
        s->large_table = reinterpret_cast<uint32_t *>(s->tmp1);
        s->large_table_words = z.tmp1 / 4;
    } else {
        s->tmp2 = s->tmp1;
        s->large_table = reinterpret_cast<uint32_t *>(p); p += z.large_table;
        s->large_table_words = z.large_table_words;
    }
}

#define HJ_CU(call)                                  \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) {                     \
            fprintf(stderr, "hjscm: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return HJ_E_DEVICE;                      \
        }                                            \
    } while (0)

static bool g_attr_done[64] = {};

int phj_enqueue(const RadixGeom &g, bool lp, const ulonglong2 *R, size_t nR, const ulonglong2 *S,
                size_t nS, const PhjScratch &s, JoinAccum *acc, cudaStream_t st, cudaEvent_t ev_mid,
                int num_sms) {
    if (nR >= (1ull << 30) || nS >= (1ull << 30)) return HJ_E_INVAL;
    const int np = g.nparts();
    const int F1 = g.F1, F2 = g.F2;
    const int maxF = F1 > F2 ? F1 : F2;
    constexpr int T = kTile;
    const size_t scatter_smem = (size_t)T * 16 + 256 * 8 + (kScatterThreads / 32) * 256 * 4 + 256 * 4 +
                                (kMaxPass2Segs + 1) * 4;
    const size_t hist_smem = (size_t)np * 4;
    int cur_dev = 0;
    HJ_CU(cudaGetDevice(&cur_dev));
    if (cur_dev < 0 || cur_dev >= 64) return HJ_E_INVAL;
    if (!g_attr_done[cur_dev]) {
        HJ_CU(cudaFuncSetAttribute(hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024));
        HJ_CU(cudaFuncSetAttribute(scatter_kernel<kScatterThreads, kScatterItems>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scatter_smem));
        HJ_CU(cudaFuncSetAttribute(join_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kJoinSmem));
        g_attr_done[cur_dev] = true;
    }
    (void)maxF;
    HJ_CU(cudaMemsetAsync(s.hist, 0, (size_t)2 * np * 4, st));
    HJ_CU(cudaMemsetAsync(s.counters, 0, kNumCounters * 4, st));

    // 1. histogram
    {
        const int hist_blocks = num_sms * (hist_smem > 64 * 1024 ? 1 : 2);
        int gR = (int)((double)hist_blocks * (double)nR / (double)(nR + nS + 1));
        if (nR && gR < 1) gR = 1;
        if (nS && gR > hist_blocks - 1) gR = hist_blocks - 1;
        hist_kernel<<<hist_blocks, 1024, hist_smem, st>>>(R, nR, S, nS, g.bits, s.hist, gR);
        HJ_CU(cudaGetLastError());
    }
    // 2. plan
    PlanArgs pa;
    pa.bits = g.bits;
    pa.passes = g.passes;
    pa.b1 = g.b1;
    pa.F1 = F1;
    pa.F2 = F2;
    pa.R = R;
    pa.S = S;
    pa.nR = nR;
    pa.nS = nS;
    pa.hist = s.hist;
    pa.start = s.start;
    pa.segs = reinterpret_cast<Seg *>(s.segs);
    pa.obase = s.obase;
    pa.counters = s.counters;
    pa.tmp1 = s.tmp1;
    pa.tmp2 = s.tmp2;
    pa.items = reinterpret_cast<JoinItem *>(s.items);
    pa.max_items = s.max_items;
    pa.large = reinterpret_cast<LargePart *>(s.large);
    pa.max_large = s.max_large;
    pa.large_table_words = s.large_table_words;
    plan_kernel<<<1, 1024, 0, st>>>(pa);
    HJ_CU(cudaGetLastError());

    // 3. scatter passes
    const int scatter_grid = num_sms * 4;
    for (int pass = 0; pass < g.passes; pass++) {
        const int F = pass == 0 ? F1 : F2;
        const size_t words = s.status_words;
        HJ_CU(cudaMemsetAsync(s.status, 0, words * 4, st));
        ScatterArgs sa;
        sa.segs = reinterpret_cast<const Seg *>(s.segs) + (size_t)pass * (kMaxPass2Segs + 1);
        sa.obase = s.obase + (size_t)pass * kMaxPass2Segs * 256;
        sa.counters = s.counters;
        sa.ctr_tile = pass == 0 ? kCtrTile1 : kCtrTile2;
        sa.ctr_ntiles = pass == 0 ? kCtrNTiles1 : kCtrNTiles2;
        sa.ctr_nsegs = pass == 0 ? kCtrNSegs1 : kCtrNSegs2;
        sa.F = F;
        sa.shift = pass == 0 ? 0 : g.b1;
        sa.status = s.status;
        sa.status_words = words;
        scatter_kernel<kScatterThreads, kScatterItems><<<scatter_grid, kScatterThreads, scatter_smem, st>>>(sa);
        HJ_CU(cudaGetLastError());
    }
    if (ev_mid) HJ_CU(cudaEventRecord(ev_mid, st));

    // 4. joins
    JoinArgs ja;
    ja.items = reinterpret_cast<const JoinItem *>(s.items);
    ja.large = reinterpret_cast<const LargePart *>(s.large);
    ja.counters = s.counters;
    ja.finR = s.tmp2;
    ja.finS = s.tmp2 + nR;
    ja.large_table = s.large_table;
    ja.bits = g.bits;
    ja.lp = lp ? 1 : 0;
    ja.acc = acc;
    join_small_kernel<<<num_sms, kJoinThreads, kJoinSmem, st>>>(ja);
    HJ_CU(cudaGetLastError());
    join_large_clear<<<num_sms * 2, 256, 0, st>>>(ja);
    join_large_build<<<num_sms * 2, 256, 0, st>>>(ja);
    join_large_probe<<<num_sms * 2, 256, 0, st>>>(ja);
    copy_error<<<1, 32, 0, st>>>(s.counters, acc);
    HJ_CU(cudaGetLastError());
    return HJ_OK;
}

}  // namespace hj
