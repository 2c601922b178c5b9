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
// B200 pipeline (one stream, no host round trip). Each relation is cut into equal chunks (about three
// per SM) and each chunk into ~32 sub-chunks; a chunk plays the role of one reference thread's
// contiguous input slice.
//   hist_chunk_kernel  one read of R and S: per chunk, the joint histogram of the low B key bits (the
//                      pass-1 digit and the pass-2 digit together) in shared memory; per sub-chunk (one
//                      warp each) the histogram of the pass-1 digit
//   colscan_kernel     per bin, exclusive prefix over the chunks of a relation (the reference's
//                      cross-thread output_offset sums, phj.c:188-200, for both passes at once)
//   plan_kernel        final partition starts, join work items, large partitions
//   units_kernel       per (chunk, pass-1 partition): its size and its start in the pass-1 output; per
//                      sub-chunk its start within that
//   scatter_kernel     per pass: persistent CTAs take work items (pass 1: sub-chunks; pass 2: (chunk,
//                      pass-1 partition) units) whose per-digit output offsets are known in advance;
//                      each 2048-tuple tile arrives by a TMA bulk copy (the next one is in flight while
//                      the current one is processed), is ranked per digit (one shared-memory atomic per
//                      tuple; stably with bit ballots for the lp joins, whose result depends on input
//                      order), staged in shared memory sorted by digit and written back as coalesced
//                      16-byte streaming stores per digit run (the shared-memory analogue of the
//                      reference's SWWCB + non-temporal flush). No inter-CTA waiting.
//   join_compact       when keys (after the radix shift) and row ids fit 32 bits: persistent CTAs take
//                      (partition, S chunk) items; 12-byte table entries with u16 bucket heads and chains
//                      built by shared-memory atomics; S streamed with evict-first vector loads
//   join_small         the general case: R_p arrives in shared memory by one TMA bulk copy, 16-byte
//                      entries, u16 head/next chains
//   join_large_*       partitions whose R side exceeds shared memory: chains in global memory
// The join kernels have a materialising variant (MAT) for the ptr_* joins: one (r.row_id, s.row_id)
// pair per match instead of the sums.
//
// Segment mode (joins that count every match, two passes, <= 14 bits, from 2^27 tuples): no histogram
// pass. seg_pass1_kernel writes pass 1 into per-(CTA, relation, digit) chains of tile-sized segments
// and counts each CTA's joint histogram itself; colscan/plan/units then treat the pass-1 CTAs as the
// chunks, and pass 2 (scatter_kernel) walks the chains as its units.
#include <cstdio>

#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {

// ------------------------------------------------------------------------------------------------
// Device-side plan structures
// ------------------------------------------------------------------------------------------------
struct JoinItem {
    uint64_t r_begin;  // index into the final R buffer
    uint64_t s_begin;  // index into the final S buffer
    uint32_t r_len;
    uint32_t s_len;
    uint32_t part0;    // 1: the partition of the keys whose radix bits are 0 (key 0's partition)
    uint32_t pad;
};

struct LargePart {
    uint64_t r_begin, s_begin;
    uint64_t r_len, s_len;
    uint64_t table_off;  // u32 words into the large table: head[nb] then next[r_len]
    uint64_t r_flat, s_flat;
    uint32_t nb_log;
    uint32_t part0;  // as JoinItem::part0
};

// counters[] slots
enum : int {
    kCtrItem1 = 0,       // scatter pass-1 work-item counter
    kCtrItem2 = 1,       // scatter pass-2 work-item counter
    kCtrNItemsA = 2,     // join items whose build side fits the compact shared-memory table (listed first)
    kCtrItemA = 3,       // compact join work-item counter
    kCtrSegAlloc = 4,    // segment mode: segment ids handed out
    kCtrLargeAgg = 5,    // 1: large partitions use key-aggregated tables (see join_large_build)
    kCtrNItems = 6,
    kCtrNLarge = 7,
    kCtrItem = 8,        // join work-item counter
    kCtrLargeR = 9,      // total R tuples in large partitions (u32 pairs: lo, hi)
    kCtrLargeS = 11,     // total S tuples in large partitions (lo, hi)
    kCtrLargeWords = 13, // table words used (lo, hi)
    kCtrErr = 15,
    kCtrMaxKey = 16,     // u64: OR of all R keys (words 16-17)
    kCtrMaxRid = 18,     // u64: OR of all R row ids (words 18-19)
    kCtrOrRidS = 20,     // u64: OR of all S row ids (words 20-21)
    kCtrItem1S = 22,     // first-match joins: pass-1 work-item counter of the probe relation's items
    kCtrItem2S = 23,     // first-match joins: pass-2 work-item counter of the probe relation's items
    kNumCounters = 24
};

// Compact final partitions. When every build key shifted right by the radix bits is below 2^31 and
// every row id (build and probe) below 2^32, the last partition pass stores each tuple as one 8-byte
// word, (key >> bits) << 32 | row id, and the joins read 8 bytes per tuple instead of 16. Inside a
// final partition the low `bits` key bits are equal, so comparing key >> bits compares keys. A probe
// key whose high part is 2^31 or more is stored as 0xffffffff: no build key has that high part. Joins
// where a build key 0 never matches (lp_join's empty-slot rule): a last pass that reads tuples stores
// that key's words with high part 0x80000000, which no build key and no probe word has (ci_word_z0);
// from segment-mode pass-1 words it keeps high part 0, and since key 0 lies in the partition of the
// keys whose radix bits are 0, where a high part of 0 means key 0, the joins skip such build words
// there (JoinItem::part0). The widths are ORed together by the pass that reads the relations first (hist_chunk_kernel or
// seg_pass1_kernel), so the choice is made on the device, before the last pass.
__device__ __forceinline__ bool ci_applies(const uint32_t *counters, int bits) {
    const unsigned long long *mx = reinterpret_cast<const unsigned long long *>(counters + kCtrMaxKey);
    return (mx[0] >> bits) < (1ull << 31) && mx[1] < (1ull << 32) && mx[2] < (1ull << 32);
}

// Segment mode can go further: pass 1 stores (key >> b1) << 32 | row id (w8_word) in segments of 4096
// words (the same 32 KB as 2048 tuples) when every build key >> b1 is below 2^31 and every row id below
// 2^32; pass 2 then reads 8-byte words in tiles of 4096 and writes compact final partitions. A probe
// key whose key >> b1 does not fit keeps its low 31 bits and gets bit 31 set: its pass-2 digit stays
// right, and after pass 2's shift its high part is still above every build key's.
__device__ __forceinline__ bool w8_fits(const uint32_t *counters, int b1) {
    const unsigned long long *mx = reinterpret_cast<const unsigned long long *>(counters + kCtrMaxKey);
    return (mx[0] >> b1) < (1ull << 31) && mx[1] < (1ull << 32) && mx[2] < (1ull << 32);
}

__device__ __forceinline__ unsigned long long w8_word(unsigned long long key, unsigned long long rid, int b1) {
    const unsigned long long hi = key >> b1;
    const unsigned long long h32 = hi < (1ull << 31) ? hi : (0x80000000ull | (hi & 0x7fffffffull));
    return (h32 << 32) | (rid & 0xffffffffull);
}

// Build relations whose key 0 never matches (z0), in the exact-offset pipeline's word pass 1: key 0's
// word takes the high part 0x80000000, which no other build word has; the last pass keeps it
// (store_elem) and stores every probe word whose high part has bit 31 set as 0xffffffff, so nothing
// matches it. (Segment mode's pass 1 stores key 0 as any key; the joins skip it in its partition.)
__device__ __forceinline__ unsigned long long w8_word_z0(unsigned long long key, unsigned long long rid, int b1,
                                                         bool z0) {
    return z0 && key == 0 ? (0x80000000ull << 32) | (rid & 0xffffffffull) : w8_word(key, rid, b1);
}

__device__ __forceinline__ unsigned long long ci_word(unsigned long long key, unsigned long long rid, int bits) {
    const unsigned long long hi = key >> bits;
    return ((hi < 0x80000000ull ? hi : 0xffffffffull) << 32) | (rid & 0xffffffffull);
}

__device__ __forceinline__ unsigned long long ci_word_z0(unsigned long long key, unsigned long long rid, int bits,
                                                         bool z0) {
    return z0 && key == 0 ? (0x80000000ull << 32) | (rid & 0xffffffffull) : ci_word(key, rid, bits);
}

// Build partitions up to this size whose keys (above the radix bits) and row ids fit 32 bits are
// joined with a 4-byte-per-field shared-memory table, two CTAs per SM.
constexpr int kCompactCap = 8192;
constexpr int kCompactThreads = 512;

// Chunking of the two relations (identical for the histogram and both scatter passes).
struct ChunkGeom {
    uint64_t chunk;  // tuples per chunk (a multiple of the tile)
    uint32_t cR, cS; // chunks of R, chunks of S (R's come first)
    uint64_t sub;    // tuples per sub-chunk (a multiple of the tile): the pass-1 work item
    uint32_t spc;    // sub-chunks per chunk
    uint32_t pad;
};

__device__ __forceinline__ uint64_t ld_u64_pair(const uint32_t *p) {
    return (uint64_t)p[0] | ((uint64_t)p[1] << 32);
}
__device__ __forceinline__ void st_u64_pair(uint32_t *p, uint64_t v) {
    p[0] = (uint32_t)v;
    p[1] = (uint32_t)(v >> 32);
}

__host__ __device__ __forceinline__ uint32_t ceil_div_u64(uint64_t a, uint64_t b) {
    return (uint32_t)((a + b - 1) / b);
}

__device__ __forceinline__ uint32_t next_pow2_u32(uint32_t x) {
    return x <= 1 ? 1u : 1u << (32 - __clz(x - 1));
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Bounded wait for the completion of phase `parity` of an mbarrier.
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for an mbarrier phase: gives up after kWaitNs of wall time (try_wait may suspend the
// thread for a hardware-defined time per call, so an iteration count alone is no time bound).
constexpr uint64_t kWaitNs = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < (1u << 30); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 63u) == 63u && globaltimer_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

// TMA bulk copy global -> shared of `bytes` (a multiple of 16, <= 1 MiB per phase), completing on
// `bar`. Issued by one thread.
__device__ __forceinline__ void tma_load_1d(void *dst_smem, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    const char *s = reinterpret_cast<const char *>(src);
    const uint32_t d = smem_addr(dst_smem);
    for (uint32_t off = 0; off < bytes; off += 32768u) {
        const uint32_t sz = bytes - off < 32768u ? bytes - off : 32768u;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d + off),
            "l"(s + off), "r"(sz), "r"(bar)
            : "memory");
    }
}

// Count the tuples [lo, hi) of `in`, read by one warp (four 512-byte loads in flight), into the joint
// histogram and into the warp's histogram of the pass-1 digit, ORing together all row ids and (BUILD)
// all keys: their widths decide whether the compact join table and the compact final partitions apply
// (a value fits k bits iff the OR of all values does).
template <bool BUILD>
__device__ __forceinline__ void hist_range_warp(const tuple_v *__restrict__ in, uint64_t lo, uint64_t hi,
                                                uint32_t *sh_hist, uint32_t *wsub, uint64_t mask, uint32_t m1,
                                                unsigned long long &kor, unsigned long long &ror) {
    uint64_t i = lo + (threadIdx.x & 31u);
    for (; i + 96 < hi; i += 128) {
        const tuple_v t0 = ld_stream(in + i), t1 = ld_stream(in + i + 32);
        const tuple_v t2 = ld_stream(in + i + 64), t3 = ld_stream(in + i + 96);
        atomicAdd(&sh_hist[t0.x & mask], 1u);
        atomicAdd(&sh_hist[t1.x & mask], 1u);
        atomicAdd(&sh_hist[t2.x & mask], 1u);
        atomicAdd(&sh_hist[t3.x & mask], 1u);
        atomicAdd(&wsub[(uint32_t)t0.x & m1], 1u);
        atomicAdd(&wsub[(uint32_t)t1.x & m1], 1u);
        atomicAdd(&wsub[(uint32_t)t2.x & m1], 1u);
        atomicAdd(&wsub[(uint32_t)t3.x & m1], 1u);
        if (BUILD) kor |= t0.x | t1.x | t2.x | t3.x;
        ror |= t0.y | t1.y | t2.y | t3.y;
    }
    for (; i < hi; i += 32) {
        const tuple_v t = ld_stream(in + i);
        atomicAdd(&sh_hist[t.x & mask], 1u);
        atomicAdd(&wsub[(uint32_t)t.x & m1], 1u);
        if (BUILD) kor |= t.x;
        ror |= t.y;
    }
}

// ------------------------------------------------------------------------------------------------
// 1. Per-chunk joint histogram of the low `bits` key bits, and per sub-chunk the histogram of the
//    pass-1 digit (the low log2(F1) bits). One CTA per chunk; each warp takes whole sub-chunks, so a
//    sub-chunk's digit histogram is complete after a warp barrier and no CTA barrier interrupts the
//    stream of loads. Every bin is written.
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(512) hist_chunk_kernel(const tuple_v *__restrict__ R, size_t nR,
                                                         const tuple_v *__restrict__ S, size_t nS, int bits,
                                                         int F1, ChunkGeom cg, uint32_t *__restrict__ chunk_hist,
                                                         uint32_t *__restrict__ subhist,
                                                         uint32_t *__restrict__ maxima) {
    extern __shared__ uint32_t sh_hist[];
    const int nbins = 1 << bits;
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31u, nw = blockDim.x >> 5;
    uint32_t *wsub = sh_hist + nbins + (size_t)w * F1;  // [warps][F1] per-warp pass-1 digit histogram
    const uint64_t mask = (uint64_t)nbins - 1;
    const uint32_t m1 = (uint32_t)F1 - 1u;
    const uint32_t c = blockIdx.x;
    const int rel = c < cg.cR ? 0 : 1;
    const uint64_t lc = rel ? c - cg.cR : c;
    const tuple_v *in = rel ? S : R;
    const uint64_t n = rel ? nS : nR;
    for (int v = threadIdx.x; v < nbins + (int)nw * F1; v += blockDim.x) sh_hist[v] = 0;
    __syncthreads();
    const uint64_t clo = lc * cg.chunk;
    const uint64_t chi = clo + cg.chunk < n ? clo + cg.chunk : n;
    unsigned long long kor = 0, ror = 0;
    for (uint32_t j = w; j < cg.spc; j += nw) {
        const uint64_t lo = clo + (uint64_t)j * cg.sub < chi ? clo + (uint64_t)j * cg.sub : chi;
        const uint64_t hi = lo + cg.sub < chi ? lo + cg.sub : chi;
        if (rel == 0)
            hist_range_warp<true>(in, lo, hi, sh_hist, wsub, mask, m1, kor, ror);
        else
            hist_range_warp<false>(in, lo, hi, sh_hist, wsub, mask, m1, kor, ror);
        __syncwarp();
        uint32_t *so = subhist + ((size_t)c * cg.spc + j) * F1;
        for (int v = lane; v < F1; v += 32) {
            so[v] = wsub[v];
            wsub[v] = 0;
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kor |= __shfl_xor_sync(0xffffffffu, kor, o);
        ror |= __shfl_xor_sync(0xffffffffu, ror, o);
    }
    if (lane == 0) {
        unsigned long long *mx = reinterpret_cast<unsigned long long *>(maxima);
        if (rel == 0) {
            if (kor) atomicOr(mx, kor);
            if (ror) atomicOr(mx + 1, ror);
        } else if (ror) {
            atomicOr(mx + 2, ror);
        }
    }
    __syncthreads();
    uint32_t *out = chunk_hist + (size_t)c * nbins;
    for (int v = threadIdx.x; v < nbins; v += blockDim.x) out[v] = sh_hist[v];
}

// ------------------------------------------------------------------------------------------------
// 2. Per bin, exclusive prefix over the chunks of its relation, and the relation totals. Four
//    consecutive lanes share one bin and split its chunks into four ranges: each lane sums its range,
//    the four sums are scanned with shuffles, then each lane writes the prefixes of its range.
// ------------------------------------------------------------------------------------------------
__global__ void colscan_kernel(const uint32_t *__restrict__ chunk_hist, uint32_t *__restrict__ prefix,
                               uint32_t *__restrict__ total, int nbins, ChunkGeom cg) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t col = g >> 2, seg = g & 3u;
    const bool active = col < 2u * (uint32_t)nbins;
    const int rel = active && col >= (uint32_t)nbins;
    const uint32_t v = active ? (rel ? col - nbins : col) : 0u;
    const uint32_t c0 = rel ? cg.cR : 0, c1 = rel ? cg.cR + cg.cS : cg.cR;
    const uint32_t per = (c1 - c0 + 3) / 4;
    const uint32_t r0 = c0 + seg * per < c1 ? c0 + seg * per : c1;
    const uint32_t r1 = r0 + per < c1 ? r0 + per : c1;
    uint32_t sum = 0;
    if (active) {
        uint32_t c = r0;
        for (; c + 8 <= r1; c += 8) {
            uint32_t x[8];
#pragma unroll
            for (int u = 0; u < 8; u++) x[u] = chunk_hist[(size_t)(c + u) * nbins + v];
#pragma unroll
            for (int u = 0; u < 8; u++) sum += x[u];
        }
        for (; c < r1; c++) sum += chunk_hist[(size_t)c * nbins + v];
    }
    // Exclusive scan of the four range sums (lanes 4k..4k+3 of the warp).
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 4; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o, 4);
        if (seg >= (uint32_t)o) incl += y;
    }
    const uint32_t colsum = __shfl_sync(0xffffffffu, incl, 3, 4);
    if (!active) return;
    uint32_t run = incl - sum;
    uint32_t c = r0;
    for (; c + 8 <= r1; c += 8) {
        uint32_t x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) x[u] = chunk_hist[(size_t)(c + u) * nbins + v];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            prefix[(size_t)(c + u) * nbins + v] = run;
            run += x[u];
        }
    }
    for (; c < r1; c++) {
        const uint32_t x = chunk_hist[(size_t)c * nbins + v];
        prefix[(size_t)c * nbins + v] = run;
        run += x;
    }
    if (seg == 3) total[(size_t)rel * nbins + v] = colsum;
}

// ------------------------------------------------------------------------------------------------
// 3. Plan: final partition starts (in (pass-1 digit, pass-2 digit) order), join work items, large
//    partitions. One CTA of 1024 threads.
// ------------------------------------------------------------------------------------------------
struct PlanArgs {
    int bits, passes, b1, F1, F2;
    uint64_t nR, nS;
    const uint32_t *total;  // [2][2^B]
    uint64_t *start;        // [2][2^B + 1]
    uint32_t *counters;
    JoinItem *items;
    uint64_t max_items;
    LargePart *large;
    uint64_t max_large;
    uint64_t large_table_words;
    int agg_ok;  // joins that need no per-match output may use key-aggregated large-partition tables
};

__device__ __forceinline__ uint32_t part_to_value(int f, int passes, int b1, int F2) {
    if (passes == 1) return (uint32_t)f;
    const uint32_t d1 = (uint32_t)f / (uint32_t)F2, d2 = (uint32_t)f % (uint32_t)F2;
    return d1 | (d2 << b1);
}

// u32 words of one large partition's table. Chains: head[nb] then next[r_len]. Key-aggregated:
// sum[r_len] (u64), head[nb], next[r_len], cnt[r_len], negpos[r_len], rounded to an even count so the
// next table's sums stay 8-byte aligned.
__device__ __forceinline__ uint64_t large_words_chain(const LargePart &L) { return (1ull << L.nb_log) + L.r_len; }
__device__ __forceinline__ uint64_t large_words_agg(const LargePart &L) {
    return ((1ull << L.nb_log) + 5 * L.r_len + 1) & ~1ull;
}

// Dynamic shared memory: the relation totals ([2][2^B] u32) when they fit (B <= 14), so that the
// per-partition loops below read shared memory instead of waiting on one global load after another.
constexpr int kPlanStageBits = 14;

__global__ void __launch_bounds__(1024, 1) plan_kernel(PlanArgs a) {
    extern __shared__ uint32_t sm_tot[];
    __shared__ uint32_t tmp[32];
    __shared__ uint64_t s_item_run, s_large_run;
    const int tid = threadIdx.x;
    const int nparts = 1 << a.bits;
    const uint32_t *tot_all = a.total;
    if (a.bits <= kPlanStageBits) {
#pragma unroll 8
        for (int i = tid; i < 2 * nparts; i += 1024) sm_tot[i] = a.total[i];
        __syncthreads();
        tot_all = sm_tot;
    }
    // Each thread owns a contiguous range of partitions.
    const int per = (nparts + 1023) / 1024;
    const int f0 = tid * per < nparts ? tid * per : nparts;
    const int f1 = f0 + per < nparts ? f0 + per : nparts;
    uint64_t base[2];  // start of this thread's first partition, per relation
    for (int rel = 0; rel < 2; rel++) {
        uint64_t *start = a.start + (size_t)rel * (nparts + 1);
        const uint32_t *tot = tot_all + (size_t)rel * nparts;
        uint32_t sum = 0;
        for (int f = f0; f < f1; f++) sum += tot[part_to_value(f, a.passes, a.b1, a.F2)];
        uint32_t all;
        uint64_t run = block_excl_scan_u32(sum, tmp, &all);
        base[rel] = run;
        for (int f = f0; f < f1; f++) {
            start[f] = run;
            run += tot[part_to_value(f, a.passes, a.b1, a.F2)];
        }
        if (tid == 0) start[nparts] = all;
    }

    // Join work items (partitions with both sides non-empty, src/algo/phj.c:459-491) and large
    // partitions. Partition sizes come from the totals, starts from the running sums above.
    const uint32_t *totR = tot_all, *totS = tot_all + nparts;
    const uint64_t small_cap = (uint64_t)kSmemCap;
    uint32_t asum = 0, bsum = 0, lsum = 0;  // items with |R_p| <= compact cap, other small items, large
    for (int f = f0; f < f1; f++) {
        const uint32_t v = part_to_value(f, a.passes, a.b1, a.F2);
        const uint64_t nr = totR[v], ns = totS[v];
        if (nr > 0 && ns > 0) {
            if (nr <= (uint64_t)kCompactCap) asum += ceil_div_u64(ns, kProbeChunk);
            else if (nr <= small_cap) bsum += ceil_div_u64(ns, kProbeChunk);
            else lsum++;
        }
    }
    uint32_t atot, btot, ltot;
    uint64_t a_idx = block_excl_scan_u32(asum, tmp, &atot);
    uint64_t b_idx = block_excl_scan_u32(bsum, tmp, &btot) + atot;
    uint64_t large_idx = block_excl_scan_u32(lsum, tmp, &ltot);
    const uint32_t ktot = atot + btot;
    uint64_t rR = base[0], rS = base[1];
    for (int f = f0; f < f1; f++) {
        const uint32_t v = part_to_value(f, a.passes, a.b1, a.F2);
        const uint64_t nr = totR[v], ns = totS[v];
        const uint64_t sR = rR, sS = rS;
        rR += nr;
        rS += ns;
        if (!(nr > 0 && ns > 0)) continue;
        if (nr <= small_cap) {
            uint64_t &item_idx = nr <= (uint64_t)kCompactCap ? a_idx : b_idx;
            const uint32_t k = ceil_div_u64(ns, kProbeChunk);
            for (uint32_t q = 0; q < k; q++, item_idx++) {
                if (item_idx < a.max_items) {
                    JoinItem it;
                    it.r_begin = sR;
                    it.s_begin = sS + (uint64_t)q * kProbeChunk;
                    it.r_len = (uint32_t)nr;
                    const uint64_t rem = ns - (uint64_t)q * kProbeChunk;
                    it.s_len = (uint32_t)(rem < (uint64_t)kProbeChunk ? rem : (uint64_t)kProbeChunk);
                    it.part0 = v == 0 ? 1u : 0u;
                    it.pad = 0;
                    a.items[item_idx] = it;
                } else {
                    atomicOr(&a.counters[kCtrErr], kErrCapacity);
                }
            }
        } else {
            if (large_idx < a.max_large) {
                LargePart lp;
                lp.r_begin = sR;
                lp.s_begin = sS;
                lp.r_len = nr;
                lp.s_len = ns;
                uint32_t nb_log = 0;
                while ((1ull << nb_log) < nr) nb_log++;
                lp.nb_log = nb_log;
                lp.part0 = v == 0 ? 1u : 0u;
                lp.table_off = 0;
                lp.r_flat = lp.s_flat = 0;
                a.large[large_idx] = lp;
            } else {
                atomicOr(&a.counters[kCtrErr], kErrCapacity);
            }
            large_idx++;
        }
    }
    if (tid == 0) a.counters[kCtrNItemsA] = atot < a.max_items ? atot : (uint32_t)a.max_items;
    if (tid == 0) {
        s_item_run = ktot;
        s_large_run = ltot;
    }
    __syncthreads();
    const uint64_t item_run = s_item_run, large_run = s_large_run;
    __syncthreads();
    if (tid == 0) {
        const uint64_t nl = large_run < a.max_large ? large_run : a.max_large;
        // Key-aggregated tables (large_words_agg) when the join allows them and they fit the table
        // area, else plain chains (large_words_chain).
        uint64_t need_agg = 0;
        for (uint64_t l = 0; l < nl; l++) need_agg += large_words_agg(a.large[l]);
        const bool agg = a.agg_ok && need_agg <= a.large_table_words;
        a.counters[kCtrLargeAgg] = agg ? 1u : 0u;
        uint64_t off = 0, rf = 0, sf = 0;
        for (uint64_t l = 0; l < nl; l++) {
            LargePart &lp = a.large[l];
            lp.table_off = off;
            lp.r_flat = rf;
            lp.s_flat = sf;
            off += agg ? large_words_agg(lp) : large_words_chain(lp);
            rf += lp.r_len;
            sf += lp.s_len;
        }
        const bool fits = off <= a.large_table_words;
        if (!fits) atomicOr(&a.counters[kCtrErr], kErrCapacity);
        a.counters[kCtrNItems] = (uint32_t)(item_run < a.max_items ? item_run : a.max_items);
        a.counters[kCtrNLarge] = (uint32_t)nl;
        st_u64_pair(&a.counters[kCtrLargeR], fits ? rf : 0);
        st_u64_pair(&a.counters[kCtrLargeS], fits ? sf : 0);
        st_u64_pair(&a.counters[kCtrLargeWords], fits ? off : 0);
    }
}

// ------------------------------------------------------------------------------------------------
// 4. Units: for every chunk c and pass-1 digit d1, the number of the chunk's tuples with that digit
//    and where they start in the pass-1 output: start[d1 * F2] + sum over d2 of prefix[c][(d1, d2)].
//    The sub-chunk histograms of the chunk become, in place, each sub-chunk's start within (c, d1).
// ------------------------------------------------------------------------------------------------
__global__ void units_kernel(const uint32_t *__restrict__ chunk_hist, const uint32_t *__restrict__ prefix,
                             const uint64_t *__restrict__ start, int bits, int b1, int F1, int F2,
                             ChunkGeom cg, uint64_t *__restrict__ unit_off, uint32_t *__restrict__ unit_cnt,
                             uint32_t *__restrict__ subhist, uint32_t *__restrict__ err) {
    // One CTA per chunk, one thread per pass-1 digit; for a fixed pass-2 digit the threads read
    // consecutive bins.
    const uint32_t c = blockIdx.x;
    const uint32_t d1 = threadIdx.x;
    if (d1 >= (uint32_t)F1) return;
    const int rel = c < cg.cR ? 0 : 1;
    const int nbins = 1 << bits;
    const uint32_t *h = chunk_hist + (size_t)c * nbins;
    const uint32_t *p = prefix + (size_t)c * nbins;
    uint64_t cnt = 0, pre = 0;
    int d2 = 0;
    for (; d2 + 8 <= F2; d2 += 8) {
        uint32_t x[8], y[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const uint32_t v = d1 | ((uint32_t)(d2 + u) << b1);
            x[u] = h[v];
            y[u] = p[v];
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
            cnt += x[u];
            pre += y[u];
        }
    }
    for (; d2 < F2; d2++) {
        const uint32_t v = d1 | ((uint32_t)d2 << b1);
        cnt += h[v];
        pre += p[v];
    }
    const uint32_t wid = c * (uint32_t)F1 + d1;
    unit_cnt[wid] = (uint32_t)cnt;
    unit_off[wid] = start[(size_t)rel * (nbins + 1) + (size_t)d1 * F2] + pre;
    uint32_t *sh = subhist + (size_t)c * cg.spc * F1 + d1;
    uint32_t run = 0;
    uint32_t j = 0;
    for (; j + 8 <= cg.spc; j += 8) {
        uint32_t x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) x[u] = sh[(size_t)(j + u) * F1];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            sh[(size_t)(j + u) * F1] = run;
            run += x[u];
        }
    }
    for (; j < cg.spc; j++) {
        const uint32_t x = sh[(size_t)j * F1];
        sh[(size_t)j * F1] = run;
        run += x;
    }
    if (cg.spc && run != (uint32_t)cnt) set_error(err, kErrCapacity);
}

// ------------------------------------------------------------------------------------------------
// 5. Stable scatter of one pass, from precomputed per-item digit offsets.
// ------------------------------------------------------------------------------------------------
struct ScatterArgs {
    int pass;        // 0: by the pass-1 digit, per chunk; 1: by the pass-2 digit, per (chunk, d1) unit
    int F, shift;    // digit of this pass: (key >> shift) & (F - 1)
    int logF;        // log2(F)
    int bits, b1, F1, F2;
    ChunkGeom cg;
    const tuple_v *inR, *inS;   // pass input (pass 0: the relations; pass 1: the pass-1 output)
    tuple_v *outR, *outS;       // pass output
    uint64_t nR, nS;
    const uint32_t *prefix;     // [chunk][2^B]
    const uint64_t *start;      // [2][2^B + 1]
    const uint64_t *unit_off;   // [chunk][F1]
    const uint32_t *unit_cnt;   // [chunk][F1]
    const uint32_t *subpre;     // [chunk][spc][F1] start of (sub-chunk, d1) within (chunk, d1)
    // Segment mode, pass 2: unit (chunk, d1) is a chain of kTile-tuple segments in inR (the pass-1
    // output of both relations): seg_head[unit], then seg_next[segment]; all but the last are full.
    const uint32_t *seg_head;   // nullptr: units are contiguous ranges (unit_off)
    const uint32_t *seg_next;
    uint32_t max_segs;
    int test_stall;             // test hook: CTA 0 withholds its first tile load (its wait must expire)
    uint32_t *counters;
    int ctr_item;
    // Work items of this launch: [item_base, item_end) of the pass's items (R's first, then S's), claimed
    // through counters[ctr_item]; item_end 0 = all of them.
    uint32_t item_base, item_end;
    // Last pass of a join that may read compact final partitions: when ci_applies holds, the output is
    // 8-byte words (ci_word) at outR8 / outS8 instead of tuples at outR / outS.
    int ci_out;
    int ci_z0;                  // build key 0 never matches: its compact words take ci_word_z0's high part
    unsigned long long *outR8, *outS8;
    // After a pass 1 that may have written 8-byte words: 1 = this launch reads words (runs when w8_fits
    // holds), 2 = this launch reads tuples (runs when it does not); 0 = no such pass 1.
    int w8;
    // Exact-offset pipeline: pass 1 stores 8-byte words (w8_word) at outR8 / outS8 when w8_fits holds,
    // and the word launch of pass 2 reads its units from inR8 / inS8 (word offsets, which may be odd:
    // such a tile's copy starts one word early and the tile skips it).
    int w8_out;
    const unsigned long long *inR8, *inS8;
};

// A tile claimed for processing: its source, length, output region and owning work item.
struct TileSlot {
    const tuple_v *in;
    tuple_v *out;
    uint64_t out_len;
    uint32_t item;   // work item (valid flag: item != ~0u)
    uint32_t cnt;    // tuples in this tile
    uint32_t first;  // first tile of its item: the item's digit offsets must be loaded
    uint32_t pad;    // elements before the tile's first in its copy (a word tile at an odd offset)
};

// Thread-0 state of the work-item iterator.
struct ItemIter {
    uint32_t item = ~0u;
    const tuple_v *in = nullptr;
    tuple_v *out = nullptr;
    uint64_t len = 0, out_len = 0, done = 0;
    uint32_t seg = 0;   // segment mode: segment of the next tile
};

// The next work item, claimed one item ahead (thread 0 only): its id comes from the counter while the
// current item is processed, and the loads of its description are issued one call later, so that
// neither the atomic nor the loads stall the CTA at the switch.
struct ItemAhead {
    uint32_t item;   // claimed id (stage >= 1)
    uint32_t stage;  // 0: nothing claimed, 1: claimed, 2: description loaded
    uint64_t len, off;
    uint32_t seg;
};

// Issue the loads that describe `ah.item` (pass 2 units; pass-1 sub-chunks need none).
__device__ __forceinline__ void item_fetch(const ScatterArgs &a, ItemAhead &ah, uint32_t nitems) {
    ah.stage = 2;
    if (a.pass == 0 || ah.item >= nitems) return;
    ah.len = a.unit_cnt[ah.item];
    if (a.seg_head)
        ah.seg = a.seg_head[ah.item];  // read even for an empty unit (then unused): no dependent load
    else
        ah.off = a.unit_off[ah.item];
}

__device__ __forceinline__ void item_decode(const ScatterArgs &a, uint32_t item, const ItemAhead &ah, ItemIter &it) {
    const ChunkGeom &cg = a.cg;
    it.item = item;
    it.done = 0;
    if (a.pass == 0) {
        // Pass 1 work item: sub-chunk j of chunk c.
        const uint32_t c = item / cg.spc, j = item % cg.spc;
        const int rel = c < cg.cR ? 0 : 1;
        const uint64_t lc = rel ? c - cg.cR : c;
        const uint64_t n = rel ? a.nS : a.nR;
        const uint64_t clo = lc * cg.chunk;
        const uint64_t chi = clo + cg.chunk < n ? clo + cg.chunk : n;
        const uint64_t lo = clo + (uint64_t)j * cg.sub;
        it.len = lo < chi ? (chi - lo < cg.sub ? chi - lo : cg.sub) : 0;
        it.in = (rel ? a.inS : a.inR) + lo;
        it.out = rel ? a.outS : a.outR;
        it.out_len = n;
    } else {
        const uint32_t c = item / a.F1;
        const int rel = c < cg.cR ? 0 : 1;
        it.len = ah.len;
        if (a.seg_head) {
            it.in = a.inR;
            it.seg = ah.seg;
        } else if (a.w8 == 1) {
            it.in = reinterpret_cast<const tuple_v *>((rel ? a.inS8 : a.inR8) + ah.off);
        } else {
            it.in = (rel ? a.inS : a.inR) + ah.off;
        }
        it.out = rel ? a.outS : a.outR;
        it.out_len = rel ? a.nS : a.nR;
    }
}

// Claim the next tile (thread 0 only): continue the current item or take new items until one has
// tuples. Returns a slot with item == ~0u when the work is exhausted. Segment mode: `pend` carries
// seg_next of the tile returned last, loaded then so that its latency passes while that tile is
// processed.
template <int T, bool WIN = false>
__device__ __forceinline__ TileSlot next_tile(const ScatterArgs &a, ItemIter &it, uint32_t nitems,
                                              uint32_t &pend, ItemAhead &ah) {
    TileSlot s;
    if (a.seg_head && it.item != ~0u && it.done > 0 && it.done < it.len) it.seg = pend;
    if (ah.stage == 1) item_fetch(a, ah, nitems);
    for (;;) {
        while (it.item == ~0u || it.done >= it.len) {
            if (ah.stage == 0) {
                ah.item = a.item_base + atomicAdd(&a.counters[a.ctr_item], 1u);
                ah.stage = 1;
            }
            if (ah.stage == 1) item_fetch(a, ah, nitems);
            const ItemAhead cur = ah;
            ah.stage = 0;
            if (cur.item >= nitems) {
                s.item = ~0u;
                s.in = nullptr;
                s.out = nullptr;
                s.out_len = 0;
                s.cnt = 0;
                s.first = 0;
                s.pad = 0;
                it.item = ~0u;
                it.len = 0;
                it.done = 0;
                return s;
            }
            // Pass 2: claim the following item now; its id and description are needed only when this
            // one is done. (Pass-1 items are long, and an item held back per CTA lengthens the tail
            // by more than the claim costs.)
            if (a.pass != 0) {
                ah.item = a.item_base + atomicAdd(&a.counters[a.ctr_item], 1u);
                ah.stage = 1;
            }
            item_decode(a, cur.item, cur, it);
        }
        if (!a.seg_head) break;
        if (it.len == 0 || it.seg < a.max_segs) break;
        // A chain that leaves the segment storage (pass 1 stopped early): drop the rest of the unit.
        set_error(&a.counters[kCtrErr], kErrCapacity);
        it.done = it.len;
    }
    s.item = it.item;
    // A segment is kTile tuples (32 KB) in either layout; T counts the launch's elements per tile.
    s.pad = 0;
    if (WIN && !a.seg_head) {
        // Words at an odd offset: copy from one word earlier (bulk copies start on 16 bytes).
        const unsigned long long *p = reinterpret_cast<const unsigned long long *>(it.in) + it.done;
        s.pad = (reinterpret_cast<uintptr_t>(p) & 8u) ? 1u : 0u;
        s.in = reinterpret_cast<const tuple_v *>(p - s.pad);
    } else {
        s.in = a.seg_head ? it.in + (uint64_t)it.seg * kTile : it.in + it.done;
    }
    s.out = it.out;
    s.out_len = it.out_len;
    s.cnt = (uint32_t)(it.len - it.done < (uint64_t)T ? it.len - it.done : (uint64_t)T);
    s.first = it.done == 0;
    it.done += s.cnt;
    if (a.seg_head && it.done < it.len) pend = a.seg_next[it.seg];
    return s;
}

// STABLE: tuples of equal digit keep their input order (needed for the build side of joins that report
// the first match in input order). Otherwise the rank of a tuple within its digit is taken with one
// shared-memory atomic, in whatever order the warps reach it: the partitions hold the same tuples,
// and the joins that count every match do not depend on their order.
// NBUF = 2: the next tile streams into a second buffer while this one is processed; NBUF = 1: one
// buffer per CTA, the CTAs of an SM overlap each other's loads instead.
// Store one element of the last pass: a tuple, its compact final word (ci), or - from an 8-byte word of
// a segment-mode pass 1, which holds key >> b1 - the final word with key >> bits.
__device__ __forceinline__ void store_elem(const tuple_v &t, tuple_v *out, unsigned long long *out8, long long dst,
                                           bool ci, int bits, int, bool z0, bool w8o, int b1) {
    if (w8o)
        st_stream8(out8 + dst, w8_word_z0(t.x, t.y, b1, z0));
    else if (ci)
        st_stream8(out8 + dst, ci_word_z0(t.x, t.y, bits, z0));
    else
        st_stream(out + dst, t);
}
__device__ __forceinline__ void store_elem(unsigned long long w, tuple_v *, unsigned long long *out8, long long dst,
                                           bool, int, int b2, bool z0, bool, int) {
    // A pass-1 high part with bit 31 set is a probe key beyond every build key, or (z0) a build key 0.
    const unsigned long long h1 = w >> 32;
    const unsigned long long h = h1 < 0x80000000ull ? h1 >> b2 : (z0 ? 0x80000000ull : 0xffffffffull);
    st_stream8(out8 + dst, (h << 32) | (w & 0xffffffffull));
}

// Elements of a tile: 16-byte tuples, or (WIN) the 8-byte words of a segment-mode pass 1 (w8_word).
template <bool WIN>
struct ScatterElem {
    using type = tuple_v;
};
template <>
struct ScatterElem<true> {
    using type = unsigned long long;
};

// Bytes a tile's bulk copy moves: a bulk copy's size must be a multiple of 16, so a word tile with an odd
// count also copies the next word of its segment (segments hold 4096 words, so an odd count is at most
// 4095 and the extra word stays inside the segment; it lands in an unused buffer slot).
template <typename E>
__device__ __forceinline__ uint32_t tile_copy_bytes(uint32_t cnt) {
    return sizeof(E) == 16 ? cnt * 16u : ((cnt + 1u) & ~1u) * (uint32_t)sizeof(E);
}

// Lanes of the warp whose digit equals this lane's: one ballot per digit bit (NB bits).
template <int NB>
__device__ __forceinline__ unsigned digit_peers(uint32_t d) {
    unsigned peers = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const unsigned bit = (d >> b) & 1u;
        const unsigned bal = __ballot_sync(0xffffffffu, bit);
        peers &= bal ^ (bit - 1u);  // bit ? bal : ~bal
    }
    return peers;
}

// The same for a digit width known only at run time (at most 9 bits; uniform across the warp).
__device__ __forceinline__ unsigned digit_peers_n(uint32_t d, int nbits) {
    switch (nbits) {
        case 6: return digit_peers<6>(d);
        case 7: return digit_peers<7>(d);
        case 8: return digit_peers<8>(d);
        default: break;
    }
    unsigned peers = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 9; b++) {
        if (b < nbits) {
            const unsigned bit = (d >> b) & 1u;
            const unsigned bal = __ballot_sync(0xffffffffu, bit);
            peers &= bal ^ (bit - 1u);
        }
    }
    return peers;
}

// Digit of an element in this pass: (key >> shift) & mask; a word holds key >> b1, which is pass 2's shift.
__device__ __forceinline__ uint32_t elem_digit(const tuple_v &v, int shift, uint64_t dmask) {
    return (uint32_t)((v.x >> shift) & dmask);
}
__device__ __forceinline__ uint32_t elem_digit(unsigned long long v, int, uint64_t dmask) {
    return (uint32_t)((v >> 32) & dmask);
}

template <int THREADS, int ITEMS, bool STABLE, int NBUF, int MINB, bool WIN = false>
__global__ void __launch_bounds__(THREADS, MINB) scatter_kernel(ScatterArgs a) {
    using E = typename ScatterElem<WIN>::type;
    constexpr int T = THREADS * ITEMS;
    // Where the prefetch of the next tile is issued: after this tile's wait barrier (atomic ranks, two
    // buffers; measured faster: one barrier less per tile), or at the top of the iteration (stable
    // ranks: measured faster there, as the rank's ballots keep warp 0 busy after the barrier).
    constexpr bool LATE = NBUF == 2 && !STABLE;
    constexpr int NW = THREADS / 32;
    // Buffer stride: word tiles keep two spare words for a copy that starts one word early (and is
    // rounded up to whole 16-byte units).
    constexpr int ST = T + (WIN ? 2 : 0);
    extern __shared__ __align__(128) unsigned char smem[];
    E *inbuf = reinterpret_cast<E *>(smem);                               // [NBUF][ST]
    long long *gbase = reinterpret_cast<long long *>(inbuf + NBUF * ST);  // [256]
    long long *running = gbase + 256;                                   // [256]
    uint32_t *tdstart = reinterpret_cast<uint32_t *>(running + 256);    // [256]
    uint16_t *whist = reinterpret_cast<uint16_t *>(tdstart + 256);      // STABLE: [NW][F]
    uint32_t *thist = reinterpret_cast<uint32_t *>(tdstart + 256);      // !STABLE: [F] tile histogram
    __shared__ __align__(8) unsigned long long bars[2];
    __shared__ uint32_t scan_tmp[32];
    __shared__ TileSlot slots[2];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int F = a.F;
    const uint64_t dmask = (uint64_t)F - 1;
    const uint32_t nchunks = a.cg.cR + a.cg.cS;
    const uint32_t nitems =
        a.item_end ? a.item_end : (a.pass == 0 ? nchunks * a.cg.spc : nchunks * (uint32_t)a.F1);
    unsigned int *err = &a.counters[kCtrErr];
    const unsigned ltmask = lanemask_lt();
    const uint32_t bar0 = smem_addr(&bars[0]);
    const int nbins = 1 << a.bits;
    const bool ci = a.ci_out && ci_applies(a.counters, a.bits);
    const bool w8o = a.w8_out && w8_fits(a.counters, a.b1);  // pass 1 of the exact pipeline stores words
    const int b2 = a.bits - a.b1;
    if (a.w8 && (a.w8 == 1) != w8_fits(a.counters, a.b1)) return;  // the other layout's launch runs
    __shared__ ItemIter it;  // used by thread 0 only
    uint32_t pend = 0;       // thread 0: next segment of the chain (segment mode)
    ItemAhead ah;            // thread 0: the item claimed ahead
    ah.item = 0;
    ah.stage = 0;
    ah.len = ah.off = 0;
    ah.seg = 0;

    if (!STABLE)
        for (int j = tid; j < 256; j += THREADS) thist[j] = 0;
    if (tid == 0) {
        it = ItemIter();
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (NBUF == 2) {
            const TileSlot s0 = next_tile<T, WIN>(a, it, nitems, pend, ah);
            slots[0] = s0;
            if (s0.item != ~0u && !(a.test_stall && blockIdx.x == 0))
                tma_load_1d(inbuf, s0.in, tile_copy_bytes<E>(s0.cnt + s0.pad), bar0);
        }
    }
    __syncthreads();

    for (uint32_t k = 0;; k++) {
        const uint32_t cur = NBUF == 2 ? (k & 1u) : 0u;
        if (NBUF == 1) {
            // One buffer: load this tile now (the barrier that ended the previous iteration ordered
            // every read of the buffer before this copy).
            if (tid == 0) {
                const TileSlot sn = next_tile<T, WIN>(a, it, nitems, pend, ah);
                slots[0] = sn;
                if (sn.item != ~0u && !(a.test_stall && blockIdx.x == 0 && k == 0))
                    tma_load_1d(inbuf, sn.in, tile_copy_bytes<E>(sn.cnt + sn.pad), bar0);
            }
            __syncthreads();
        }
        const TileSlot sl = slots[cur];
        if (sl.item == ~0u) break;
        E *buf = inbuf + (size_t)cur * ST + sl.pad;
        // Stable ranks: prefetch the next tile into the other buffer now; the barrier that ended the
        // previous iteration ordered every access to it before this copy.
        if (NBUF == 2 && !LATE && tid == 0) {
            const TileSlot sn = next_tile<T, WIN>(a, it, nitems, pend, ah);
            slots[cur ^ 1u] = sn;
            if (sn.item != ~0u)
                tma_load_1d(inbuf + (size_t)(cur ^ 1u) * ST, sn.in, tile_copy_bytes<E>(sn.cnt + sn.pad),
                            bar0 + 8u * (cur ^ 1u));
        }
        // First tile of a work item: load the item's per-digit output offsets.
        if (sl.first && tid < F) {
            long long off;
            if (a.pass == 0) {
                const uint32_t c = sl.item / a.cg.spc;
                off = (long long)(a.unit_off[(size_t)c * a.F1 + tid] + a.subpre[(size_t)sl.item * a.F1 + tid]);
            } else {
                const uint32_t c = sl.item / a.F1, d1 = sl.item % a.F1;
                const int rel = c < a.cg.cR ? 0 : 1;
                const uint32_t v = d1 | ((uint32_t)tid << a.b1);
                off = (long long)(a.start[(size_t)rel * (nbins + 1) + (size_t)d1 * a.F2 + tid] +
                                  a.prefix[(size_t)c * nbins + v]);
            }
            running[tid] = off;
        }
        const uint32_t cnt = sl.cnt;
        const uint32_t par = NBUF == 2 ? ((k >> 1) & 1u) : (k & 1u);
        const bool ok = mbar_wait(bar0 + 8u * cur, par);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                set_error(err, kErrSpinLimit);
                // Before leaving, let every copy this CTA issued land (bounded waits as well): no copy
                // may write into shared memory the CTA no longer owns. The load into this buffer was
                // issued unless the stall hook withheld it (CTA 0's first tile); a prefetch into the
                // other buffer is in flight only with stable ranks (issued above) if it has a tile.
                if (!(a.test_stall && blockIdx.x == 0 && k == 0)) mbar_wait(bar0 + 8u * cur, par);
                if (NBUF == 2 && !LATE && slots[cur ^ 1u].item != ~0u)
                    mbar_wait(bar0 + 8u * (cur ^ 1u), ((k + 1) >> 1) & 1u);
            }
            break;
        }
        // Atomic ranks: prefetch the next tile into the other buffer now. Every thread has passed the
        // barrier above, so the previous tile's staging and write-out, the last accesses to that
        // buffer, are done, and no barrier has to end the iteration.
        if (NBUF == 2 && LATE && tid == 0) {
            const TileSlot sn = next_tile<T, WIN>(a, it, nitems, pend, ah);
            slots[cur ^ 1u] = sn;
            if (sn.item != ~0u)
                tma_load_1d(inbuf + (size_t)(cur ^ 1u) * ST, sn.in, tile_copy_bytes<E>(sn.cnt + sn.pad),
                            bar0 + 8u * (cur ^ 1u));
        }

        // Elements of this tile: warp w owns [w*32*ITEMS, (w+1)*32*ITEMS), one row of 32 per item.
        E v[ITEMS];
        uint32_t d[ITEMS];
        const bool full = cnt == (uint32_t)T;
        if (full) {
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                v[i] = buf[w * 32 * ITEMS + i * 32 + lane];
                d[i] = elem_digit(v[i], a.shift, dmask);
            }
        } else {
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const uint32_t idx = (uint32_t)(w * 32 * ITEMS + i * 32 + lane);
                if (idx < cnt) {
                    v[i] = buf[idx];
                    d[i] = elem_digit(v[i], a.shift, dmask);
                } else {
                    v[i] = E{};
                    d[i] = (uint32_t)F;
                }
            }
        }
        uint32_t rk[ITEMS];
        if constexpr (STABLE) {
            uint16_t *wh = whist + w * F;
            for (int j = lane; j < F; j += 32) wh[j] = 0;
            __syncwarp();
            // Stable rank within the warp: items in order, lanes in order. The lanes holding the same
            // digit are found with one ballot per digit bit (plus the bit that marks padding lanes of
            // a partial tile), which is cheaper here than match.any.
            const int nbits = a.logF + (cnt < (uint32_t)T ? 1 : 0);
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                // A row of padding only (a partial tile): nothing to rank (uniform across the warp).
                if ((uint32_t)(w * 32 * ITEMS + i * 32) >= cnt) {
                    rk[i] = 0;
                    continue;
                }
                const unsigned peers = digit_peers_n(d[i], nbits);
                const bool valid = d[i] < (uint32_t)F;
                uint32_t pre = 0;
                if (valid) pre = wh[d[i]];
                rk[i] = pre + __popc(peers & ltmask);
                __syncwarp();
                if (valid && (peers & ltmask) == 0) wh[d[i]] = (uint16_t)(pre + __popc(peers));
                __syncwarp();
            }
            __syncthreads();
            // Tile histogram per digit and exclusive prefix over warps.
            uint32_t h = 0;
            if (tid < F) {
                for (int q = 0; q < NW; q++) {
                    const uint32_t c = whist[q * F + tid];
                    whist[q * F + tid] = (uint16_t)h;
                    h += c;
                }
            }
            const uint32_t ex = block_excl_scan_u32(tid < F ? h : 0u, scan_tmp, nullptr);
            if (tid < F) {
                tdstart[tid] = ex;
                gbase[tid] = running[tid] - (long long)ex;
                running[tid] += h;
            }
        } else {
#pragma unroll
            for (int i = 0; i < ITEMS; i++)
                if (d[i] < (uint32_t)F) rk[i] = atomicAdd(&thist[d[i]], 1u);
            __syncthreads();
            // Warp 0 scans the tile histogram: lane l owns digits [l*K, l*K + K).
            if (w == 0) {
                const int K = (F + 31) >> 5;
                const int d0 = lane * K;
                uint32_t hv[8];
                uint32_t sum = 0;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    hv[j] = (j < K && d0 + j < F) ? thist[d0 + j] : 0u;
                    sum += hv[j];
                }
                uint32_t incl = sum;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                uint32_t ex = incl - sum;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if (j < K && d0 + j < F) {
                        const int dd = d0 + j;
                        thist[dd] = 0;
                        tdstart[dd] = ex;
                        const long long r0 = running[dd];
                        gbase[dd] = r0 - (long long)ex;
                        running[dd] = r0 + hv[j];
                        ex += hv[j];
                    }
                }
            }
        }
        __syncthreads();
        // Stage the tile sorted by digit, in place (the digit is recomputed: fewer live registers).
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t idx = (uint32_t)(w * 32 * ITEMS + i * 32 + lane);
            if (full || idx < cnt) {
                const uint32_t di = elem_digit(v[i], a.shift, dmask);
                const uint32_t pos = tdstart[di] + (STABLE ? whist[w * F + di] : 0u) + rk[i];
                buf[pos] = v[i];
            }
        }
        __syncthreads();
        // Write each digit run: consecutive threads write consecutive 16-byte tuples (8-byte words for
        // compact final partitions). Full tiles load their staged tuples in two halves so that the stores
        // issue back to back.
        // A destination outside the output (negative included) fails the unsigned bound check. Build
        // key-0 words exist only for first-match joins (ci_z0), in the launches of the build relation.
        unsigned long long *out8 = sl.out == a.outS ? a.outS8 : a.outR8;
        const bool z0 = a.ci_z0 && sl.out == a.outR;
        if (full) {
#pragma unroll
            for (int hh = 0; hh < 2; hh++) {
                E t[ITEMS / 2];
                long long dst[ITEMS / 2];
#pragma unroll
                for (int i = 0; i < ITEMS / 2; i++) t[i] = buf[tid + (hh * ITEMS / 2 + i) * THREADS];
#pragma unroll
                for (int i = 0; i < ITEMS / 2; i++)
                    dst[i] = gbase[elem_digit(t[i], a.shift, dmask)] + (long long)(tid + (hh * ITEMS / 2 + i) * THREADS);
#pragma unroll
                for (int i = 0; i < ITEMS / 2; i++) {
                    if ((uint64_t)dst[i] < sl.out_len)
                        store_elem(t[i], sl.out, out8, dst[i], ci, a.bits, b2, z0, w8o, a.b1);
                    else
                        set_error(err, kErrBounds);
                }
            }
        } else
        for (uint32_t j = tid; j < cnt; j += THREADS) {
            const E t = buf[j];
            const long long dst = gbase[elem_digit(t, a.shift, dmask)] + (long long)j;
            if ((uint64_t)dst < sl.out_len)
                store_elem(t, sl.out, out8, dst, ci, a.bits, b2, z0, w8o, a.b1);
            else
                set_error(err, kErrBounds);
        }
        // The next copy into this buffer (at the top of the next iteration with one buffer or stable
        // ranks) must wait for this write-out; otherwise the next tile's wait barrier orders them.
        if (!LATE) __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------------
// 5b. Segment mode, pass 1: partition into chains of segments, counting the histograms on the way.
//
// The exact-offset pipeline reads both relations once for histograms before pass 1 may write. For
// the joins that count every match, the order of tuples within a partition does not matter, and
// pass 1 can write without knowing offsets: every (CTA, relation, pass-1 digit) owns a chain of
// kTile-tuple segments, taken from a global counter (in slabs of kSegSlab per CTA), filled in order
// and linked through seg_next. Since a tile holds at most kTile tuples of one digit, a tile's run of
// a digit ends the current segment at most once. The same CTA counts the joint histogram of the low
// `bits` key bits of its tuples in 16-bit counters (two per word), and adds them to its row of hist
// when the relation ends. No counter overflows: `since` bounds every counter (a tile adds at most its
// size), and before a tile could take the bound past 65535 the CTA moves every counter above
// kSegSpillAt into its row and sets the bound to the largest counter left. That gives pass 2 its exact
// offsets: pass 2 takes (CTA, digit) chains as its units and writes the final partitions as in the
// exact-offset pipeline.
// ------------------------------------------------------------------------------------------------
constexpr uint32_t kSegNone = 0xffffffffu;
constexpr uint32_t kSegSlab = 32;          // segment ids a CTA takes from the global counter at once
constexpr int kSegCtasPerSm = 2;           // shared memory: two tile buffers + 32 KB of counters
constexpr int kSegMaxBits = 14;
constexpr uint32_t kSegSpillAt = 8192;

struct SegArgs {
    const tuple_v *R, *S;
    uint64_t nR, nS;
    int bits, F1;              // joint bins 2^bits; pass-1 digit = key & (F1 - 1)
    int b1;                    // log2(F1)
    int w8_first;              // a pass that wrote 8-byte words ran first: run only if w8_fits fails
    uint32_t it_tiles;         // tiles per work item
    uint32_t tilesR, tilesS;   // tiles of each relation
    uint32_t itemsR, items;    // items of R (first), all items
    tuple_v *out;              // segment storage: segment i holds tuples [i*kTile, (i+1)*kTile)
    uint32_t max_segs;
    uint32_t *seg_head;        // [2*grid][F1]
    uint32_t *seg_next;        // [max_segs]
    uint32_t *hist;            // [2*grid][2^bits]: row c = R tuples of CTA c, row grid + c = its S tuples
    uint32_t *counters;        // kCtrItem1 (items), kCtrSegAlloc, kCtrErr, kCtrMaxKey/kCtrMaxRid
    int test_stall;            // test hook: CTA 0 withholds its first tile load (its wait must expire)
};

struct SegSlot {
    const tuple_v *in;
    uint32_t cnt;              // tuples in the tile (0: no more tiles)
    int rel;
};

// Where a digit's run of the staged tile goes: staged index j < split to base + j (the rest of the
// current segment), j >= split to base2 + j (the new segment).
struct SegRun {
    long long base, base2;
    uint32_t split, pad;
};

// Thread 0: the next tile of this CTA's current work item, claiming items as needed. STATIC_R: the build
// relation's items [r_next, r_end) belong to this CTA and come first, in order; the probe relation's
// items are claimed from the counter.
template <bool STATIC_R>
__device__ __forceinline__ SegSlot seg_next_tile(const SegArgs &a, uint32_t &item, uint32_t &t_next,
                                                 uint32_t &t_end, uint32_t &r_next, uint32_t r_end) {
    SegSlot s;
    while (item == ~0u || t_next >= t_end) {
        if (STATIC_R && r_next < r_end)
            item = r_next++;
        else
            item = atomicAdd(&a.counters[kCtrItem1], 1u) + (STATIC_R ? a.itemsR : 0u);
        if (item >= a.items) {
            item = ~0u;
            s.in = nullptr;
            s.cnt = 0;
            s.rel = 0;
            return s;
        }
        const bool rel = item >= a.itemsR;
        const uint32_t k = rel ? item - a.itemsR : item;
        const uint32_t nt = rel ? a.tilesS : a.tilesR;
        t_next = k * a.it_tiles;
        t_end = t_next + a.it_tiles < nt ? t_next + a.it_tiles : nt;
    }
    const bool rel = item >= a.itemsR;
    const uint64_t n = rel ? a.nS : a.nR;
    const uint64_t lo = (uint64_t)t_next * kTile;
    s.in = (rel ? a.S : a.R) + lo;
    s.cnt = (uint32_t)(n - lo < (uint64_t)kTile ? n - lo : (uint64_t)kTile);
    s.rel = rel ? 1 : 0;
    t_next++;
    return s;
}

// Add the CTA's 16-bit counter pairs to its histogram row (reductions: no round trip) and clear them.
// All threads; the caller synchronises before and after.
__device__ __forceinline__ void seg_flush(uint32_t *jh, uint32_t *row, int nbins) {
    for (int w = threadIdx.x; w < (nbins >> 1); w += blockDim.x) {
        const uint32_t v = jh[w];
        if (!v) continue;
        jh[w] = 0;
        if (v & 0xffffu) atomicAdd(&row[2 * w], v & 0xffffu);
        if (v >> 16) atomicAdd(&row[2 * w + 1], v >> 16);
    }
}

// K = ceil(F1 / 32): pass-1 digits per lane of warp 0, which keeps their segment state in registers.
// W8: store 8-byte words (w8_word) in segments of 2 * kTile words (the same 32 KB); the launch that stores
// tuples after it runs only when the widths did not allow words (w8_first).
// STABLE_R (first-match joins): every build-relation chain keeps input order. CTA c takes the build
// relation's items [c * itemsR / G, (c + 1) * itemsR / G) in order before any probe item, and ranks
// their tiles stably (warp-ordered ballots, as the stable scatter does), so pass 2, which writes each
// digit's chains in CTA order and each chain in order, leaves every final build partition in input
// order. Probe tiles keep the atomic rank: their order inside a partition changes no result.
// Build key 0 of first-match joins needs nothing here: its word (high part 0) reaches key 0's final
// partition, whose joins skip it (JoinItem::part0); a select per word cost pass 1 3%.
template <int THREADS, int ITEMS, int K, bool W8 = false, bool STABLE_R = false>
__global__ void __launch_bounds__(THREADS, kSegCtasPerSm) seg_pass1_kernel(SegArgs a) {
    constexpr int T = THREADS * ITEMS;
    static_assert(T == kTile, "a tile fills one segment of tuples");
    constexpr uint32_t SEGW = W8 ? 2 * T : T;  // elements per segment
    if (!W8 && a.w8_first && w8_fits(a.counters, a.b1)) return;
    unsigned long long *out8 = reinterpret_cast<unsigned long long *>(a.out);
    static_assert(K >= 1 && K <= 8, "at most 256 pass-1 digits");
    extern __shared__ __align__(128) unsigned char smem[];
    tuple_v *inbuf = reinterpret_cast<tuple_v *>(smem);              // [2][T]
    SegRun *runs = reinterpret_cast<SegRun *>(inbuf + 2 * T);          // [256] where each digit's run goes
    uint32_t *thist = reinterpret_cast<uint32_t *>(runs + 256);        // [256] tile histogram
    uint32_t *tdstart = thist + 256;                                   // [256] digit start in the staged tile
    uint32_t *jh = tdstart + 256;                                      // [2^bits / 2] counter pairs
    uint16_t *whist = reinterpret_cast<uint16_t *>(jh + (1 << a.bits) / 2);  // STABLE_R: [warps][F1]
    __shared__ __align__(8) unsigned long long bars[2];
    __shared__ SegSlot slots[2];
    __shared__ uint32_t s_item, s_tnext, s_tend, s_rnext, s_rend;  // thread 0's item iterator

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int F = a.F1;
    const uint32_t dmask = (uint32_t)F - 1u;
    const int nbins = 1 << a.bits;
    const uint64_t bmask = (uint64_t)nbins - 1;
    const uint32_t G = gridDim.x, c = blockIdx.x;
    unsigned int *err = &a.counters[kCtrErr];
    const uint32_t bar0 = smem_addr(&bars[0]);
    const uint64_t cap = (uint64_t)a.max_segs * SEGW;

    for (int j = tid; j < 256; j += THREADS) thist[j] = 0;
    for (int j = tid; j < (nbins >> 1); j += THREADS) jh[j] = 0;
    // Warp 0, lane l: current segment and fill of digits l*K .. l*K + K - 1.
    uint32_t scur[K], sfill[K];
#pragma unroll
    for (int j = 0; j < K; j++) {
        scur[j] = kSegNone;
        sfill[j] = 0;
    }
    // This CTA's rows of hist start at zero; counters are added to them.
    for (int j = tid; j < 2 * nbins; j += THREADS)
        a.hist[((size_t)(j >= nbins ? G : 0) + c) * nbins + (j >= nbins ? j - nbins : j)] = 0;
    uint32_t slab_lo = 0, slab_rem = 0;  // thread 0 (lane 0 of warp 0): ids left in this CTA's slab
    if (tid == 0) {
        s_item = ~0u;
        s_tnext = s_tend = 0;
        s_rnext = (uint32_t)((uint64_t)c * a.itemsR / G);
        s_rend = (uint32_t)((uint64_t)(c + 1) * a.itemsR / G);
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        uint32_t item = s_item, tn = s_tnext, te = s_tend, rn = s_rnext;
        const SegSlot s0 = seg_next_tile<STABLE_R>(a, item, tn, te, rn, s_rend);
        s_item = item;
        s_tnext = tn;
        s_tend = te;
        s_rnext = rn;
        slots[0] = s0;
        if (s0.cnt && !(a.test_stall && blockIdx.x == 0)) tma_load_1d(inbuf, s0.in, s0.cnt * 16u, bar0);
    }
    __syncthreads();

    int phase_rel = 0;           // relation whose tuples the counters and segment state hold
    uint32_t since = 0;          // upper bound of every counter (uniform)
    // ORs of the high 32 bits of build keys, build row ids and probe row ids: every width test
    // (w8_fits, ci_applies, compact_applies) compares with a power of two of 2^32 or more.
    uint32_t kor = 0, ror = 0, rors = 0;
    __shared__ uint32_t s_max[THREADS / 32];

    for (uint32_t k = 0;; k++) {
        const uint32_t cur = k & 1u;
        const SegSlot sl = slots[cur];
        if (sl.cnt == 0) break;
        tuple_v *buf = inbuf + (size_t)cur * T;
        // R tiles come before S tiles in every CTA's sequence: on the first S tile, R's counters go
        // to their row and the segment state starts over.
        if (sl.rel != phase_rel) {
            seg_flush(jh, a.hist + ((size_t)phase_rel * G + c) * nbins, nbins);
#pragma unroll
            for (int j = 0; j < K; j++) {
                scur[j] = kSegNone;
                sfill[j] = 0;
            }
            phase_rel = sl.rel;
            since = 0;
            __syncthreads();
        }
        const uint32_t cnt = sl.cnt;
        if (since + cnt > 65535u) {
            // Move the large counters to the row; the largest one kept is the new bound.
            uint32_t *hrow = a.hist + ((size_t)phase_rel * G + c) * nbins;
            uint32_t mx = 0;
            for (int q = tid; q < (nbins >> 1); q += THREADS) {
                const uint32_t v0 = jh[q];
                uint32_t lo = v0 & 0xffffu, hi = v0 >> 16;
                if (lo > kSegSpillAt) {
                    atomicAdd(&hrow[2 * q], lo);
                    lo = 0;
                }
                if (hi > kSegSpillAt) {
                    atomicAdd(&hrow[2 * q + 1], hi);
                    hi = 0;
                }
                if (v0 != (lo | (hi << 16))) jh[q] = lo | (hi << 16);
                mx = max(mx, max(lo, hi));
            }
            mx = __reduce_max_sync(0xffffffffu, mx);
            if (lane == 0) s_max[w] = mx;
            __syncthreads();
            since = 0;
#pragma unroll
            for (int q = 0; q < THREADS / 32; q++) since = max(since, s_max[q]);
            __syncthreads();
        }
        since += cnt;
        const bool ok = mbar_wait(bar0 + 8u * cur, (k >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                set_error(err, kErrSpinLimit);
                // Let this buffer's copy land first (bounded), unless the stall hook withheld it (CTA 0's
                // first tile); nothing else is in flight (the next tile's copy is issued below).
                if (!(a.test_stall && blockIdx.x == 0 && k == 0)) mbar_wait(bar0 + 8u * cur, (k >> 1) & 1u);
            }
            break;
        }
        // Prefetch the next tile into the other buffer: every thread has passed the barrier above, so
        // the previous tile's staging and write-out, the last accesses to that buffer, are done.
        if (tid == 0) {
            uint32_t item = s_item, tn = s_tnext, te = s_tend, rn = s_rnext;
            const SegSlot sn = seg_next_tile<STABLE_R>(a, item, tn, te, rn, s_rend);
            s_item = item;
            s_tnext = tn;
            s_tend = te;
            s_rnext = rn;
            slots[cur ^ 1u] = sn;
            if (sn.cnt) tma_load_1d(inbuf + (size_t)(cur ^ 1u) * T, sn.in, sn.cnt * 16u, bar0 + 8u * (cur ^ 1u));
        }

        tuple_v v[ITEMS];
        uint32_t rk[ITEMS];
        const bool st = STABLE_R && sl.rel == 0;  // uniform: this tile takes the stable rank
        uint32_t xo = 0, yo = 0;
        if (cnt == (uint32_t)T) {
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                v[i] = buf[w * 32 * ITEMS + i * 32 + lane];
                const uint32_t d = (uint32_t)v[i].x & dmask;
                if (!st) rk[i] = atomicAdd(&thist[d], 1u);
                const uint32_t bin = (uint32_t)(v[i].x & bmask);
                atomicAdd(&jh[bin >> 1], 1u << ((bin & 1u) << 4));
                xo |= (uint32_t)(v[i].x >> 32);
                yo |= (uint32_t)(v[i].y >> 32);
            }
        } else {
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const uint32_t idx = (uint32_t)(w * 32 * ITEMS + i * 32 + lane);
                if (idx < cnt) {
                    v[i] = buf[idx];
                    const uint32_t d = (uint32_t)v[i].x & dmask;
                    if (!st) rk[i] = atomicAdd(&thist[d], 1u);
                    const uint32_t bin = (uint32_t)(v[i].x & bmask);
                    atomicAdd(&jh[bin >> 1], 1u << ((bin & 1u) << 4));
                    xo |= (uint32_t)(v[i].x >> 32);
                    yo |= (uint32_t)(v[i].y >> 32);
                }
            }
        }
        if (sl.rel == 0) {
            kor |= xo;
            ror |= yo;
        } else {
            rors |= yo;
        }
        if (STABLE_R && st) {
            // Stable rank within the warp: items in order, lanes in order; the lanes holding one digit
            // are found with one ballot per digit bit (plus the bit that marks padding lanes).
            uint16_t *wh = whist + w * F;
            for (int j = lane; j < F; j += 32) wh[j] = 0;
            __syncwarp();
            const unsigned ltmask = lanemask_lt();
            // Digit bits: K = F1 / 32 for K >= 2 gives log2(F1) exactly; K = 1 covers F1 <= 32 with 5
            // bits (the unused high bits are zero in every lane). A partial tile's padding lanes carry
            // digit F1, one bit more.
            constexpr int NB = K == 1 ? 5 : K == 2 ? 6 : K == 4 ? 7 : 8;
            const bool fullt = cnt == (uint32_t)T;
#pragma unroll
            for (int i = 0; i < ITEMS; i++) {
                const uint32_t idx = (uint32_t)(w * 32 * ITEMS + i * 32 + lane);
                const uint32_t d = idx < cnt ? (uint32_t)v[i].x & dmask : (uint32_t)F;
                const unsigned peers = fullt ? digit_peers<NB>(d) : digit_peers<NB + 1>(d);
                const bool valid = d < (uint32_t)F;
                uint32_t pre = 0;
                if (valid) pre = wh[d];
                rk[i] = pre + __popc(peers & ltmask);
                __syncwarp();
                if (valid && (peers & ltmask) == 0) wh[d] = (uint16_t)(pre + __popc(peers));
                __syncwarp();
            }
            __syncthreads();
            // Tile count per digit, and each warp's start within the digit's run.
            if (tid < F) {
                uint32_t h = 0;
                for (int q = 0; q < THREADS / 32; q++) {
                    const uint32_t n = whist[q * F + tid];
                    whist[q * F + tid] = (uint16_t)h;
                    h += n;
                }
                thist[tid] = h;
            }
        }
        __syncthreads();
        // Warp 0, step 1: digit starts in the staged tile, and which digits' runs need a new segment
        // (a run that does not fit the rest of its current segment). Lane l owns digits [l*K, l*K + K).
        uint32_t hv[K];      // warp 0: tile count of each owned digit
        uint32_t exl = 0;    // warp 0: tuples (low 16 bits) and new segments (high 16 bits) before lane l
        uint32_t ntot = 0;   // warp 0: new segments of the tile
        if (w == 0) {
            const int d0 = lane * K;
            uint32_t packed = 0;
#pragma unroll
            for (int j = 0; j < K; j++) {
                hv[j] = d0 + j < F ? thist[d0 + j] : 0u;
                const bool nw = hv[j] && (scur[j] == kSegNone || sfill[j] + hv[j] > SEGW);
                packed += hv[j] + (nw ? 0x10000u : 0u);
            }
            uint32_t incl = packed;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            ntot = __shfl_sync(0xffffffffu, incl, 31) >> 16;
            exl = incl - packed;
            uint32_t ex = exl & 0xffffu;
#pragma unroll
            for (int j = 0; j < K; j++) {
                const int d = d0 + j;
                if (d < F) {
                    thist[d] = 0;
                    tdstart[d] = ex;
                    ex += hv[j];
                }
            }
        }
        __syncthreads();
        // Stage the tile sorted by digit, in place.
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t idx = (uint32_t)(w * 32 * ITEMS + i * 32 + lane);
            if (idx < cnt) {
                const uint32_t d = (uint32_t)v[i].x & dmask;
                buf[tdstart[d] + (STABLE_R && st ? (uint32_t)whist[w * F + d] : 0u) + rk[i]] = v[i];
            }
        }
        // Warp 0, step 2 (while the other warps stage): where each digit's run goes, the rest of its
        // current segment, then (when that fills) a new segment.
        if (w == 0) {
            const int d0 = lane * K;
            // New segment ids: first what is left of the slab, then a fresh slab.
            uint32_t old_lo = 0, old_rem = 0, nb = 0;
            if (ntot) {
                if (lane == 0) {
                    old_lo = slab_lo;
                    old_rem = slab_rem;
                    if (ntot <= slab_rem) {
                        slab_lo += ntot;
                        slab_rem -= ntot;
                    } else {
                        const uint32_t deficit = ntot - slab_rem;
                        const uint32_t take = deficit > kSegSlab ? deficit : kSegSlab;
                        nb = atomicAdd(&a.counters[kCtrSegAlloc], take);
                        slab_lo = nb + deficit;
                        slab_rem = take - deficit;
                    }
                }
                old_lo = __shfl_sync(0xffffffffu, old_lo, 0);
                old_rem = __shfl_sync(0xffffffffu, old_rem, 0);
                nb = __shfl_sync(0xffffffffu, nb, 0);
            }
            uint32_t ex = exl & 0xffffu, e = exl >> 16;
#pragma unroll
            for (int j = 0; j < K; j++) {
                const int d = d0 + j;
                if (d < F) {
                    const uint32_t h = hv[j];
                    if (h) {
                        const uint32_t sc = scur[j], fill = sfill[j];
                        SegRun r;
                        if (sc != kSegNone && fill + h <= SEGW) {
                            r.base = r.base2 = (long long)sc * SEGW + fill - ex;
                            r.split = ex + h;
                            sfill[j] = fill + h;
                        } else {
                            const uint32_t id = e < old_rem ? old_lo + e : nb + (e - old_rem);
                            e++;
                            if (id < a.max_segs) {
                                if (sc == kSegNone) {
                                    // The whole run starts the chain.
                                    a.seg_head[((size_t)phase_rel * G + c) * F + d] = id;
                                    r.base = r.base2 = (long long)id * SEGW - ex;
                                    r.split = ex + h;
                                    sfill[j] = h;
                                } else {
                                    // The run fills the current segment, then goes on in segment
                                    // id: staged index ex + (SEGW - fill) lands at id * SEGW.
                                    a.seg_next[sc] = id;
                                    r.base = (long long)sc * SEGW + fill - ex;
                                    r.base2 = r.base + ((long long)id - (long long)sc - 1) * SEGW;
                                    r.split = ex + (SEGW - fill);
                                    sfill[j] = h - (SEGW - fill);
                                }
                                scur[j] = id;
                            } else {
                                // Cannot happen with the storage phj_carve reserves; the run's
                                // stores fail their bounds check and report it.
                                set_error(err, kErrCapacity);
                                r.base = r.base2 = -(long long)cap - (long long)SEGW;
                                r.split = ex + h;
                                scur[j] = kSegNone;
                                sfill[j] = 0;
                            }
                        }
                        runs[d] = r;
                    }
                    ex += h;
                }
            }
        }
        __syncthreads();
        // Write each digit run: consecutive threads write consecutive 16-byte tuples (8-byte words).
        // A destination outside the segment storage (negative included) fails the unsigned bound check.
        if (cnt == (uint32_t)T) {
#pragma unroll
            for (int hh = 0; hh < 2; hh++) {
                tuple_v t[ITEMS / 2];
                long long dst[ITEMS / 2];
#pragma unroll
                for (int i = 0; i < ITEMS / 2; i++) t[i] = buf[tid + (hh * ITEMS / 2 + i) * THREADS];
#pragma unroll
                for (int i = 0; i < ITEMS / 2; i++) {
                    const uint32_t j = (uint32_t)(tid + (hh * ITEMS / 2 + i) * THREADS);
                    const SegRun r = runs[(uint32_t)t[i].x & dmask];
                    dst[i] = (j < r.split ? r.base : r.base2) + (long long)j;
                }
#pragma unroll
                for (int i = 0; i < ITEMS / 2; i++) {
                    if ((uint64_t)dst[i] < cap) {
                        if (W8)
                            st_stream8(out8 + dst[i], w8_word(t[i].x, t[i].y, a.b1));
                        else
                            st_stream(a.out + dst[i], t[i]);
                    } else {
                        set_error(err, kErrBounds);
                    }
                }
            }
        } else {
            for (uint32_t j = tid; j < cnt; j += THREADS) {
                const tuple_v t = buf[j];
                const SegRun r = runs[(uint32_t)t.x & dmask];
                const long long dst = (j < r.split ? r.base : r.base2) + (long long)j;
                if ((uint64_t)dst < cap) {
                    if (W8)
                        st_stream8(out8 + dst, w8_word(t.x, t.y, a.b1));
                    else
                        st_stream(a.out + dst, t);
                } else {
                    set_error(err, kErrBounds);
                }
            }
        }
        // No barrier here: the next tile's wait barrier orders this write-out before the next prefetch
        // into this buffer and before the next tile's planning rewrites runs and tdstart.
    }
    // The counters of the relation in progress go to their row (the other row is complete).
    __syncthreads();
    seg_flush(jh, a.hist + ((size_t)phase_rel * G + c) * nbins, nbins);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kor |= __shfl_xor_sync(0xffffffffu, kor, o);
        ror |= __shfl_xor_sync(0xffffffffu, ror, o);
        rors |= __shfl_xor_sync(0xffffffffu, rors, o);
    }
    if (lane == 0 && (kor | ror | rors)) {
        unsigned long long *mx = reinterpret_cast<unsigned long long *>(a.counters + kCtrMaxKey);
        if (kor) atomicOr(mx, (unsigned long long)kor << 32);
        if (ror) atomicOr(mx + 1, (unsigned long long)ror << 32);
        if (rors) atomicOr(mx + 2, (unsigned long long)rors << 32);
    }
}

// After a pass 1 that wrote 8-byte words: if the widths did not allow them, pass 1 runs again with
// tuples, from fresh item and segment counters (its own CTAs zero their histogram rows).
__global__ void seg_reset_if_wide(uint32_t *counters, int b1) {
    if (threadIdx.x == 0 && !w8_fits(counters, b1)) {
        counters[kCtrItem1] = 0;
        counters[kCtrSegAlloc] = 0;
    }
}

// 4. Partition join in shared memory.
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return smem_addr(p); }

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
    int lp;     // first match per probe tuple (lowest build position) instead of all matches
    int skip0;  // build tuples with key 0 never match (key 0 marks an empty slot in lp_join)
    JoinAccum *acc;
    MatOut mat; // materialising joins (MAT kernels): where the (r.row_id, s.row_id) pairs go
    int ci;     // the final partitions may be compact words (when ci_applies holds) at finR8 / finS8
    const unsigned long long *finR8, *finS8;
    int w8_b1;  // a pass 1 that may store words (either pipeline): its shift (reported when w8_fits held); -1 otherwise
};

// A tuple of a final partition: the stored tuple, or for compact partitions {key >> bits, row id}.
// Joins compare x for equality and hash x >> shift with shift = bits (tuples) or 0 (compact words).
__device__ __forceinline__ tuple_v ld_fin(const tuple_v *p16, const unsigned long long *p8, uint64_t i, bool ci) {
    if (ci) {
        const unsigned long long w = ld_stream8(p8 + i);
        return make_ulonglong2(w >> 32, w & 0xffffffffull);
    }
    return ld_stream(p16 + i);
}

__device__ __forceinline__ tuple_v fin_r(const JoinArgs &a, bool ci, uint64_t i) {
    if (ci) {
        const unsigned long long w = a.finR8[i];
        return make_ulonglong2(w >> 32, w & 0xffffffffull);
    }
    return a.finR[i];
}

constexpr int kHeadMax = 16384;  // next_pow_2(kSmemCap)
constexpr size_t kJoinSmem = (size_t)kSmemCap * 16 + kHeadMax * 2 + (size_t)kSmemCap * 2;

// The compact table applies when every build key, shifted right by the radix bits, and every build
// row id fit in 32 bits (OR of all of them gathered by the histogram pass).
__device__ __forceinline__ bool compact_applies(const JoinArgs &a) {
    const unsigned long long *mx = reinterpret_cast<const unsigned long long *>(a.counters + kCtrMaxKey);
    return (mx[0] >> a.bits) < (1ull << 32) && mx[1] < (1ull << 32);
}

constexpr size_t kCompactSmem = (size_t)kCompactCap * (4 + 4 + 2 + 2);

// First-match joins: record (acc->dup_flag) that some probe tuple of this block matched two or more
// build tuples. Only then does the first match depend on the order inside a build partition; a join
// whose partition passes ranked the build relation without keeping its input order is then run again
// with ordered passes. Called by every thread of the block.
__device__ __forceinline__ void flag_multi(bool multi, unsigned int *flag) {
    if (__syncthreads_or(multi) && threadIdx.x == 0) atomicOr(flag, 1u);
}

// Partition join with 4-byte keys (key >> bits) and 4-byte row ids in shared memory, packed into one
// 8-byte word per build tuple (key-high << 32 | row id: one load per visited node): 96 KiB per CTA,
// two CTAs per SM, so one CTA's build overlaps the other's probe. Same results as join_small_kernel;
// within a partition the low `bits` key bits are equal, so comparing key >> bits is comparing keys.
// MAT: write one (r.row_id, s.row_id) pair per match (the ptr_* joins) instead of summing; the probe
// then runs in block-wide rounds (count, reserve output slots, walk again and write). LP: first match
// (the lowest build position) per probe tuple.
template <bool MAT, bool CI = false, bool LP = false>
__global__ void __launch_bounds__(kCompactThreads, 2) join_compact_kernel(JoinArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned long long *rw = reinterpret_cast<unsigned long long *>(smem);  // [kCompactCap]
    uint16_t *head = reinterpret_cast<uint16_t *>(rw + kCompactCap);         // [kCompactCap]
    uint16_t *nxt = head + kCompactCap;                                      // [kCompactCap]
    __shared__ unsigned long long red[64];
    __shared__ uint32_t s_item;
    __shared__ uint32_t scan_tmp[32];
    __shared__ unsigned long long s_base;
    if (!compact_applies(a)) return;
    const int tid = threadIdx.x;
    unsigned int *err = &a.counters[kCtrErr];
    const uint32_t nA = a.counters[kCtrNItemsA];
    // Compiled once per partition layout; only the launch matching the device's choice runs.
    if (CI != (!MAT && a.ci && ci_applies(a.counters, a.bits))) return;
    constexpr bool ci = CI;
    const int B = ci ? 0 : a.bits;  // shift from a stored x to the key's bits above the radix bits
    constexpr bool lp = LP;
    const bool skip0 = a.skip0 != 0;
    unsigned long long cnt = 0, sum = 0;
    bool multi = false;  // first-match joins: a probe tuple matched two build tuples
    for (;;) {
        if (tid == 0) s_item = atomicAdd(&a.counters[kCtrItemA], 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= nA) break;
        const JoinItem item = a.items[it];
        const uint32_t nr = item.r_len;
        const uint32_t nb = next_pow2_u32(nr);
        const uint64_t hmask = nb - 1;
        uint32_t *head32 = reinterpret_cast<uint32_t *>(head);
        for (uint32_t q = tid; q < (nb + 1) / 2; q += kCompactThreads) head32[q] = 0;
        __syncthreads();
        // Load and chain the build side; lp_join skips key 0, which reads as an empty slot there (in
        // compact final partitions such a key's words have a high part that no probe word has).
        const tuple_v *R = a.finR + item.r_begin;
        const unsigned long long *R8 = a.finR8 + item.r_begin;
        for (uint32_t i0 = tid; i0 < nr; i0 += 4 * kCompactThreads) {
            tuple_v t[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t i = i0 + u * kCompactThreads;
                t[u] = i < nr ? ld_fin(R, R8, i, ci) : make_ulonglong2(0, 0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t i = i0 + u * kCompactThreads;
                if (i >= nr) continue;
                rw[i] = ((t[u].x >> B) << 32) | (t[u].y & 0xffffffffull);
                if (skip0 && t[u].x == 0 && (!ci || item.part0)) continue;
                nxt[i] = (uint16_t)atomic_exch_u16(&head[(t[u].x >> B) & hmask], i + 1);
            }
        }
        __syncthreads();
        const tuple_v *S = a.finS + item.s_begin;
        const unsigned long long *S8 = a.finS8 + item.s_begin;
        const uint32_t ns = item.s_len;
        if constexpr (MAT) {
            constexpr int U = 4;  // probe tuples per thread and round: loads in flight, fewer rounds
            for (uint32_t base = 0; base < ns; base += U * kCompactThreads) {
                tuple_v sv[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const uint32_t j = base + u * kCompactThreads + tid;
                    sv[u] = j < ns ? ld_stream(S + j) : make_ulonglong2(0, 0);
                }
                uint32_t mm[U], best[U], m = 0;
#pragma unroll
                for (int u = 0; u < U; u++) {
                    mm[u] = best[u] = 0;
                    if (base + u * kCompactThreads + tid >= ns) continue;
                    const uint64_t khi = sv[u].x >> B;
                    uint32_t e = head[khi & hmask], steps = 0;
                    while (e) {
                        if ((rw[e - 1] >> 32) == khi) {
                            if (!lp) mm[u]++;
                            else if (best[u] == 0 || e < best[u]) best[u] = e;
                        }
                        e = nxt[e - 1];
                        if (++steps > nr) {
                            set_error(err, kErrProbeLimit);
                            break;
                        }
                    }
                    if (lp) mm[u] = best[u] ? 1u : 0u;
                    m += mm[u];
                }
                unsigned long long o = mat_reserve(m, scan_tmp, &s_base, &a.acc->pairs);
                cnt += m;
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (!mm[u]) continue;
                    if (lp) {
                        mat_put(a.mat, o++, rw[best[u] - 1] & 0xffffffffull, sv[u].y, err);
                        continue;
                    }
                    const uint64_t khi = sv[u].x >> B;
                    uint32_t e = head[khi & hmask], steps = 0;
                    while (e && steps++ <= nr) {
                        const unsigned long long w = rw[e - 1];
                        if ((w >> 32) == khi) mat_put(a.mat, o++, w & 0xffffffffull, sv[u].y, err);
                        e = nxt[e - 1];
                    }
                }
            }
        } else
        // Eight probe tuples per thread in flight (four left the DRAM queue short: 2.01 -> 1.92 ms
        // for the headline join phase).
        for (uint32_t j0 = tid; j0 < ns; j0 += 8 * kCompactThreads) {
            tuple_v sv[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const uint32_t j = j0 + u * kCompactThreads;
                sv[u] = j < ns ? ld_fin(S, S8, j, ci) : make_ulonglong2(0, 0);
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const uint32_t j = j0 + u * kCompactThreads;
                if (j >= ns) continue;
                const uint64_t khi = sv[u].x >> B;
                uint32_t e = head[khi & hmask];
                uint32_t best = 0, steps = 0, nm = 0;
                while (e) {
                    const unsigned long long w = rw[e - 1];
                    if ((w >> 32) == khi) {
                        if (lp) {
                            if (best == 0 || e < best) best = e;
                            nm++;
                        } else {
                            cnt++;
                            sum += (w & 0xffffffffull) + sv[u].y;
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
                    sum += (rw[best - 1] & 0xffffffffull) + sv[u].y;
                    multi |= nm > 1;
                }
            }
        }
        __syncthreads();
    }
    block_sum2_to(cnt, sum, red, &a.acc->matched, &a.acc->checksum);
    if (LP && !MAT) flag_multi(multi, &a.acc->dup_flag);
}

template <bool MAT, bool CI = false>
__global__ void __launch_bounds__(kJoinThreads, 1) join_small_kernel(JoinArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    tuple_v *rt = reinterpret_cast<tuple_v *>(smem);                      // [kSmemCap]
    uint16_t *head = reinterpret_cast<uint16_t *>(rt + kSmemCap);         // [kHeadMax]
    uint16_t *nxt = head + kHeadMax;                                       // [kSmemCap]
    __shared__ __align__(8) unsigned long long bar_storage;
    __shared__ unsigned long long red[64];
    __shared__ uint32_t s_item;
    __shared__ uint32_t scan_tmp[32];
    __shared__ unsigned long long s_base;
    const int tid = threadIdx.x;
    const uint32_t bar = smem_u32(&bar_storage);
    unsigned int *err = &a.counters[kCtrErr];
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t nitems = a.counters[kCtrNItems];
    // Compiled once per partition layout; only the launch matching the device's choice runs.
    if (CI != (!MAT && a.ci && ci_applies(a.counters, a.bits))) return;
    constexpr bool ci = CI;
    const int B = ci ? 0 : a.bits;  // shift from a stored x to the key's bits above the radix bits
    const bool lp = a.lp != 0;
    const bool skip0 = a.skip0 != 0;
    // Items [0, nA) went to the compact kernel if the build side's keys and row ids fit it.
    const uint32_t first_item = compact_applies(a) ? a.counters[kCtrNItemsA] : 0u;
    unsigned long long cnt = 0, sum = 0;
    uint32_t phase = 0;
    bool ok = true, multi = false;
    for (;;) {
        if (tid == 0) s_item = first_item + atomicAdd(&a.counters[kCtrItem], 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= nitems) break;
        const JoinItem item = a.items[it];
        const uint32_t nr = item.r_len;
        const uint32_t nb = next_pow2_u32(nr);
        const uint64_t hmask = nb - 1;
        if (!ci && tid == 0) {
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
        if (ci) {
            // Compact final partitions: expand the build side's words into {key >> bits, row id}.
            for (uint32_t i = tid; i < nr; i += kJoinThreads)
                rt[i] = ld_fin(a.finR + item.r_begin, a.finR8 + item.r_begin, i, true);
        } else {
            if (!mbar_wait(bar, phase)) {
                set_error(err, kErrSpinLimit);
                ok = false;
            }
            // An expired wait: let the R-tile copy land (bounded) before the CTA leaves its shared memory.
            if (!ok && tid == 0) mbar_wait(bar, phase);
            phase ^= 1u;
        }
        if (__syncthreads_or(!ok)) break;
        // Build: chain every R tuple (lp_join skips key 0, which reads as an empty slot there).
        for (uint32_t i = tid; i < nr; i += kJoinThreads) {
            const uint64_t k = rt[i].x;
            if (skip0 && k == 0 && (!ci || item.part0)) continue;
            const uint32_t h = (uint32_t)((k >> B) & hmask);
            nxt[i] = (uint16_t)atomic_exch_u16(&head[h], i + 1);
        }
        __syncthreads();
        // Probe.
        const tuple_v *S = a.finS + item.s_begin;
        const uint32_t ns = item.s_len;
        if constexpr (MAT) {
            constexpr int U = 4;  // probe tuples per thread and round
            for (uint32_t base = 0; base < ns; base += U * kJoinThreads) {
                tuple_v sv[U];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const uint32_t j = base + u * kJoinThreads + tid;
                    sv[u] = j < ns ? ld_stream(S + j) : make_ulonglong2(0, 0);
                }
                uint32_t mm[U], best[U], m = 0;
#pragma unroll
                for (int u = 0; u < U; u++) {
                    mm[u] = best[u] = 0;
                    if (base + u * kJoinThreads + tid >= ns) continue;
                    const uint64_t k = sv[u].x;
                    uint32_t e = head[(k >> B) & hmask], steps = 0;
                    while (e) {
                        if (rt[e - 1].x == k) {
                            if (!lp) mm[u]++;
                            else if (best[u] == 0 || e < best[u]) best[u] = e;
                        }
                        e = nxt[e - 1];
                        if (++steps > nr) {
                            set_error(err, kErrProbeLimit);
                            break;
                        }
                    }
                    if (lp) mm[u] = best[u] ? 1u : 0u;
                    m += mm[u];
                }
                unsigned long long o = mat_reserve(m, scan_tmp, &s_base, &a.acc->pairs);
                cnt += m;
#pragma unroll
                for (int u = 0; u < U; u++) {
                    if (!mm[u]) continue;
                    if (lp) {
                        mat_put(a.mat, o++, rt[best[u] - 1].y, sv[u].y, err);
                        continue;
                    }
                    const uint64_t k = sv[u].x;
                    uint32_t e = head[(k >> B) & hmask], steps = 0;
                    while (e && steps++ <= nr) {
                        if (rt[e - 1].x == k) mat_put(a.mat, o++, rt[e - 1].y, sv[u].y, err);
                        e = nxt[e - 1];
                    }
                }
            }
        } else
        for (uint32_t j0 = tid; j0 < ns; j0 += 4 * kJoinThreads) {
            tuple_v s[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t j = j0 + u * kJoinThreads;
                s[u] = j < ns ? ld_fin(S, a.finS8 + item.s_begin, j, ci) : make_ulonglong2(0, 0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t j = j0 + u * kJoinThreads;
                if (j >= ns) continue;
                const uint64_t k = s[u].x;
                uint32_t e = head[(k >> B) & hmask];
                uint32_t best = 0, nm = 0;
                uint32_t steps = 0;
                while (e) {
                    const tuple_v r = rt[e - 1];
                    if (r.x == k) {
                        if (lp) {
                            if (best == 0 || e < best) best = e;
                            nm++;
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
                    multi |= nm > 1;
                }
            }
        }
        __syncthreads();
    }
    block_sum2_to(cnt, sum, red, &a.acc->matched, &a.acc->checksum);
    if (!MAT) flag_multi(multi, &a.acc->dup_flag);
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

// Key-aggregated table of one large partition (see large_words_agg): one chain node per distinct build
// key, holding the count of its build tuples, the wrapping sum of their row ids and the smallest
// position among them (as the maximum of ~position). A probe then costs one lookup however many build
// tuples share its key, where a chain of every build tuple costs a walk over all of them (a hot build
// key makes that quadratic).
struct LargeAgg {
    unsigned long long *sum;
    uint32_t *head, *next, *cnt, *negpos;
};

__device__ __forceinline__ LargeAgg large_agg(uint32_t *table, const LargePart &L) {
    LargeAgg t;
    uint32_t *base = table + L.table_off;
    t.sum = reinterpret_cast<unsigned long long *>(base);
    t.head = base + 2 * L.r_len;
    t.next = t.head + (1ull << L.nb_log);
    t.cnt = t.next + L.r_len;
    t.negpos = t.cnt + L.r_len;
    return t;
}

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t *p) {
    return *reinterpret_cast<const volatile uint32_t *>(p);
}

// The node (index + 1) of key k in bucket h, inserting build tuple i as its node when the key is absent.
// Lock-free: a node is published by a CAS on the bucket head after its next link is written; a failed
// CAS means another insert succeeded, and only the nodes it added (above the old head) are re-checked.
// Returns 0 (and sets the error word) if the walk exceeds the partition's size.
__device__ __forceinline__ uint32_t large_agg_find_or_insert(const LargeAgg &t, const JoinArgs &a, bool ci,
                                                             uint64_t r_begin, uint64_t r_len, uint64_t h,
                                                             uint64_t k, uint32_t i, uint32_t *err) {
    uint32_t stop = 0;
    uint32_t e = ld_volatile_u32(&t.head[h]);
    uint64_t steps = 0;
    for (;;) {
        for (uint32_t x = e; x && x != stop; x = ld_volatile_u32(&t.next[x - 1])) {
            if (fin_r(a, ci, r_begin + x - 1).x == k) return x;
            if (++steps > r_len) {
                set_error(err, kErrProbeLimit);
                return 0;
            }
        }
        *reinterpret_cast<volatile uint32_t *>(&t.next[i]) = e;
        __threadfence();
        const uint32_t old = atomicCAS(&t.head[h], e, i + 1);
        if (old == e) return i + 1;
        stop = e;
        e = old;
        if (++steps > r_len) {
            set_error(err, kErrProbeLimit);
            return 0;
        }
    }
}

__global__ void join_large_build(JoinArgs a) {
    const int nl = (int)a.counters[kCtrNLarge];
    const uint64_t total = ld_u64_pair(&a.counters[kCtrLargeR]);
    const bool ci = a.ci && ci_applies(a.counters, a.bits);
    const int bshift = ci ? 0 : a.bits;
    if (a.counters[kCtrLargeAgg]) {
        // Warp-uniform rounds: lanes holding equal keys of one partition combine their count, row-id sum
        // and smallest position first, so a hot key costs one update per warp.
        const unsigned lane = threadIdx.x & 31;
        for (uint64_t g0 = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); g0 < total;
             g0 += (uint64_t)gridDim.x * blockDim.x) {
            const uint64_t g = g0 + lane;
            bool act = g < total;
            int l = 0;
            uint64_t i = 0;
            tuple_v r = make_ulonglong2(0, 0);
            if (act) {
                l = find_large(a.large, nl, g, true);
                i = g - a.large[l].r_flat;
                r = fin_r(a, ci, a.large[l].r_begin + i);
                act = !(a.skip0 && r.x == 0 && (!ci || a.large[l].part0));
            }
            const unsigned act_mask = __ballot_sync(0xffffffffu, act);
            if (!act) continue;
            // Group lanes by key and partition: a compact word holds only key >> bits, which keys of two
            // partitions can share (full keys of different partitions differ in their low bits anyway).
            const unsigned long long gkey = ci ? (r.x | ((unsigned long long)(unsigned)l << 32)) : r.x;
            const unsigned peers = __match_any_sync(act_mask, gkey);
            // Row-id sum of the group in three pieces of at most 24 bits (32 addends cannot overflow them).
            const unsigned s0 = __reduce_add_sync(peers, (unsigned)(r.y & 0xffffffu));
            const unsigned s1 = __reduce_add_sync(peers, (unsigned)((r.y >> 24) & 0xffffffu));
            const unsigned s2 = __reduce_add_sync(peers, (unsigned)(r.y >> 48));
            const unsigned minpos = __reduce_min_sync(peers, (unsigned)i);
            if ((int)lane != __ffs(peers) - 1) continue;
            const LargePart &L = a.large[l];
            const LargeAgg t = large_agg(a.large_table, L);
            const uint64_t h = (r.x >> bshift) & ((1ull << L.nb_log) - 1);
            const uint32_t node = large_agg_find_or_insert(t, a, ci, L.r_begin, L.r_len, h, r.x, (uint32_t)i,
                                                           &a.counters[kCtrErr]);
            if (!node) continue;
            atomicAdd(&t.cnt[node - 1], (uint32_t)__popc(peers));
            atomicAdd(&t.sum[node - 1], (unsigned long long)s0 + ((unsigned long long)s1 << 24) +
                                            ((unsigned long long)s2 << 48));
            atomicMax(&t.negpos[node - 1], ~minpos);
        }
        return;
    }
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const int l = find_large(a.large, nl, g, true);
        const LargePart &L = a.large[l];
        const uint64_t i = g - L.r_flat;
        const uint64_t k = fin_r(a, ci, L.r_begin + i).x;
        if (a.skip0 && k == 0 && (!ci || L.part0)) continue;
        uint32_t *head = a.large_table + L.table_off;
        uint32_t *nxt = head + (1ull << L.nb_log);
        const uint64_t h = (k >> bshift) & ((1ull << L.nb_log) - 1);
        nxt[i] = atomicExch(&head[h], (uint32_t)(i + 1));
    }
}

template <bool MAT>
__global__ void join_large_probe(JoinArgs a) {
    __shared__ unsigned long long red[64];
    __shared__ uint32_t scan_tmp[32];
    __shared__ unsigned long long s_base;
    const int nl = (int)a.counters[kCtrNLarge];
    const uint64_t total = ld_u64_pair(&a.counters[kCtrLargeS]);
    unsigned long long cnt = 0, sum = 0;
    bool multi = false;  // first-match joins: a probe tuple matched two build tuples
    const bool ci = !MAT && a.ci && ci_applies(a.counters, a.bits);
    const int bshift = ci ? 0 : a.bits;
    if constexpr (MAT) {
        unsigned int *err = &a.counters[kCtrErr];
        // Block-uniform rounds over the flattened probe tuples of all large partitions.
        for (uint64_t g0 = blockIdx.x * (uint64_t)blockDim.x; g0 < total; g0 += (uint64_t)gridDim.x * blockDim.x) {
            const uint64_t g = g0 + threadIdx.x;
            uint32_t m = 0, best = 0, e0 = 0;
            tuple_v s = make_ulonglong2(0, 0);
            const LargePart *Lp = nullptr;
            if (g < total) {
                Lp = &a.large[find_large(a.large, nl, g, false)];
                s = ld_stream(a.finS + Lp->s_begin + (g - Lp->s_flat));
                const uint32_t *head = a.large_table + Lp->table_off;
                const uint32_t *nxt = head + (1ull << Lp->nb_log);
                const tuple_v *rr = a.finR + Lp->r_begin;
                e0 = head[(s.x >> a.bits) & ((1ull << Lp->nb_log) - 1)];
                uint64_t steps = 0;
                for (uint32_t e = e0; e;) {
                    if (rr[e - 1].x == s.x) {
                        if (!a.lp) m++;
                        else if (best == 0 || e < best) best = e;
                    }
                    e = nxt[e - 1];
                    if (++steps > Lp->r_len) {
                        set_error(err, kErrProbeLimit);
                        break;
                    }
                }
                if (a.lp) m = best ? 1u : 0u;
            }
            unsigned long long o = mat_reserve(m, scan_tmp, &s_base, &a.acc->pairs);
            cnt += m;
            if (m) {
                const uint32_t *nxt = a.large_table + Lp->table_off + (1ull << Lp->nb_log);
                const tuple_v *rr = a.finR + Lp->r_begin;
                if (a.lp) {
                    mat_put(a.mat, o, rr[best - 1].y, s.y, err);
                } else {
                    uint64_t steps = 0;
                    for (uint32_t e = e0; e && steps++ <= Lp->r_len; e = nxt[e - 1])
                        if (rr[e - 1].x == s.x) mat_put(a.mat, o++, rr[e - 1].y, s.y, err);
                }
            }
        }
    } else if (a.counters[kCtrLargeAgg]) {
        for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
             g += (uint64_t)gridDim.x * blockDim.x) {
            const int l = find_large(a.large, nl, g, false);
            const LargePart &L = a.large[l];
            const tuple_v s = ld_fin(a.finS, a.finS8, L.s_begin + (g - L.s_flat), ci);
            const LargeAgg t = large_agg(a.large_table, L);
            uint32_t e = t.head[(s.x >> bshift) & ((1ull << L.nb_log) - 1)];
            uint64_t steps = 0;
            while (e && fin_r(a, ci, L.r_begin + e - 1).x != s.x) {
                e = t.next[e - 1];
                if (++steps > L.r_len) {
                    set_error(&a.counters[kCtrErr], kErrProbeLimit);
                    e = 0;
                }
            }
            if (!e) continue;
            if (a.lp) {
                const uint32_t first = ~t.negpos[e - 1];
                multi |= t.cnt[e - 1] > 1;
                if (first < L.r_len) {
                    cnt++;
                    sum += fin_r(a, ci, L.r_begin + first).y + s.y;
                } else {
                    set_error(&a.counters[kCtrErr], kErrBounds);
                }
            } else {
                const unsigned long long c = t.cnt[e - 1];
                cnt += c;
                sum += t.sum[e - 1] + c * s.y;
            }
        }
    } else
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const int l = find_large(a.large, nl, g, false);
        const LargePart &L = a.large[l];
        const tuple_v s = ld_fin(a.finS, a.finS8, L.s_begin + (g - L.s_flat), ci);
        const uint32_t *head = a.large_table + L.table_off;
        const uint32_t *nxt = head + (1ull << L.nb_log);
        uint32_t e = head[(s.x >> bshift) & ((1ull << L.nb_log) - 1)];
        uint32_t best = 0, nm = 0;
        uint64_t steps = 0;
        while (e) {
            const tuple_v r = fin_r(a, ci, L.r_begin + e - 1);
            if (r.x == s.x) {
                if (a.lp) {
                    if (best == 0 || e < best) best = e;
                    nm++;
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
            sum += fin_r(a, ci, L.r_begin + best - 1).y + s.y;
            multi |= nm > 1;
        }
    }
    block_sum2_to(cnt, sum, red, &a.acc->matched, &a.acc->checksum);
    if (!MAT) flag_multi(multi, &a.acc->dup_flag);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (nl) atomicAdd(&a.acc->large_parts, (unsigned long long)nl);
        if (ci) atomicOr(&a.acc->flags, (unsigned long long)HJ_RES_COMPACT_PARTITIONS);
        if (a.w8_b1 >= 0 && w8_fits(a.counters, a.w8_b1))
            atomicOr(&a.acc->flags, (unsigned long long)HJ_RES_WORD_PASS1);
    }
}

__global__ void copy_error(const uint32_t *counters, JoinAccum *acc) {
    if (threadIdx.x == 0 && counters[kCtrErr]) atomicOr(&acc->error, counters[kCtrErr]);
}

// ------------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------------
int radix_geom(int bits, int passes, RadixGeom *g, int b1_req) {
    if (bits < 1 || bits > 15) return HJ_E_INVAL;
    if (passes != 1 && passes != 2) return HJ_E_INVAL;
    // Partition contents do not depend on how the bits are split across passes; a single pass runs
    // as one physical pass only while its fanout fits the shared-memory staging (<= 256 digits).
    int P = passes;
    if (P == 1 && bits > 8) P = 2;
    if (P == 2 && bits < 2) P = 1;
    g->bits = bits;
    g->passes = P;
    int b1 = bits / 2;
    if (b1_req > 0) {
        b1 = b1_req;
        if (b1 > 8) b1 = 8;
        if (b1 > bits - 1) b1 = bits - 1;
        if (b1 < bits - 8) b1 = bits - 8;
        if (b1 < 1) b1 = 1;
    }
    g->b1 = P == 2 ? b1 : bits;
    g->b2 = bits - g->b1;
    if (g->b1 > 8 || g->b2 > 8) return HJ_E_INVAL;
    g->F1 = 1 << g->b1;
    g->F2 = 1 << g->b2;
    return HJ_OK;
}

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Pass-1 work items: about kSubPerChunk sub-chunks per chunk (two per warp of the histogram kernel).
constexpr int kSubPerChunk = 32;

static ChunkGeom chunk_geom(size_t nR, size_t nS, int num_sms) {
    // About three chunks per SM (the scatter kernel's residency), each a whole number of tiles.
    const uint64_t tiles = (uint64_t)ceil_div_u64(nR, kTile) + ceil_div_u64(nS, kTile);
    const uint64_t target = (uint64_t)(num_sms > 0 ? num_sms : 148) * 3;
    uint64_t ct = (tiles + target - 1) / target;
    if (ct < 1) ct = 1;
    // Pass 1 takes sub-chunks as work items, so that CTAs that run ahead take more of them instead of
    // idling while the slowest chunk finishes.
    const uint64_t st = (ct + kSubPerChunk - 1) / kSubPerChunk;
    ChunkGeom cg;
    cg.chunk = ct * kTile;
    cg.cR = ceil_div_u64(nR, cg.chunk);
    cg.cS = ceil_div_u64(nS, cg.chunk);
    cg.sub = st * kTile;
    cg.spc = (uint32_t)((ct + st - 1) / st);
    cg.pad = 0;
    return cg;
}

struct PhjSizes {
    size_t chunk_hist, prefix, total, start, units_off, units_cnt, subhist, counters, items, large, large_table,
        tmp1, tmp2, seg_head, seg_next;
    size_t max_items, max_large, large_table_words;
    uint32_t max_segs, seg_grid, it_tiles;
    ChunkGeom cg;
};

// Segment mode from 2^27 tuples. Its pass 2 has one unit per (pass-1 CTA, relation, digit) and a
// partial tile per unit whatever the size, and its pass 1 runs at two CTAs per SM. At 2^24 x 2^26
// (2^26.3 tuples) the joins of both pipelines took the same time; the saved histogram read grows with
// the size (1.3 ms of 11.8 at 2^27 x 2^29). The partly filled segments also reserve storage
// (2 * CTAs * F1 * kTile tuples).
constexpr uint64_t kSegMinTuples = 1ull << 27;

bool phj_seg_applies(const RadixGeom &g, bool, size_t nR, size_t nS) {
    return g.passes == 2 && g.bits <= kSegMaxBits && (uint64_t)nR + nS >= kSegMinTuples;
}

static PhjSizes phj_sizes(const RadixGeom &g, size_t nR, size_t nS, int num_sms, bool seg) {
    PhjSizes z;
    const size_t np = (size_t)g.nparts();
    const int sms = num_sms > 0 ? num_sms : 148;
    if (seg) {
        // "Chunks" are the pass-1 CTAs, one per relation each.
        z.seg_grid = (uint32_t)(sms * kSegCtasPerSm);
        z.cg.chunk = 0;
        z.cg.cR = z.cg.cS = z.seg_grid;
        z.cg.sub = 0;
        z.cg.spc = 0;
        z.cg.pad = 0;
        const uint64_t tiles = (uint64_t)ceil_div_u64(nR, kTile) + ceil_div_u64(nS, kTile);
        uint64_t it = tiles / ((uint64_t)z.seg_grid * 8);
        z.it_tiles = (uint32_t)(it < 1 ? 1 : it > 16 ? 16 : it);
        // Every segment but the current one of each (CTA, relation, digit) is full; each CTA leaves
        // fewer than kSegSlab ids of its last slab unused.
        const uint64_t segs = (uint64_t)(nR + nS) / kTile + 2ull * z.seg_grid * g.F1 + (uint64_t)z.seg_grid * kSegSlab;
        z.max_segs = (uint32_t)segs;
    } else {
        z.cg = chunk_geom(nR, nS, num_sms);
        z.seg_grid = 0;
        z.it_tiles = 0;
        z.max_segs = 0;
    }
    const size_t nchunks = (size_t)z.cg.cR + z.cg.cS;
    z.chunk_hist = align_up(nchunks * np * 4, 256);
    z.prefix = z.chunk_hist;
    z.total = align_up(2 * np * 4, 256);
    z.start = align_up(2 * (np + 1) * 8, 256);
    z.units_off = align_up(nchunks * (size_t)g.F1 * 8, 256);
    z.units_cnt = align_up(nchunks * (size_t)g.F1 * 4, 256);
    z.subhist = align_up(nchunks * (size_t)z.cg.spc * g.F1 * 4, 256);
    z.counters = 256;
    z.max_items = np + nS / kProbeChunk + 2;
    z.items = align_up(z.max_items * sizeof(JoinItem), 256);
    z.max_large = np < nR / kSmemCap + 1 ? np : nR / kSmemCap + 1;
    z.large = align_up(z.max_large * sizeof(LargePart), 256);
    z.tmp1 = seg ? align_up((size_t)z.max_segs * kTile * 16, 256) : align_up((nR + nS) * 16, 256);
    z.tmp2 = g.passes == 2 ? align_up((nR + nS) * 16, 256) : 0;
    z.seg_head = seg ? align_up((size_t)2 * z.seg_grid * g.F1 * 4, 256) : 0;
    z.seg_next = seg ? align_up((size_t)z.max_segs * 4, 256) : 0;
    // Large-partition tables: chains take head <= 2*|R_p| words and next = |R_p| words; key-aggregated
    // tables another 4*|R_p| words plus one word of alignment each. With two passes they reuse the
    // pass-1 buffer, which is dead once pass 2 has run (tables that do not fit it fall back to chains).
    z.large_table_words = 7 * nR + 2 * z.max_large + 2;
    z.large_table = g.passes == 2 ? 0 : align_up(z.large_table_words * 4, 256);
    return z;
}

size_t phj_scratch_bytes(const RadixGeom &g, size_t nR, size_t nS, int num_sms, bool seg) {
    PhjSizes z = phj_sizes(g, nR, nS, num_sms, seg);
    return z.chunk_hist + z.prefix + z.total + z.start + z.units_off + z.units_cnt + z.subhist + z.counters + z.items +
           z.large + z.large_table + z.tmp1 + z.tmp2 + z.seg_head + z.seg_next;
}

void phj_carve(const RadixGeom &g, size_t nR, size_t nS, int num_sms, char *base, PhjScratch *s, bool seg) {
    PhjSizes z = phj_sizes(g, nR, nS, num_sms, seg);
    char *p = base;
    s->seg = seg;
    s->seg_grid = z.seg_grid;
    s->max_segs = z.max_segs;
    s->it_tiles = z.it_tiles;
    s->chunk = z.cg.chunk;
    s->cR = z.cg.cR;
    s->cS = z.cg.cS;
    s->sub = z.cg.sub;
    s->spc = z.cg.spc;
    s->chunk_hist = reinterpret_cast<uint32_t *>(p); p += z.chunk_hist;
    s->prefix = reinterpret_cast<uint32_t *>(p); p += z.prefix;
    s->total = reinterpret_cast<uint32_t *>(p); p += z.total;
    s->start = reinterpret_cast<uint64_t *>(p); p += z.start;
    s->unit_off = reinterpret_cast<uint64_t *>(p); p += z.units_off;
    s->unit_cnt = reinterpret_cast<uint32_t *>(p); p += z.units_cnt;
    s->subhist = reinterpret_cast<uint32_t *>(p); p += z.subhist;
    s->seg_head = reinterpret_cast<uint32_t *>(p); p += z.seg_head;
    s->seg_next = reinterpret_cast<uint32_t *>(p); p += z.seg_next;
    s->counters = reinterpret_cast<uint32_t *>(p); p += z.counters;
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

#define HJ_CU(call)                                                                   \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            fprintf(stderr, "hjscm: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return HJ_E_DEVICE;                                                       \
        }                                                                             \
    } while (0)

static bool g_attr_done[64] = {};

// Dynamic shared memory of seg_pass1_kernel: two tile buffers, per-digit state, 2^bits 16-bit counters,
// and for the stable build-relation rank one 16-bit counter per (warp, digit).
static size_t seg_smem_bytes(int bits, bool stable) {
    // tile buffers, runs[256], thist[256], tdstart[256], counter pairs, whist
    return (size_t)2 * kTile * 16 + 256 * sizeof(SegRun) + 256 * 4 * 2 + ((size_t)1 << bits) * 2 +
           (stable ? (size_t)(kScatterThreads / 32) * 256 * 2 : 0);
}

int phj_prepare_device() {
    int cur_dev = 0;
    HJ_CU(cudaGetDevice(&cur_dev));
    if (cur_dev < 0 || cur_dev >= 64) return HJ_E_INVAL;
    if (g_attr_done[cur_dev]) return HJ_OK;
    const size_t scatter_smem = (size_t)kScatterBufs * (kTile * 16 + 16) + 256 * 8 * 2 + 256 * 4 + (kScatterThreads / 32) * 256 * 2;
    HJ_CU(cudaFuncSetAttribute(hist_chunk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 136 * 1024));
    HJ_CU(cudaFuncSetAttribute(plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)((size_t)2 * (1u << kPlanStageBits) * 4)));
    HJ_CU(cudaFuncSetAttribute(scatter_kernel<kScatterThreads, kScatterItems, true, kScatterBufs, kScatterCtasPerSm>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scatter_smem));
    HJ_CU(cudaFuncSetAttribute(scatter_kernel<kScatterThreads, kScatterItems, false, kScatterBufs, kScatterCtasPerSm>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scatter_smem));
#define HJ_SEG_ATTR(KK, W, ST)                                                                             \
    HJ_CU(cudaFuncSetAttribute(seg_pass1_kernel<kScatterThreads, kScatterItems, KK, W, ST>,                  \
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)seg_smem_bytes(kSegMaxBits, ST)))
#define HJ_SEG_ATTR4(W, ST) \
    HJ_SEG_ATTR(1, W, ST);  \
    HJ_SEG_ATTR(2, W, ST);  \
    HJ_SEG_ATTR(4, W, ST);  \
    HJ_SEG_ATTR(8, W, ST)
    HJ_SEG_ATTR4(false, false);
    HJ_SEG_ATTR4(true, false);
    HJ_SEG_ATTR4(false, true);
    HJ_SEG_ATTR4(true, true);
#undef HJ_SEG_ATTR4
#undef HJ_SEG_ATTR
    HJ_CU(cudaFuncSetAttribute(
        scatter_kernel<kScatterThreads, 2 * kScatterItems, false, kScatterBufs, kScatterWordCtasPerSm, true>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scatter_smem));
    HJ_CU(cudaFuncSetAttribute(
        scatter_kernel<kScatterThreads, 2 * kScatterItems, true, kScatterBufs, kScatterWordCtasPerSm, true>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scatter_smem));
    HJ_CU(cudaFuncSetAttribute(join_small_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJoinSmem));
    HJ_CU(cudaFuncSetAttribute(join_small_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kJoinSmem));
    HJ_CU(cudaFuncSetAttribute(join_compact_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kCompactSmem));
    HJ_CU(cudaFuncSetAttribute(join_compact_kernel<false, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kCompactSmem));
    HJ_CU(cudaFuncSetAttribute(join_compact_kernel<false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kCompactSmem));
    HJ_CU(cudaFuncSetAttribute(join_compact_kernel<true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kCompactSmem));
    HJ_CU(cudaFuncSetAttribute(join_small_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJoinSmem));
    HJ_CU(cudaFuncSetAttribute(join_compact_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kCompactSmem));
    HJ_CU(cudaFuncSetAttribute(join_compact_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kCompactSmem));
    g_attr_done[cur_dev] = true;
    return nphj_prepare_device();
}

int phj_enqueue(const RadixGeom &g, bool lp, bool skip0, const ulonglong2 *R, size_t nR, const ulonglong2 *S,
                size_t nS, const PhjScratch &s, JoinAccum *acc, cudaStream_t st, cudaEvent_t ev_mid,
                int num_sms, cudaEvent_t *ph, uint32_t *launches, const MatOut *mat, int test_flags,
                bool ordered) {
    uint32_t nlaunch = 0;
    // Stable ranks of the build relation: first-match joins that keep the input order.
    const bool stable = lp && ordered;
#define HJ_PH(i) \
    if (ph) HJ_CU(record_event(ph[i], st))
    if (nR >= (1ull << 32) || nS >= (1ull << 32)) return HJ_E_INVAL;
    const int np = g.nparts();
    const int F1 = g.F1, F2 = g.F2;
    constexpr int T = kTile;
    // tile buffers (word tiles: 16 spare bytes each), gbase, running, tdstart, per-warp digit counts
    const size_t scatter_smem = (size_t)kScatterBufs * (T * 16 + 16) + 256 * 8 * 2 + 256 * 4 + (kScatterThreads / 32) * 256 * 2;
    const size_t hist_smem = (size_t)np * 4 + (size_t)16 * F1 * 4;  // 16 warps
    ChunkGeom cg;
    cg.chunk = s.chunk;
    cg.cR = s.cR;
    cg.cS = s.cS;
    cg.sub = s.sub;
    cg.spc = s.spc;
    cg.pad = 0;
    const uint32_t nchunks = cg.cR + cg.cS;
    // A segment-mode scratch holds the segment storage, not the exact-offset pipeline's buffers.
    const bool segm = s.seg;
    // 8-byte words in the partitions (compact final partitions, and in segment mode an 8-byte pass 1):
    // joins without per-match output (all but the materialising ones), unless the caller asked for
    // tuples (test_flags bit 2), when the widths allow them (decided on the device).
    const int ci_ok = (!mat && !(test_flags & 2)) ? 1 : 0;
    const bool seg_words = segm && ci_ok;
    // The exact-offset pipeline with two passes stores pass 1 as words too (when w8_fits holds, which
    // the histogram pass's ORs decide before pass 1) when its pass-2 units (chunk, pass-1 digit) average
    // a full 4096-word tile, or when asked (test_flags bit 4). Pass 2 over 4096-word tiles is slower than
    // over 2048-tuple tiles when most tiles are partial (2^24 x 2^26: 1.91 against 1.82 ms; 2^27 x 2^29:
    // 9.01 against 10.68 ms).
    const bool exact_words =
        !segm && ci_ok && g.passes == 2 && ((test_flags & 4) || cg.chunk / (uint64_t)F1 >= 2ull * kTile);
    if (segm && (g.passes != 2 || g.bits > kSegMaxBits)) return HJ_E_INVAL;
    {
        const int rc = phj_prepare_device();
        if (rc) return rc;
    }
    HJ_CU(cudaMemsetAsync(s.counters, 0, kNumCounters * 4, st));

    HJ_PH(0);
    if (segm) {
        // 1'. pass 1 into segment chains, with the per-CTA histograms
        SegArgs ga;
        ga.R = R;
        ga.S = S;
        ga.nR = nR;
        ga.nS = nS;
        ga.bits = g.bits;
        ga.F1 = F1;
        ga.it_tiles = s.it_tiles;
        ga.tilesR = ceil_div_u64(nR, T);
        ga.tilesS = ceil_div_u64(nS, T);
        ga.itemsR = (ga.tilesR + s.it_tiles - 1) / s.it_tiles;
        ga.items = ga.itemsR + (ga.tilesS + s.it_tiles - 1) / s.it_tiles;
        ga.out = s.tmp1;
        ga.max_segs = s.max_segs;
        ga.seg_head = s.seg_head;
        ga.seg_next = s.seg_next;
        ga.hist = s.chunk_hist;
        ga.counters = s.counters;
        ga.test_stall = (test_flags & 1) ? 1 : 0;
        ga.b1 = g.b1;
        ga.w8_first = 0;
        // Ordered first-match joins keep every build partition in input order (the stable build-relation form).
        const size_t sm = seg_smem_bytes(g.bits, stable);
        auto launch_pass1 = [&](bool words) {
#define HJ_SEG_LAUNCH_W(KK, W)                                                                                   \
    if (stable)                                                                                                  \
        seg_pass1_kernel<kScatterThreads, kScatterItems, KK, W, true><<<s.seg_grid, kScatterThreads, sm, st>>>(ga); \
    else                                                                                                         \
        seg_pass1_kernel<kScatterThreads, kScatterItems, KK, W, false><<<s.seg_grid, kScatterThreads, sm, st>>>(ga)
#define HJ_SEG_LAUNCH(KK)         \
    if (words) {                  \
        HJ_SEG_LAUNCH_W(KK, true);  \
    } else {                      \
        HJ_SEG_LAUNCH_W(KK, false); \
    }
            if (F1 <= 32) {
                HJ_SEG_LAUNCH(1);
            } else if (F1 <= 64) {
                HJ_SEG_LAUNCH(2);
            } else if (F1 <= 128) {
                HJ_SEG_LAUNCH(4);
            } else {
                HJ_SEG_LAUNCH(8);
            }
#undef HJ_SEG_LAUNCH
#undef HJ_SEG_LAUNCH_W
        };
        if (seg_words) {
            // Pass 1 in 8-byte words; if the widths turn out not to allow them, the counters are reset and
            // pass 1 runs again with tuples (that launch returns at once otherwise).
            launch_pass1(true);
            seg_reset_if_wide<<<1, 32, 0, st>>>(s.counters, g.b1);
            ga.w8_first = 1;
            ga.test_stall = 0;
            nlaunch += 2;
        }
        launch_pass1(false);
        HJ_CU(cudaGetLastError());
        nlaunch++;
    } else {
        // 1. per-chunk histograms
        hist_chunk_kernel<<<nchunks, 512, hist_smem, st>>>(R, nR, S, nS, g.bits, F1, cg, s.chunk_hist, s.subhist,
                                                           s.counters + kCtrMaxKey);
        HJ_CU(cudaGetLastError());
    }
    HJ_PH(1);
    // 2. prefix over chunks, 3. plan, 4. units
    colscan_kernel<<<(8 * np + 255) / 256, 256, 0, st>>>(s.chunk_hist, s.prefix, s.total, np, cg);
    PlanArgs pa;
    pa.bits = g.bits;
    pa.passes = g.passes;
    pa.b1 = g.b1;
    pa.F1 = F1;
    pa.F2 = F2;
    pa.nR = nR;
    pa.nS = nS;
    pa.total = s.total;
    pa.start = s.start;
    pa.counters = s.counters;
    pa.items = reinterpret_cast<JoinItem *>(s.items);
    pa.max_items = s.max_items;
    pa.large = reinterpret_cast<LargePart *>(s.large);
    pa.max_large = s.max_large;
    pa.large_table_words = s.large_table_words;
    pa.agg_ok = mat ? 0 : 1;
    plan_kernel<<<1, 1024, g.bits <= kPlanStageBits ? (size_t)2 * np * 4 : 0, st>>>(pa);
    {
        const int ut = F1 < 32 ? 32 : F1;
        units_kernel<<<nchunks, ut, 0, st>>>(s.chunk_hist, s.prefix, s.start, g.bits, g.b1, F1, g.passes == 2 ? F2 : 1,
                                             cg, s.unit_off, s.unit_cnt, s.subhist, s.counters + kCtrErr);
    }
    HJ_CU(cudaGetLastError());
    nlaunch += segm ? 3 : 4;
    HJ_PH(2);

    // 5. scatter passes (segment mode: pass 2 only, its units are the pass-1 chains)
    const int scatter_grid = num_sms * kScatterCtasPerSm;
    for (int pass = segm ? 1 : 0; pass < g.passes; pass++) {
        ScatterArgs sa;
        sa.pass = pass;
        sa.F = pass == 0 ? F1 : F2;
        sa.logF = pass == 0 ? g.b1 : g.b2;
        sa.shift = pass == 0 ? 0 : g.b1;
        sa.bits = g.bits;
        sa.b1 = g.b1;
        sa.F1 = F1;
        sa.F2 = g.passes == 2 ? F2 : 1;
        sa.cg = cg;
        sa.inR = pass == 0 ? R : s.tmp1;
        sa.inS = pass == 0 ? S : s.tmp1 + nR;
        tuple_v *out = pass == 0 ? s.tmp1 : s.tmp2;
        sa.outR = out;
        sa.outS = out + nR;
        sa.nR = nR;
        sa.nS = nS;
        sa.prefix = s.prefix;
        sa.start = s.start;
        sa.unit_off = s.unit_off;
        sa.unit_cnt = s.unit_cnt;
        sa.subpre = s.subhist;
        sa.seg_head = segm ? s.seg_head : nullptr;
        sa.seg_next = segm ? s.seg_next : nullptr;
        sa.max_segs = segm ? s.max_segs : 0;
        sa.test_stall = (pass == 0 && (test_flags & 1)) ? 1 : 0;
        sa.counters = s.counters;
        sa.ctr_item = pass == 0 ? kCtrItem1 : kCtrItem2;
        sa.item_base = sa.item_end = 0;
        sa.ci_out = (pass == g.passes - 1) ? ci_ok : 0;
        sa.ci_z0 = skip0 ? 1 : 0;
        sa.outR8 = reinterpret_cast<unsigned long long *>(out);
        sa.outS8 = sa.outR8 + nR;
        sa.w8 = 0;
        sa.w8_out = (exact_words && pass == 0) ? 1 : 0;
        sa.inR8 = reinterpret_cast<const unsigned long long *>(s.tmp1);
        sa.inS8 = sa.inR8 + nR;
        const bool words_in = (segm && seg_words) || (exact_words && pass == 1);
        // One pass over [item_base, item_end): after a pass 1 that may have stored words, the launch over
        // 4096-word tiles and the tuple launch after it (which runs only if pass 1 stored tuples).
        auto launch_scatter = [&](bool stable) {
#define HJ_SCATTER(ST)                                                                                         \
    if (words_in) {                                                                                            \
        sa.w8 = 1;                                                                                             \
        scatter_kernel<kScatterThreads, 2 * kScatterItems, ST, kScatterBufs, kScatterWordCtasPerSm, true>        \
            <<<num_sms * kScatterWordCtasPerSm, kScatterThreads, scatter_smem, st>>>(sa);                      \
        nlaunch++;                                                                                             \
        sa.w8 = 2;                                                                                             \
    }                                                                                                          \
    scatter_kernel<kScatterThreads, kScatterItems, ST, kScatterBufs, kScatterCtasPerSm>                          \
        <<<scatter_grid, kScatterThreads, scatter_smem, st>>>(sa)
            if (stable) {
                HJ_SCATTER(true);
            } else {
                HJ_SCATTER(false);
            }
#undef HJ_SCATTER
        };
        if (stable) {
            // Ordered first-match joins need each final build partition in input order (the join keeps
            // the lowest position among equal keys), so the build relation's items take the stable rank.
            // The probe relation's order inside a partition changes nothing (each probe tuple finds its
            // first match on its own), so its items take the cheaper atomic rank, in a second launch.
            const uint32_t per_chunk = pass == 0 ? cg.spc : (uint32_t)F1;
            const uint32_t r_items = cg.cR * per_chunk, all_items = (cg.cR + cg.cS) * per_chunk;
            sa.item_end = r_items;
            if (r_items) {
                launch_scatter(true);
                nlaunch++;
            }
            sa.item_base = r_items;
            sa.item_end = all_items;
            sa.ctr_item = pass == 0 ? kCtrItem1S : kCtrItem2S;
            sa.test_stall = 0;
            sa.w8 = 0;
            if (all_items > r_items) launch_scatter(false);
        } else {
            launch_scatter(false);
        }
        HJ_CU(cudaGetLastError());
        nlaunch++;
        HJ_PH(segm ? 3 : 3 + pass);
    }
    if (ph && g.passes == 1) HJ_CU(record_event(ph[4], st));
    if (ev_mid) HJ_CU(record_event(ev_mid, st));

    // 6. joins
    JoinArgs ja;
    ja.items = reinterpret_cast<const JoinItem *>(s.items);
    ja.large = reinterpret_cast<const LargePart *>(s.large);
    ja.counters = s.counters;
    ja.finR = s.tmp2;
    ja.finS = s.tmp2 + nR;
    ja.large_table = s.large_table;
    ja.bits = g.bits;
    ja.lp = lp ? 1 : 0;
    ja.skip0 = skip0 ? 1 : 0;
    ja.acc = acc;
    ja.mat = mat ? *mat : MatOut{nullptr, 0};
    ja.ci = ci_ok;
    ja.finR8 = reinterpret_cast<const unsigned long long *>(s.tmp2);
    ja.finS8 = ja.finR8 + nR;
    ja.w8_b1 = (seg_words || exact_words) ? g.b1 : -1;
    if (mat) {
        if (lp)
            join_compact_kernel<true, false, true><<<num_sms * 2, kCompactThreads, kCompactSmem, st>>>(ja);
        else
            join_compact_kernel<true><<<num_sms * 2, kCompactThreads, kCompactSmem, st>>>(ja);
        join_small_kernel<true><<<num_sms, kJoinThreads, kJoinSmem, st>>>(ja);
    } else {
        // One launch per partition layout (tuples, compact words); the one that does not match the
        // device's choice returns at once.
        if (lp)
            join_compact_kernel<false, false, true><<<num_sms * 2, kCompactThreads, kCompactSmem, st>>>(ja);
        else
            join_compact_kernel<false, false><<<num_sms * 2, kCompactThreads, kCompactSmem, st>>>(ja);
        join_small_kernel<false, false><<<num_sms, kJoinThreads, kJoinSmem, st>>>(ja);
        if (ci_ok) {
            if (lp)
                join_compact_kernel<false, true, true><<<num_sms * 2, kCompactThreads, kCompactSmem, st>>>(ja);
            else
                join_compact_kernel<false, true><<<num_sms * 2, kCompactThreads, kCompactSmem, st>>>(ja);
            join_small_kernel<false, true><<<num_sms, kJoinThreads, kJoinSmem, st>>>(ja);
            nlaunch += 2;
        }
    }
    HJ_CU(cudaGetLastError());
    HJ_PH(segm ? 4 : 5);
    join_large_clear<<<num_sms * 2, 256, 0, st>>>(ja);
    join_large_build<<<num_sms * 2, 256, 0, st>>>(ja);
    if (mat)
        join_large_probe<true><<<num_sms * 2, 256, 0, st>>>(ja);
    else
        join_large_probe<false><<<num_sms * 2, 256, 0, st>>>(ja);
    copy_error<<<1, 32, 0, st>>>(s.counters, acc);
    HJ_CU(cudaGetLastError());
    HJ_PH(segm ? 5 : 6);
    nlaunch += 6;
    if (launches) *launches = nlaunch;
#undef HJ_PH
    return HJ_OK;
}

}  // namespace hj
