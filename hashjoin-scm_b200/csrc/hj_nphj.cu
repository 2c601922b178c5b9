// hj_nphj.cu - non-partitioned joins (nphj_sc / nphj_lp) on one global open-addressing table.
//
// Reference (src/algo/nphj.c):
//   nphj_sc  build_hashtable_nphj_sc (nphj.c:132-301): |R|/2 buckets of two tuples plus overflow
//            buckets, a spinlock per bucket; probe_hashtable_nphj_sc (nphj.c:304-442) walks the whole
//            chain and counts every equal key.
//   nphj_lp  lp_insert_with_pos (nphj.c:1056-1070): CAS on hashkey (stored as h+1) claims a slot;
//            lp_lookup_with_pos (nphj.c:1146-1167) stops at the first equal key. With duplicate R keys
//            the winner is a thread race; the contract here is the single-thread outcome, the first R
//            tuple in input order.
//
// B200 design: one table of 16-byte slots {key, val} with capacity ~|R|/load, hashed by a
// multiply-xorshift and linear probing. A slot is claimed by a 64-bit CAS of its key from EMPTY
// (all ones). The build notices any key inserted twice (the later inserter always walks over the
// earlier one's slot, because slots never empty). Without duplicates both algorithms stop at the
// first match; with duplicates sc keeps walking to the empty slot and lp rebuilds the table with the
// minimum input position per key (atomicMin) and resolves row ids in one gather pass. R tuples whose
// key equals the EMPTY pattern are kept in a side record instead of the table.
//
// Compact slots (nphj_sc): when every build key is below 2^32 - 1 and every build row id below 2^32
// (a first pass over R finds out), a slot is one 8-byte word (key << 32 | row id). The table then takes
// half the bytes (64 MB for |R| = 2^22, where L2 holds it) and a probe reads 8 bytes. Used when the
// 16-byte table would exceed 64 MB.
//
// Sliced build of a compact table: the table is cut into slices of kSliceSlots slots and a key's
// probe sequence wraps around inside its slice. The first pass over R also counts the build tuples of
// every slice per block of R; a column scan turns the counts into each block's output offsets; the
// build tuples are scattered by slice into a staging array as compact words; then one CTA per slice
// builds that slice's table in shared memory (shared-memory CAS) and writes it out whole. The build then
// makes no global atomics: claiming random global slots one CAS at a time is bound by the L2 atomic
// rate (about 20 G claims per second here), well below the bandwidth of the passes that replace it. If
// any slice would be filled above 7/8, the table is built by global CAS instead (the probe follows the
// mode the build used).
#include <cstdio>
#include <mutex>

#include "hj_common.cuh"
#include "hj_internal.h"
#include "hj_nphj.cuh"

namespace hj {

constexpr unsigned long long kEmpty = kTableEmpty;

struct NphjSide {
    unsigned long long cnt;      // R tuples with key == kEmpty
    unsigned long long sum;      // sum of their row ids
    unsigned long long minpos;   // smallest input position among them
    unsigned int dup;            // the build saw an equal key twice
    unsigned int err;
    unsigned long long kmax;     // largest build key (compact-slot test)
    unsigned long long ror;      // OR of all build row ids
    unsigned int sliced;         // the compact table is built (and probed) slice by slice
    unsigned int overflow;       // a slice's staged tuples exceeded kSliceMaxFill (no sliced build)
};

constexpr unsigned long long kCompactEmpty = ~0ull;
constexpr unsigned long long kCompactMinTableBytes = 64ull << 20;
// Compact tables up to this size are probed four keys per thread (more misses in flight); larger
// ones one key per thread. Measured on B200: four per thread is 15-20% faster on 64 MB and 256 MB
// tables, one per thread 11% faster on a 512 MB table and 17% on a 1 GB one.
constexpr unsigned long long kCompactDeepProbeBytes = 384ull << 20;

constexpr int kSliceLog = 13;
constexpr unsigned kSliceSlots = 1u << kSliceLog;        // 64 KB of compact slots per slice
constexpr unsigned kSliceMaxFill = kSliceSlots / 8 * 7;  // fuller slices: global-CAS build instead
constexpr unsigned kSliceMaxCount = 40960;              // slices the per-block histograms hold in shared memory
constexpr int kSliceThreads = 512;

// Every build key below 2^32 - 1 (so no slot can equal the empty pattern) and every row id below 2^32.
__device__ __forceinline__ bool nphj_compact(const NphjSide *side) {
    return *reinterpret_cast<const volatile unsigned long long *>(&side->kmax) < 0xffffffffull &&
           *reinterpret_cast<const volatile unsigned long long *>(&side->ror) < (1ull << 32);
}

struct NphjArgs {
    const tuple_v *R, *S;
    unsigned long long nR, nS;
    tuple_v *table;
    unsigned long long cap;
    NphjSide *side;
    JoinAccum *acc;
    int lp;     // first match per probe tuple instead of all matches
    int skip0;  // key 0 never matches (the phj_radix_lp rule)
    unsigned long long *side_pos;  // materialising joins: input positions of the side record's tuples
    MatOut mat;
    int compact_ok;  // the join may use compact slots (not materialising; key 0 may match)
    // Compact tables: capacity (a multiple of kSliceSlots) and the sliced build's buffers.
    unsigned long long ccap;
    unsigned int nslices;      // ccap / kSliceSlots; 0: no sliced build
    unsigned int hist_blocks;  // blocks of the width and scatter passes (each a contiguous range of R)
    unsigned long long *stage; // [nslices][kSliceMaxFill] build tuples as compact words, by slice
    uint32_t *slice_fill;      // [nslices] tuples staged per slice (claimed by the scatter blocks)
    // Sliced builds: the clear and the 16-byte probe of the other table forms run inside the slice build
    // and the compact probe when the device finds that the table is not built by slices, instead of as
    // launches of their own that return at once.
    int fused_fallback;
};

__device__ __forceinline__ bool compact_sliced(const NphjSide *side) {
    return *reinterpret_cast<const volatile unsigned int *>(&side->sliced) != 0;
}

// The join runs on the compact table: allowed, the widths fit, and for first-match joins the table is
// built by slices (the sliced build keeps one slot per key, with the first build tuple in input order;
// otherwise a first-match join uses the 16-byte table and its duplicate rebuild).
__device__ __forceinline__ bool use_compact(const NphjArgs &a) {
    return a.compact_ok && nphj_compact(a.side) && (!a.lp || compact_sliced(a.side));
}

__device__ __forceinline__ unsigned slice_of(unsigned long long key, unsigned long long ccap) {
    return (unsigned)(table_hash(key, ccap) >> kSliceLog);
}

// Next slot of a compact table's probe sequence: inside the slice when the table was built by slices.
__device__ __forceinline__ unsigned long long compact_next(unsigned long long h, bool sliced, unsigned long long ccap) {
    if (sliced) return (h & ~(unsigned long long)(kSliceSlots - 1)) | ((h + 1) & (kSliceSlots - 1));
    return h + 1 == ccap ? 0 : h + 1;
}

__device__ __forceinline__ void block_range(unsigned long long n, unsigned long long *lo, unsigned long long *hi) {
    const unsigned long long per = (n + gridDim.x - 1) / gridDim.x;
    *lo = blockIdx.x * per < n ? blockIdx.x * per : n;
    *hi = *lo + per < n ? *lo + per : n;
}

// Largest build key and OR of build row ids: the compact-slot test of a join whose compact table is
// not built by slices (the sliced build takes them in nphj_slice_scatter).
__global__ void __launch_bounds__(kSliceThreads) nphj_widths(NphjArgs a) {
    unsigned long long lo, hi;
    block_range(a.nR, &lo, &hi);
    unsigned long long kmax = 0, ror = 0;
    constexpr int U = 4;
    for (unsigned long long i0 = lo + threadIdx.x; i0 < hi; i0 += U * blockDim.x) {
        tuple_v t[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned long long i = i0 + u * blockDim.x;
            t[u] = i < hi ? ld_stream(a.R + i) : make_ulonglong2(0, 0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            kmax = max(kmax, t[u].x);
            ror |= t[u].y;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
        ror |= __shfl_xor_sync(0xffffffffu, ror, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&a.side->kmax, kmax);
        atomicOr(&a.side->ror, ror);
    }
}

// Empties the table the build will claim slots in: the 16-byte table when the keys or row ids are too
// wide for compact slots, the compact table when it is built by global CAS. A table built by slices
// is written whole by nphj_slice_build.
__device__ __forceinline__ void clear_table_body(const NphjArgs &a, bool sliced) {
    const bool compact = a.compact_ok && nphj_compact(a.side) && (!a.lp || sliced);  // use_compact
    if (compact && sliced) return;
    const unsigned long long words16 = compact ? a.ccap / 2 : a.cap;  // 16-byte units
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < words16;
         i += (unsigned long long)gridDim.x * blockDim.x)
        a.table[i] = make_ulonglong2(kEmpty, kEmpty);
}

__global__ void nphj_clear_table(NphjArgs a) { clear_table_body(a, compact_sliced(a.side)); }

// The sliced build's one pass over R: block b takes a contiguous range of R, takes the width ORs of the
// compact test and counts the range's tuples per slice in shared memory, claims each slice's space in
// the staging array with one global atomic per slice (in any order across blocks: no join semantics here
// depends on the order of tuples inside a slice), then reads its range again (from L2: it has just been
// read) and writes each tuple as a compact word (key << 32 | row id; first-match joins: key << 32 | input
// position) at its slice's claim plus its shared-memory rank. Claims past kSliceMaxFill mark the build
// not sliced; their tuples are not staged.
__global__ void __launch_bounds__(kSliceThreads) nphj_slice_scatter(NphjArgs a) {
    extern __shared__ uint32_t sh_cnt[];  // [nslices]: counts, then the next staging index of each slice
    for (unsigned j = threadIdx.x; j < a.nslices; j += blockDim.x) sh_cnt[j] = 0;
    __syncthreads();
    unsigned long long lo, hi;
    block_range(a.nR, &lo, &hi);
    constexpr int U = 4;
    unsigned long long kmax = 0, ror = 0;
    for (unsigned long long i0 = lo + threadIdx.x; i0 < hi; i0 += U * blockDim.x) {
        tuple_v t[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned long long i = i0 + u * blockDim.x;
            t[u] = i < hi ? ld_keep(a.R + i) : make_ulonglong2(0, 0);  // read again below
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            kmax = max(kmax, t[u].x);
            ror |= t[u].y;
            if (i0 + u * blockDim.x < hi && t[u].x < 0xffffffffull) atomicAdd(&sh_cnt[slice_of(t[u].x, a.ccap)], 1u);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
        ror |= __shfl_xor_sync(0xffffffffu, ror, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&a.side->kmax, kmax);
        atomicOr(&a.side->ror, ror);
    }
    __syncthreads();
    for (unsigned j = threadIdx.x; j < a.nslices; j += blockDim.x) {
        const uint32_t c = sh_cnt[j];
        if (!c) continue;
        const uint32_t b = atomicAdd(&a.slice_fill[j], c);
        if (b + c > kSliceMaxFill) atomicOr(&a.side->overflow, 1u);
        sh_cnt[j] = b;
    }
    __syncthreads();
    for (unsigned long long i0 = lo + threadIdx.x; i0 < hi; i0 += U * blockDim.x) {
        tuple_v t[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned long long i = i0 + u * blockDim.x;
            t[u] = i < hi ? ld_stream(a.R + i) : make_ulonglong2(0, 0);
            // Second and last read of R here: its lines go back to the normal eviction priority, so
            // the table the probe reads next keeps its place in L2.
            if (i < hi && (reinterpret_cast<uintptr_t>(a.R + i) & 127u) == 0)
                asm volatile("applypriority.global.L2::evict_normal [%0], 128;" ::"l"(a.R + i) : "memory");
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned long long i = i0 + u * blockDim.x;
            if (i >= hi || t[u].x >= 0xffffffffull) continue;
            const unsigned sl = slice_of(t[u].x, a.ccap);
            const uint32_t p = atomicAdd(&sh_cnt[sl], 1u);
            if (p < kSliceMaxFill) a.stage[(size_t)sl * kSliceMaxFill + p] = (t[u].x << 32) | (a.lp ? i : t[u].y);
        }
    }
}

__device__ void build_body(const NphjArgs &a);

__global__ void __launch_bounds__(kSliceThreads) nphj_slice_build(NphjArgs a) {
    extern __shared__ unsigned long long tab[];  // [kSliceSlots]
    // The mode of the build, now that the scatter has taken the widths and the slice fills: sliced when
    // the table is compact and no slice overflowed. Every block decides the same; block 0 records it for
    // the kernels after this one. Otherwise the table of the other form is cleared here for the build
    // that follows (nphj_build).
    const bool sliced = nphj_compact(a.side) && *reinterpret_cast<volatile unsigned int *>(&a.side->overflow) == 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.side->sliced = sliced ? 1u : 0u;
    if (!sliced) {
        clear_table_body(a, false);
        return;
    }
    bool seen_dup = false;
    unsigned long long *ctab = reinterpret_cast<unsigned long long *>(a.table);
    for (unsigned sl = blockIdx.x; sl < a.nslices; sl += gridDim.x) {
        for (unsigned j = threadIdx.x; j < kSliceSlots; j += blockDim.x) tab[j] = kCompactEmpty;
        __syncthreads();
        const uint32_t lo = sl * kSliceMaxFill, n = a.slice_fill[sl];
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned long long v = a.stage[lo + i];
            const unsigned long long k = v >> 32;
            unsigned h = (unsigned)table_hash(k, a.ccap) & (kSliceSlots - 1);
            for (unsigned steps = 0;;) {
                const unsigned long long cur = atomicCAS(&tab[h], kCompactEmpty, v);
                if (cur == kCompactEmpty) break;
                if ((cur >> 32) == k) {
                    seen_dup = true;
                    if (a.lp) {
                        atomicMin(&tab[h], v);
                        break;
                    }
                }
                h = (h + 1) & (kSliceSlots - 1);
                if (++steps >= kSliceSlots) {
                    set_error(&a.acc->error, kErrProbeLimit);
                    break;
                }
            }
        }
        __syncthreads();
        if (a.lp) {
            // Positions -> row ids; eight gathers in flight per thread.
            constexpr int G = 8;
            for (unsigned j0 = threadIdx.x; j0 < kSliceSlots; j0 += G * blockDim.x) {
                unsigned long long w[G], rid[G];
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const unsigned j = j0 + g * blockDim.x;
                    w[g] = j < kSliceSlots ? tab[j] : kCompactEmpty;
                    const unsigned long long p = w[g] & 0xffffffffull;
                    rid[g] = (w[g] != kCompactEmpty && p < a.nR) ? a.R[p].y : 0ull;
                }
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const unsigned j = j0 + g * blockDim.x;
                    if (j >= kSliceSlots || w[g] == kCompactEmpty) continue;
                    if ((w[g] & 0xffffffffull) >= a.nR) set_error(&a.acc->error, kErrBounds);
                    tab[j] = (w[g] & ~0xffffffffull) | rid[g];
                }
            }
            __syncthreads();
        }
        ulonglong2 *dst = reinterpret_cast<ulonglong2 *>(ctab + (size_t)sl * kSliceSlots);
        const ulonglong2 *src = reinterpret_cast<const ulonglong2 *>(tab);
        for (unsigned j = threadIdx.x; j < kSliceSlots / 2; j += blockDim.x) dst[j] = src[j];
        __syncthreads();
    }
    if (__syncthreads_or(seen_dup) && threadIdx.x == 0) atomicOr(&a.side->dup, 1u);
}

// Compact build by global CAS (the table was not built by slices): the CAS writes key and row id together.
__device__ __forceinline__ void nphj_insert_compact(const NphjArgs &a, unsigned long long *ctab, const tuple_v t,
                                                    bool &seen_dup) {
    const unsigned long long v = (t.x << 32) | t.y;
    unsigned long long h = table_hash(t.x, a.ccap);
    for (unsigned long long steps = 0;;) {
        const unsigned long long cur = atomicCAS(ctab + h, kCompactEmpty, v);
        if (cur == kCompactEmpty) return;
        if ((cur >> 32) == t.x) seen_dup = true;
        if (++h == a.ccap) h = 0;
        if (++steps >= a.ccap) {
            set_error(&a.acc->error, kErrProbeLimit);
            return;
        }
    }
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long *p) {
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

// Insert R tuple i at its own slot; records duplicates.
__device__ __forceinline__ void nphj_insert(const NphjArgs &a, const tuple_v t, unsigned long long i, bool &seen_dup) {
    if (a.skip0 && t.x == 0) return;
    if (t.x == kEmpty) {
        const unsigned long long q = atomicAdd(&a.side->cnt, 1ull);
        if (q >= 1ull) seen_dup = true;
        if (a.side_pos) a.side_pos[q] = i;
        atomicAdd(&a.side->sum, (unsigned long long)t.y);
        atomicMin(&a.side->minpos, i);
        return;
    }
    unsigned long long h = table_hash(t.x, a.cap);
    for (unsigned long long steps = 0;;) {
        // Claim with a CAS straight away: at load <= 0.5 most first slots are empty.
        const unsigned long long cur = atomicCAS(&a.table[h].x, kEmpty, (unsigned long long)t.x);
        if (cur == kEmpty) {
            a.table[h].y = t.y;
            return;
        }
        if (cur == t.x) seen_dup = true;
        if (++h == a.cap) h = 0;
        if (++steps >= a.cap) {
            set_error(&a.acc->error, kErrProbeLimit);
            return;
        }
    }
}

// Build of the table forms other than the sliced one: the compact table by global CAS, or the 16-byte
// table. All threads of a block call it (block-wide vote at the end).
__device__ void build_body(const NphjArgs &a) {
    constexpr int U = 4;
    bool seen_dup = false;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    if (use_compact(a)) {
        if (compact_sliced(a.side)) return;  // nphj_slice_build built the table
        unsigned long long *ctab = reinterpret_cast<unsigned long long *>(a.table);
        for (unsigned long long i0 = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i0 < a.nR;
             i0 += U * stride) {
            tuple_v t[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const unsigned long long i = i0 + u * stride;
                t[u] = i < a.nR ? ld_stream(a.R + i) : make_ulonglong2(0, 0);
            }
#pragma unroll
            for (int u = 0; u < U; u++)
                if (i0 + u * stride < a.nR) nphj_insert_compact(a, ctab, t[u], seen_dup);
        }
        if (__syncthreads_or(seen_dup) && threadIdx.x == 0) atomicOr(&a.side->dup, 1u);
        return;
    }
    for (unsigned long long i0 = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i0 < a.nR;
         i0 += U * stride) {
        tuple_v t[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned long long i = i0 + u * stride;
            t[u] = i < a.nR ? ld_stream(a.R + i) : make_ulonglong2(0, 0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned long long i = i0 + u * stride;
            if (i < a.nR) nphj_insert(a, t[u], i, seen_dup);
        }
    }
    if (__syncthreads_or(seen_dup) && threadIdx.x == 0) atomicOr(&a.side->dup, 1u);
}

__global__ void nphj_build(NphjArgs a) { build_body(a); }

// Duplicate-key rebuild for nphj_lp: one slot per distinct key holding the minimum input position.
__global__ void nphj_lp_refill(NphjArgs a) {
    if (use_compact(a) || !(*reinterpret_cast<volatile unsigned int *>(&a.side->dup))) return;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < a.cap;
         i += (unsigned long long)gridDim.x * blockDim.x)
        a.table[i] = make_ulonglong2(kEmpty, kEmpty);
}

__global__ void nphj_lp_dedup_build(NphjArgs a) {
    if (use_compact(a) || !(*reinterpret_cast<volatile unsigned int *>(&a.side->dup))) return;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < a.nR;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const unsigned long long k = a.R[i].x;
        if (k == kEmpty || (a.skip0 && k == 0)) continue;
        unsigned long long h = table_hash(k, a.cap);
        unsigned long long steps = 0;
        for (;;) {
            unsigned long long *kp = &a.table[h].x;
            unsigned long long cur = ld_volatile_u64(kp);
            if (cur == kEmpty) cur = atomicCAS(kp, kEmpty, k);
            if (cur == kEmpty || cur == k) {
                atomicMin(&a.table[h].y, i);
                break;
            }
            if (++h == a.cap) h = 0;
            if (++steps >= a.cap) {
                set_error(&a.acc->error, kErrProbeLimit);
                break;
            }
        }
    }
}

__global__ void nphj_lp_resolve(NphjArgs a) {
    if (use_compact(a) || !(*reinterpret_cast<volatile unsigned int *>(&a.side->dup))) return;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < a.cap;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        tuple_v s = a.table[i];
        if (s.x != kEmpty) {
            if (s.y < a.nR)
                a.table[i].y = a.R[s.y].y;
            else
                set_error(&a.acc->error, kErrBounds);
        }
    }
}

// Probe of a compact-slot table (see nphj_build); a no-op otherwise. V probes per thread: four for
// tables up to kCompactDeepProbeBytes (the 8-byte slots leave the registers for it), one above.
__device__ __forceinline__ void probe16_body(const NphjArgs &a, unsigned long long *red);

template <int V>
__global__ void __launch_bounds__(256) nphj_probe_compact(NphjArgs a) {
    __shared__ unsigned long long red[64];
    if (!use_compact(a)) {
        if (a.fused_fallback) probe16_body(a, red);
        return;
    }
    // Compact slots: no build key is the empty pattern, so there is no side record; a probe key
    // at or above 2^32 - 1 cannot match.
    const unsigned long long *ctab = reinterpret_cast<const unsigned long long *>(a.table);
    const bool first_only = a.lp || *reinterpret_cast<volatile unsigned int *>(&a.side->dup) == 0;
    const bool sliced = compact_sliced(a.side);
    const unsigned long long max_steps = sliced ? kSliceSlots : a.ccap;
    unsigned long long cnt = 0, sum = 0;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long j0 = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; j0 < a.nS;
         j0 += V * stride) {
        tuple_v sv[V];
        unsigned long long h[V], e[V];
        bool walk[V];
#pragma unroll
        for (int u = 0; u < V; u++) {
            const unsigned long long j = j0 + u * stride;
            sv[u] = j < a.nS ? ld_stream(a.S + j) : make_ulonglong2(0, 0);
            walk[u] = j < a.nS && sv[u].x < 0xffffffffull;
        }
#pragma unroll
        for (int u = 0; u < V; u++) {
            if (walk[u]) {
                h[u] = table_hash(sv[u].x, a.ccap);
                e[u] = ld_slot8(ctab + h[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < V; u++) {
            if (!walk[u]) continue;
            unsigned long long hh = h[u], ee = e[u];
            for (unsigned long long steps = 0;;) {
                if (ee == kCompactEmpty) break;
                if ((ee >> 32) == sv[u].x) {
                    cnt++;
                    sum += (ee & 0xffffffffull) + sv[u].y;
                    if (first_only) break;
                }
                hh = compact_next(hh, sliced, a.ccap);
                if (++steps >= max_steps) {
                    set_error(&a.acc->error, kErrProbeLimit);
                    break;
                }
                ee = ld_slot8(ctab + hh);
            }
        }
    }
    block_sum2_to(cnt, sum, red, &a.acc->matched, &a.acc->checksum);
}

// Two probes per thread at eight 256-thread blocks per SM measured best for tables that sit in L2
// (more probes per thread cost occupancy through registers).
__device__ __forceinline__ void probe16_body(const NphjArgs &a, unsigned long long *red) {
    constexpr int U = 2;
    ProbeArgs P;
    P.table = a.table;
    P.cap = a.cap;
    P.lp = a.lp != 0;
    P.skip0 = a.skip0 != 0;
    P.first_only = P.lp || *reinterpret_cast<volatile unsigned int *>(&a.side->dup) == 0;
    P.side_cnt = a.side->cnt;
    P.side_sum = a.side->sum;
    P.side_first_rid = P.side_cnt ? a.R[a.side->minpos].y : 0;
    P.err = &a.acc->error;
    unsigned long long cnt = 0, sum = 0;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long j0 = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; j0 < a.nS;
         j0 += U * stride) {
        tuple_v sv[U];
        bool valid[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned long long j = j0 + u * stride;
            valid[u] = j < a.nS;
            sv[u] = valid[u] ? ld_stream(a.S + j) : make_ulonglong2(0, 0);
        }
        probe_group<U>(P, sv, valid, cnt, sum);
    }
    block_sum2_to(cnt, sum, red, &a.acc->matched, &a.acc->checksum);
}

__global__ void __launch_bounds__(256, 8) nphj_probe(NphjArgs a) {
    __shared__ unsigned long long red[64];
    if (use_compact(a)) return;  // nphj_probe_compact probes instead
    probe16_body(a, red);
}

// Materialising probe: block-wide rounds of one probe tuple per thread; each thread counts its matches,
// the block reserves output slots with one atomic, then each thread walks again and writes its pairs.
__global__ void __launch_bounds__(256) nphj_probe_mat(NphjArgs a) {
    __shared__ uint32_t scan_tmp[32];
    __shared__ unsigned long long s_base;
    const bool lp = a.lp != 0, skip0 = a.skip0 != 0;
    const bool first_only = lp || *reinterpret_cast<volatile unsigned int *>(&a.side->dup) == 0;
    const unsigned long long side_cnt = a.side->cnt;
    unsigned int *err = &a.acc->error;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long j0 = blockIdx.x * (unsigned long long)blockDim.x; j0 < a.nS; j0 += stride) {
        const unsigned long long j = j0 + threadIdx.x;
        const bool valid = j < a.nS;
        const tuple_v sv = valid ? ld_stream(a.S + j) : make_ulonglong2(0, 0);
        uint32_t m = 0;
        unsigned long long h0 = 0;
        const bool walk = valid && sv.x != kEmpty && !(skip0 && sv.x == 0);
        if (valid && sv.x == kEmpty) {
            m = side_cnt ? (lp ? 1u : (uint32_t)side_cnt) : 0u;
        } else if (walk) {
            h0 = table_hash(sv.x, a.cap);
            unsigned long long h = h0;
            for (unsigned long long steps = 0;;) {
                const tuple_v e = ld_slot(a.table + h);
                if (e.x == kEmpty) break;
                if (e.x == sv.x) {
                    m++;
                    if (first_only) break;
                }
                if (++h == a.cap) h = 0;
                if (++steps >= a.cap) {
                    set_error(err, kErrProbeLimit);
                    break;
                }
            }
        }
        unsigned long long o = mat_reserve(m, scan_tmp, &s_base, &a.acc->pairs);
        if (!m) continue;
        if (sv.x == kEmpty) {
            if (lp)
                mat_put(a.mat, o, a.R[a.side->minpos].y, sv.y, err);
            else
                for (unsigned long long q = 0; q < side_cnt; q++) mat_put(a.mat, o + q, a.R[a.side_pos[q]].y, sv.y, err);
            continue;
        }
        unsigned long long h = h0;
        for (unsigned long long steps = 0, w = 0; w < m && steps < a.cap; steps++) {
            const tuple_v e = ld_slot(a.table + h);
            if (e.x == kEmpty) break;
            if (e.x == sv.x) mat_put(a.mat, o + w++, e.y, sv.y, err);
            if (++h == a.cap) h = 0;
        }
    }
}

// Retrieve phase of the materialising joins (the reference's ptr_retrieve, src/inc/utils.c:712-724):
// gather R[r_row_id - 1].row_id + S[s_row_id - 1].row_id for every pair and sum with wrap-around.
__global__ void mat_retrieve(const ulonglong2 *__restrict__ pairs, const unsigned long long *n_dev,
                             unsigned long long cap, const tuple_v *__restrict__ R, unsigned long long nR,
                             const tuple_v *__restrict__ S, unsigned long long nS, JoinAccum *acc) {
    unsigned long long n = *n_dev;
    if (n > cap) n = cap;
    unsigned long long sum = 0;
    bool bad = false;
    // Eight pairs per thread and step: their 16 gathers are all in flight before any is summed.
    constexpr int U = 8;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i0 = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i0 < n;
         i0 += U * stride) {
        ulonglong2 p[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const unsigned long long i = i0 + u * stride;
            p[u] = i < n ? ld_stream(pairs + i) : make_ulonglong2(0, 0);
        }
        unsigned long long rv[U], sv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const bool live = i0 + u * stride < n;
            const bool ok = p[u].x - 1 < nR && p[u].y - 1 < nS;
            bad = bad || (live && !ok);
            rv[u] = live && ok ? __ldg(&R[p[u].x - 1].y) : 0ull;
            sv[u] = live && ok ? __ldg(&S[p[u].y - 1].y) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < U; u++) sum += rv[u] + sv[u];
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) set_error(&acc->error, kErrRowId);
    sum = warp_sum_u64(sum);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(&acc->checksum, sum);
}

// Default load factor of the global table: 0.4 for build relations up to 5 M tuples, 0.5 above. Below
// that size the table is about the size of L2 and shorter probe chains pay for the larger table
// (nphj_sc 2^22 x 2^23 on B200: probe 0.115 -> 0.102 ms); above it the larger table costs more than
// the chains save (2^24 x 2^25: 1.27 ms at 0.5, 1.41 at 0.4).
double nphj_default_load(size_t nR) { return nR <= 5000000 ? 0.4 : 0.5; }

static unsigned long long nphj_cap(size_t nR, double load) {
    if (!(load > 0.05 && load < 0.95)) load = nphj_default_load(nR);
    unsigned long long cap = (unsigned long long)((double)nR / load) + 2;
    if (cap < 16) cap = 16;
    return cap;
}

size_t nphj_scratch_bytes(size_t nR, double load, bool mat) {
    return (size_t)nphj_cap(nR, load) * 16 + 256 + (mat ? (size_t)nR * 8 : 0);
}

#define HJ_CU(call)                                                                   \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            fprintf(stderr, "hjscm: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return HJ_E_DEVICE;                                                       \
        }                                                                             \
    } while (0)

static std::mutex g_nphj_attr_mu;
static bool g_nphj_attr_done[64];

// Shared-memory limits of the sliced build's kernels, once per device.
int nphj_prepare_device() {
    int dev = 0;
    HJ_CU(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return HJ_E_INVAL;
    std::lock_guard<std::mutex> lk(g_nphj_attr_mu);
    if (g_nphj_attr_done[dev]) return HJ_OK;
    HJ_CU(cudaFuncSetAttribute(nphj_slice_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(kSliceMaxCount * 4)));
    HJ_CU(cudaFuncSetAttribute(nphj_slice_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kSliceSlots * 8)));
    g_nphj_attr_done[dev] = true;
    return HJ_OK;
}

int nphj_enqueue(bool lp, bool skip0, const ulonglong2 *R, size_t nR, const ulonglong2 *S, size_t nS, void *table,
                 size_t table_bytes, double load, JoinAccum *acc, cudaStream_t st, cudaEvent_t ev_mid,
                 int num_sms, cudaEvent_t *ph, uint32_t *launches, const MatOut *mat, int phases) {
    const bool do_build = (phases & kNphjBuild) != 0, do_probe = (phases & kNphjProbe) != 0;
    const unsigned long long cap = nphj_cap(nR, load);
    if (cap * 16 + 256 + (mat ? (unsigned long long)nR * 8 : 0ull) > table_bytes) return HJ_E_INVAL;
    NphjArgs a;
    a.R = R;
    a.S = S;
    a.nR = nR;
    a.nS = nS;
    a.table = reinterpret_cast<tuple_v *>(table);
    a.cap = cap;
    a.side = reinterpret_cast<NphjSide *>(reinterpret_cast<char *>(table) + cap * 16);
    a.acc = acc;
    a.lp = lp ? 1 : 0;
    a.skip0 = skip0 ? 1 : 0;
    a.side_pos = mat ? reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(table) + cap * 16 + 256)
                     : nullptr;
    a.mat = mat ? *mat : MatOut{nullptr, 0};
    // Compact slots pay off once the 16-byte table outgrows a share of L2; below that the extra pass
    // over R costs more than it saves.
    a.compact_ok = (!mat && !skip0 && cap * 16 > kCompactMinTableBytes) ? 1 : 0;
    // Compact table: capacity rounded up to whole slices; behind it (inside the 16-byte table's bytes)
    // the sliced build's staging array, histograms and slice starts.
    a.ccap = (cap + kSliceSlots - 1) / kSliceSlots * kSliceSlots;
    a.nslices = 0;
    a.fused_fallback = 0;
    a.hist_blocks = (unsigned)num_sms * 2;
    a.stage = nullptr;
    a.slice_fill = nullptr;
    if (a.compact_ok) {
        const unsigned long long ns = a.ccap / kSliceSlots;
        char *p = reinterpret_cast<char *>(table) + ((a.ccap * 8 + 255) & ~255ull);
        char *const end = reinterpret_cast<char *>(table) + cap * 16;
        char *q = p + ((ns * kSliceMaxFill * 8 + 255) & ~255ull);
        if (ns <= kSliceMaxCount && q + ns * 4 <= end) {
            a.nslices = (unsigned)ns;
            a.stage = reinterpret_cast<unsigned long long *>(p);
            a.slice_fill = reinterpret_cast<uint32_t *>(q);
            a.fused_fallback = 1;
        }
    }
    if (a.compact_ok) {
        const int rc = nphj_prepare_device();
        if (rc) return rc;
    }
    const int grid = num_sms * 8;
    // Joins that may use compact slots launch the 16-byte-table kernels (and the table clear) as
    // fallbacks that usually return at once; their grid is kept small, since a launch of idle blocks
    // still costs time in proportion to the blocks.
    const int fb_grid = a.compact_ok ? num_sms * 4 : grid;
    uint32_t nl = 0;
    if (do_build) {
    if (!a.compact_ok) HJ_CU(cudaMemsetAsync(table, 0xff, cap * 16, st));
    HJ_CU(cudaMemsetAsync(a.side, 0, sizeof(NphjSide), st));
    HJ_CU(cudaMemsetAsync(&a.side->minpos, 0xff, sizeof(unsigned long long), st));
    // Phase slots: build spans [0, 1], probe spans [4, 5]; the others stay empty.
    if (ph) HJ_CU(record_event(ph[0], st));
    if (a.compact_ok) {
        if (a.nslices) {
            // One pass over R (widths, per-slice claims, staging), the slice build (or, when the table
            // is not built by slices, the clear of the table the fallback build needs).
            HJ_CU(cudaMemsetAsync(a.slice_fill, 0, (size_t)a.nslices * 4, st));
            nphj_slice_scatter<<<a.hist_blocks, kSliceThreads, (size_t)a.nslices * 4, st>>>(a);
            const unsigned bgrid = a.nslices < (unsigned)num_sms * 3 ? a.nslices : (unsigned)num_sms * 3;
            nphj_slice_build<<<bgrid, kSliceThreads, kSliceSlots * 8, st>>>(a);
            nl += 2;
        } else {
            nphj_widths<<<a.hist_blocks, kSliceThreads, 0, st>>>(a);
            nphj_clear_table<<<num_sms * 2, 256, 0, st>>>(a);
            nl += 2;
        }
    }
    // The build of the other table forms (a compact table by global CAS, or the 16-byte table); it
    // returns at once when the table was built by slices.
    nphj_build<<<fb_grid, 256, 0, st>>>(a);
    nl++;
    if (lp) {
        nphj_lp_refill<<<fb_grid, 256, 0, st>>>(a);
        nphj_lp_dedup_build<<<fb_grid, 256, 0, st>>>(a);
        nphj_lp_resolve<<<fb_grid, 256, 0, st>>>(a);
        nl += 3;
    }
    HJ_CU(cudaGetLastError());
    }  // do_build
    if (!do_probe) {
        if (launches) *launches = nl;
        return HJ_OK;
    }
    if (ev_mid) HJ_CU(record_event(ev_mid, st));
    if (ph) {
        for (int i = 1; i <= 4; i++) HJ_CU(record_event(ph[i], st));
    }
    if (nS) {
        if (mat) {
            nphj_probe_mat<<<grid, 256, 0, st>>>(a);
        } else {
            if (!a.fused_fallback) nphj_probe<<<fb_grid, 256, 0, st>>>(a);
            if (a.compact_ok) {
                if (a.ccap * 8 <= kCompactDeepProbeBytes)
                    nphj_probe_compact<4><<<grid, 256, 0, st>>>(a);
                else
                    nphj_probe_compact<1><<<grid, 256, 0, st>>>(a);
            }
        }
    }
    HJ_CU(cudaGetLastError());
    if (ph) {
        HJ_CU(record_event(ph[5], st));
        HJ_CU(record_event(ph[6], st));
    }
    if (launches) *launches = nl + (nS ? (mat || !a.compact_ok || a.fused_fallback ? 1u : 2u) : 0u);
    return HJ_OK;
}

int mat_retrieve_enqueue(const ulonglong2 *pairs, const unsigned long long *n_dev, unsigned long long cap,
                         const ulonglong2 *R, size_t nR, const ulonglong2 *S, size_t nS, JoinAccum *acc,
                         cudaStream_t st, int num_sms) {
    mat_retrieve<<<num_sms * 8, 256, 0, st>>>(pairs, n_dev, cap, R, nR, S, nS, acc);
    HJ_CU(cudaGetLastError());
    return HJ_OK;
}

}  // namespace hj
