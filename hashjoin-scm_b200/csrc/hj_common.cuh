// hj_common.cuh - device-side building blocks shared by the join kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/hjscm.h"

namespace hj {

// 16-byte tuple as one vector register pair: x = key, y = row_id (src/inc/store.h:87-96).
using tuple_v = ulonglong2;

constexpr int kWarp = 32;

// Device error word bits, OR-ed in by kernels and turned into HJ_E_* codes by the host.
enum : uint32_t {
    kErrProbeLimit = 1u << 0,   // a table walk exceeded capacity
    kErrSpinLimit = 1u << 1,    // a bounded wait (look-back, barrier) gave up
    kErrBounds = 1u << 2,       // a computed output index fell outside its buffer
    kErrCapacity = 1u << 3,     // a work list or table ran out of room
    kErrOutput = 1u << 4,       // materialised pairs did not fit the output buffer
    kErrRowId = 1u << 5,        // a materialised row id is not a 1-based position of its relation
};

// Device-resident per-join accumulators and flags (one 64-byte line).
struct JoinAccum {
    unsigned long long matched;
    unsigned long long checksum;
    unsigned int error;
    unsigned int dup_flag;      // set by NPHJ builds that saw an equal key twice
    unsigned long long large_parts;
    unsigned long long pairs;   // materialising joins: output slots reserved so far
    unsigned long long flags;   // HJ_RES_* bits of hj_result_t.flags
    unsigned long long pad[2];
};

__device__ __forceinline__ void set_error(unsigned int *err, uint32_t bit) { atomicOr(err, bit); }

// L2 policy that marks lines evict-first (createpolicy, sm_80+).
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// Read-only load that L2 keeps as long as it can (a relation read twice in a row: the second read is
// served from L2).
__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ tuple_v ld_keep(const tuple_v *p) {
    tuple_v v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
                 : "=l"(v.x), "=l"(v.y)
                 : "l"(p), "l"(policy_evict_last()));
    return v;
}

// Streaming 16-byte load that skips L1 and marks the L2 line evict-first: every input tuple of a
// partition pass or probe is read exactly once.
__device__ __forceinline__ tuple_v ld_stream(const tuple_v *p) {
    tuple_v v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;"
                 : "=l"(v.x), "=l"(v.y)
                 : "l"(p), "l"(policy_evict_first()));
    return v;
}

// Streaming store: the partition output is re-read only by the next pass, after the whole pass.
__device__ __forceinline__ void st_stream(tuple_v *p, tuple_v v) {
    asm volatile("st.global.cs.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(v.x), "l"(v.y) : "memory");
}

// 8-byte variants for partitions stored as compact words (key bits above the radix bits << 32 | row id).
__device__ __forceinline__ unsigned long long ld_stream8(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u64 %0, [%1], %2;"
                 : "=l"(v)
                 : "l"(p), "l"(policy_evict_first()));
    return v;
}

__device__ __forceinline__ void st_stream8(unsigned long long *p, unsigned long long v) {
    asm volatile("st.global.cs.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of two u64 values (wrapping); result valid in thread 0. `red` needs 2*32 u64.
__device__ __forceinline__ void block_sum2_to(unsigned long long a, unsigned long long b,
                                              unsigned long long *red, unsigned long long *dst_a,
                                              unsigned long long *dst_b) {
    a = warp_sum_u64(a);
    b = warp_sum_u64(b);
    const unsigned w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane_id() == 0) {
        red[w] = a;
        red[32 + w] = b;
    }
    __syncthreads();
    if (w == 0) {
        unsigned long long x = lane_id() < nw ? red[lane_id()] : 0ull;
        unsigned long long y = lane_id() < nw ? red[32 + lane_id()] : 0ull;
        x = warp_sum_u64(x);
        y = warp_sum_u64(y);
        if (lane_id() == 0) {
            if (x) atomicAdd(dst_a, x);
            if (y) atomicAdd(dst_b, y);
        }
    }
    __syncthreads();
}

// Exclusive scan of one u32 per thread across the block (blockDim <= 1024). `tmp` needs 32 u32.
// Returns the exclusive prefix; *total receives the block total.
__device__ __forceinline__ uint32_t block_excl_scan_u32(uint32_t v, uint32_t *tmp, uint32_t *total) {
    const unsigned lane = lane_id(), w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) tmp[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < nw ? tmp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= (unsigned)o) s += y;
        }
        tmp[lane] = s;  // inclusive warp totals
    }
    __syncthreads();
    uint32_t warp_base = w ? tmp[w - 1] : 0u;
    if (total) *total = tmp[nw - 1];
    __syncthreads();
    return warp_base + x - v;
}

// Output of a materialising join: (r.row_id, s.row_id) pairs; the slot cursor is JoinAccum::pairs.
struct MatOut {
    ulonglong2 *pairs;
    unsigned long long cap;
};

// One round of a materialising probe loop: every thread of the block passes the number of pairs it
// will write; returns the thread's first output slot. One global atomic per block and round. Must be
// reached by all threads of the block (it contains barriers); s_base is one shared u64.
__device__ __forceinline__ unsigned long long mat_reserve(uint32_t m, uint32_t *scan_tmp, unsigned long long *s_base,
                                                          unsigned long long *cursor) {
    uint32_t total = 0;
    const uint32_t ex = block_excl_scan_u32(m, scan_tmp, &total);
    if (threadIdx.x == 0) *s_base = total ? atomicAdd(cursor, (unsigned long long)total) : 0ull;
    __syncthreads();
    const unsigned long long b = *s_base + ex;
    __syncthreads();
    return b;
}

__device__ __forceinline__ void mat_put(const MatOut &o, unsigned long long slot, unsigned long long r_rid,
                                        unsigned long long s_rid, unsigned int *err) {
    if (slot < o.cap)
        o.pairs[slot] = make_ulonglong2(r_rid, s_rid);
    else
        set_error(err, kErrOutput);
}

// Hash for the global (non-partitioned) tables: multiply-xorshift, then range reduction by the high
// 64 bits of a 64x64 product so any capacity works. Results do not depend on the hash function: the
// reference's identity hash (src/algo/params.h:9-11) only decides which slot a key lands in.
__device__ __forceinline__ uint64_t table_hash(uint64_t key, uint64_t cap) {
    uint64_t h = key * 0x9e3779b97f4a7c15ull;
    h ^= h >> 29;
    h *= 0xbf58476d1ce4e5b9ull;
    h ^= h >> 32;
    return __umul64hi(h, cap);
}

}  // namespace hj
