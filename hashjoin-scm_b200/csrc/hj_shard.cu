// hj_shard.cu - routing of tuples to the ranks of a sharded join.
//
// A join sharded over G GPUs sends every tuple to the rank that owns its key, joins locally and adds up
// the G results. Co-partitions of a radix join are independent (src/algo/phj.c:1257-1311), and so are
// the key ranges of any key -> rank function, so one exchange step suffices. The owner of a key is
// mulhi(mix(key ^ 0x5ca1ab1e5eed0001), G): a multiply-xorshift mix (the same family as the tables'
// hash, on a different input) reduced to [0, G) by a multiply-high, so neither the radix digits (the
// low key bits) nor the table hash of a rank's keys is skewed by the routing.
//
// hj_shard_route groups the tuples of one relation by owner, stably: within an owner's range the
// tuples keep their input order, so after an all-to-all that concatenates the ranks' pieces in rank
// order, each rank's build relation is in global input order (first-match joins stay exact).
//
// Kernels (all block ranges are contiguous slices of the input, in block order):
//   route_count    per block and owner: tuples (shared-memory counters)
//   route_offsets  one CTA: each block's start per owner (exclusive scan down the columns, then owner
//                  bases), and the owner totals
//   route_scatter  per block, tiles of 8 tuples per thread: per-owner exclusive scans across the
//                  block's threads give each tuple its stable position.
#include <cstdio>

#include "../host/hj_feistel.h"
#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {

constexpr int kRouteThreads = 256;
constexpr int kRouteItems = 8;
constexpr int kRouteMaxShards = 32;

__device__ __forceinline__ unsigned shard_of(unsigned long long key, unsigned nshards) {
    return (unsigned)__umul64hi(hj_mix64(key ^ 0x5ca1ab1e5eed0001ull), (unsigned long long)nshards);
}

__device__ __forceinline__ void route_block_range(unsigned long long n, unsigned long long *lo,
                                                  unsigned long long *hi) {
    // Whole tiles per block, so that a tile never straddles two blocks.
    constexpr unsigned long long T = (unsigned long long)kRouteThreads * kRouteItems;
    const unsigned long long tiles = (n + T - 1) / T;
    const unsigned long long per = (tiles + gridDim.x - 1) / gridDim.x * T;
    *lo = blockIdx.x * per < n ? blockIdx.x * per : n;
    *hi = *lo + per < n ? *lo + per : n;
}

__global__ void __launch_bounds__(kRouteThreads) route_count(const tuple_v *__restrict__ in, unsigned long long n,
                                                             unsigned nshards, uint32_t *__restrict__ blk_cnt) {
    __shared__ uint32_t cnt[kRouteMaxShards];
    if (threadIdx.x < kRouteMaxShards) cnt[threadIdx.x] = 0;
    __syncthreads();
    unsigned long long lo, hi;
    route_block_range(n, &lo, &hi);
    for (unsigned long long i = lo + threadIdx.x; i < hi; i += blockDim.x)
        atomicAdd(&cnt[shard_of(ld_stream(in + i).x, nshards)], 1u);
    __syncthreads();
    if (threadIdx.x < nshards) blk_cnt[(size_t)blockIdx.x * nshards + threadIdx.x] = cnt[threadIdx.x];
}

// One CTA of 1024 threads; lane = owner, warp w sums a contiguous run of block rows.
__global__ void __launch_bounds__(1024) route_offsets(const uint32_t *__restrict__ blk_cnt, unsigned nblocks,
                                                      unsigned nshards, unsigned long long *__restrict__ blk_off,
                                                      unsigned long long *__restrict__ totals) {
    __shared__ unsigned long long part[32][33];
    const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const bool valid = lane < nshards;
    const unsigned rpw = (nblocks + 31) / 32;
    const unsigned r0 = w * rpw, r1 = min(nblocks, r0 + rpw);
    unsigned long long sum = 0;
    for (unsigned r = r0; r < r1 && valid; r++) sum += blk_cnt[(size_t)r * nshards + lane];
    part[w][lane] = sum;
    __syncthreads();
    if (w == 0) {
        unsigned long long run = 0;
        for (int q = 0; q < 32; q++) {
            const unsigned long long v = part[q][lane];
            part[q][lane] = run;
            run += v;
        }
        // Owner bases: exclusive scan of the owner totals across the lanes.
        unsigned long long incl = valid ? run : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += v;
        }
        const unsigned long long base = incl - (valid ? run : 0);
        if (valid) totals[lane] = run;
        for (int q = 0; q < 32; q++) part[q][lane] += base;
    }
    __syncthreads();
    unsigned long long run = part[w][lane];
    for (unsigned r = r0; r < r1 && valid; r++) {
        const size_t q = (size_t)r * nshards + lane;
        blk_off[q] = run;
        run += blk_cnt[q];
    }
}

__global__ void __launch_bounds__(kRouteThreads) route_scatter(const tuple_v *__restrict__ in, unsigned long long n,
                                                               unsigned nshards,
                                                               const unsigned long long *__restrict__ blk_off,
                                                               tuple_v *__restrict__ out, unsigned int *err) {
    __shared__ unsigned long long base[kRouteMaxShards];  // next output index of each owner for this block
    __shared__ uint32_t warp_tot[kRouteMaxShards][kRouteThreads / 32];
    const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x < nshards) base[threadIdx.x] = blk_off[(size_t)blockIdx.x * nshards + threadIdx.x];
    __syncthreads();
    unsigned long long lo, hi;
    route_block_range(n, &lo, &hi);
    constexpr unsigned T = kRouteThreads * kRouteItems;
    for (unsigned long long t0 = lo; t0 < hi; t0 += T) {
        // Thread t takes tuples [t * ITEMS, (t + 1) * ITEMS) of the tile, in order.
        tuple_v v[kRouteItems];
        unsigned own[kRouteItems];
#pragma unroll
        for (int u = 0; u < kRouteItems; u++) {
            const unsigned long long i = t0 + (unsigned long long)threadIdx.x * kRouteItems + u;
            if (i < hi) {
                v[u] = ld_stream(in + i);
                own[u] = shard_of(v[u].x, nshards);
            } else {
                v[u] = make_ulonglong2(0, 0);
                own[u] = kRouteMaxShards;
            }
        }
        unsigned long long my_pos[kRouteItems];
        for (unsigned s = 0; s < nshards; s++) {
            uint32_t c = 0;
#pragma unroll
            for (int u = 0; u < kRouteItems; u++) c += own[u] == s;
            // Exclusive scan of c across the block's threads (thread order = input order).
            uint32_t incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= (unsigned)o) incl += x;
            }
            if (lane == 31) warp_tot[s][w] = incl;
            __syncthreads();
            uint32_t before = 0, total = 0;
            for (unsigned q = 0; q < kRouteThreads / 32; q++) {
                const uint32_t x = warp_tot[s][q];
                if (q < w) before += x;
                total += x;
            }
            unsigned long long p = base[s] + before + incl - c;
#pragma unroll
            for (int u = 0; u < kRouteItems; u++)
                if (own[u] == s) my_pos[u] = p++;
            __syncthreads();
            if (threadIdx.x == 0) base[s] += total;
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < kRouteItems; u++) {
            if (own[u] >= nshards) continue;
            if (my_pos[u] < n)
                out[my_pos[u]] = v[u];
            else
                set_error(err, kErrBounds);
        }
    }
}

}  // namespace hj

namespace {
size_t route_blocks(size_t n, int num_sms) {
    const size_t T = (size_t)hj::kRouteThreads * hj::kRouteItems;
    const size_t tiles = (n + T - 1) / T;
    size_t b = (size_t)num_sms * 2;
    if (tiles < b) b = tiles ? tiles : 1;
    return b;
}
size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }
}  // namespace

extern "C" {

size_t hj_shard_route_scratch_bytes(size_t n, int nshards) {
    if (nshards < 1) nshards = 1;
    // Enough for any device's SM count (the block count is at most 2 * 1024 SMs).
    const size_t blocks = route_blocks(n, 1024);
    return a256(blocks * nshards * 4) + a256(blocks * nshards * 8) + 256;
}

int hj_shard_route(const hj_tuple_t *in_dev, size_t n, int nshards, hj_tuple_t *out_dev, uint64_t *counts_dev,
                   void *scratch_dev, size_t scratch_bytes, void *stream) {
    if (nshards < 1 || nshards > hj::kRouteMaxShards || !counts_dev || (n && (!in_dev || !out_dev))) return HJ_E_INVAL;
    if (scratch_bytes < hj_shard_route_scratch_bytes(n, nshards) || !scratch_dev) return HJ_E_INVAL;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return HJ_E_DEVICE;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned blocks = (unsigned)route_blocks(n, sms);
    char *p = reinterpret_cast<char *>(scratch_dev);
    uint32_t *blk_cnt = reinterpret_cast<uint32_t *>(p);
    unsigned long long *blk_off = reinterpret_cast<unsigned long long *>(p + a256((size_t)blocks * nshards * 4));
    unsigned int *err = reinterpret_cast<unsigned int *>(p + a256((size_t)blocks * nshards * 4) +
                                                         a256((size_t)blocks * nshards * 8));
    if (cudaMemsetAsync(err, 0, 4, st) != cudaSuccess) return HJ_E_DEVICE;
    if (n == 0) return cudaMemsetAsync(counts_dev, 0, sizeof(uint64_t) * nshards, st) == cudaSuccess ? HJ_OK : HJ_E_DEVICE;
    const hj::tuple_v *in = reinterpret_cast<const hj::tuple_v *>(in_dev);
    hj::route_count<<<blocks, hj::kRouteThreads, 0, st>>>(in, n, (unsigned)nshards, blk_cnt);
    hj::route_offsets<<<1, 1024, 0, st>>>(blk_cnt, blocks, (unsigned)nshards, blk_off,
                                          reinterpret_cast<unsigned long long *>(counts_dev));
    hj::route_scatter<<<blocks, hj::kRouteThreads, 0, st>>>(in, n, (unsigned)nshards, blk_off,
                                                            reinterpret_cast<hj::tuple_v *>(out_dev), err);
    return cudaGetLastError() == cudaSuccess ? HJ_OK : HJ_E_DEVICE;
}

}  // extern "C"
