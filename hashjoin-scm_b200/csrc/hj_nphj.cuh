// hj_nphj.cuh - probe side of the global open-addressing table, shared by the single-join kernels
// (hj_nphj.cu) and the multi-join kernels of batches (hj_batch.cu).
#pragma once

#include "hj_common.cuh"

namespace hj {

constexpr unsigned long long kTableEmpty = ~0ull;

// Read-only 16-byte load of a table slot: the table was finished by an earlier kernel.
__device__ __forceinline__ tuple_v ld_slot(const tuple_v *p) {
    tuple_v v;
    asm volatile("ld.global.nc.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}

// Read-only 8-byte load of a compact table slot.
__device__ __forceinline__ unsigned long long ld_slot8(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.global.nc.u64 %0, [%1];" : "=l"(v) : "l"(p));
    return v;
}

struct ProbeArgs {
    const tuple_v *table;
    unsigned long long cap;
    bool first_only;     // stop at the first equal key (lp semantics, or no duplicate build keys)
    bool lp;             // one match per probe tuple
    bool skip0;          // key 0 never matches
    unsigned long long side_cnt, side_sum;  // build tuples with the empty-pattern key
    unsigned long long side_first_rid;      // row id of the first of them (lp)
    unsigned int *err;
};

// Probe U tuples whose loads were issued together: the first table slot of every tuple is requested
// before any of them is examined, so U random L2 accesses are in flight per thread.
template <int U>
__device__ __forceinline__ void probe_group(const ProbeArgs &P, const tuple_v (&s)[U], const bool (&valid)[U],
                                            unsigned long long &cnt, unsigned long long &sum) {
    unsigned long long h[U];
    tuple_v e[U];
    bool walk[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
        walk[u] = valid[u] && s[u].x != kTableEmpty && !(P.skip0 && s[u].x == 0);
        if (walk[u]) {
            h[u] = table_hash(s[u].x, P.cap);
            e[u] = ld_slot(P.table + h[u]);
        }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
        if (valid[u] && s[u].x == kTableEmpty) {
            if (P.side_cnt) {
                if (P.lp) {
                    cnt++;
                    sum += P.side_first_rid + s[u].y;
                } else {
                    cnt += P.side_cnt;
                    sum += P.side_sum + P.side_cnt * s[u].y;
                }
            }
            continue;
        }
        if (!walk[u]) continue;
        unsigned long long hh = h[u];
        tuple_v ee = e[u];
        for (unsigned long long steps = 0;;) {
            if (ee.x == kTableEmpty) break;
            if (ee.x == s[u].x) {
                cnt++;
                sum += ee.y + s[u].y;
                if (P.first_only) break;
            }
            if (++hh == P.cap) hh = 0;
            if (++steps >= P.cap) {
                set_error(P.err, kErrProbeLimit);
                break;
            }
            ee = ld_slot(P.table + hh);
        }
    }
}

}  // namespace hj
