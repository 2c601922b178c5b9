// hj_wave.cuh - waves of non-partitioned joins.
//
// A wave runs many independent joins, each with its own global hash table, with one multi-join build
// kernel and one multi-join probe kernel over flat lists of (join, range) chunks, so the launch count
// does not grow with the number of joins. Batches (hj_batch.cu) pack their small joins into waves at
// plan time; the join server (hj_server.cu) forms a wave from the small requests queued at each
// dispatch (continuous batching).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "hj_common.cuh"

namespace hj {

struct MSide {
    unsigned long long cnt, sum;  // build tuples whose key is the empty pattern: count, row-id sum
    unsigned long long notpos;    // max of ~position over them (0 = none), i.e. ~(smallest position)
    unsigned int dup;             // an equal key was inserted twice
    unsigned int pad;
};

struct MJob {
    const tuple_v *R, *S;
    unsigned long long nR, nS;
    tuple_v *table;
    unsigned long long cap;
    MSide *side;
    JoinAccum *acc;
    unsigned int lp, skip0;
};

// A piece of one job's build or probe side: the multi-join kernels take these as work items, so a
// block always works on a single job.
struct MChunk {
    unsigned int job;
    unsigned int len;
    unsigned long long begin;
};

constexpr unsigned kBuildChunk = 8192, kProbeChunkMJ = 16384;

// Chunk length for `total` tuples of a wave: the fixed piece, or a smaller one (a multiple of 256, at
// least 256) when the wave is too small to give every SM four chunks; a lone small request would
// otherwise run on a handful of CTAs, each working through thousands of dependent table accesses.
inline unsigned mj_piece(unsigned long long total, unsigned max_piece, int num_sms) {
    const unsigned long long want = (unsigned long long)(num_sms > 0 ? num_sms : 148) * 4;
    unsigned long long p = (total + want - 1) / want;
    p = (p + 255) / 256 * 256;
    return p < 256 ? 256u : p > max_piece ? max_piece : (unsigned)p;
}

// Table slots of one job (load factor 0.5, two spare slots).
inline unsigned long long mj_slots(size_t nR) { return (unsigned long long)((double)nR / 0.5) + 2; }

// Device view of one wave: descriptors, prefix sums of build / probe / table sizes over the jobs (count
// + 1 entries each), and the tables and side records the wave clears before building.
struct WaveDev {
    const MJob *jobs;
    int count;
    const MChunk *r_chunks, *s_chunks;
    int n_r_chunks, n_s_chunks;
    const unsigned long long *r_flat, *t_flat;
    unsigned long long total_r, total_t;
    bool any_lp;
    void *tables;
    MSide *sides;
};

// Enqueue a wave on `st`: clear its tables and side records, build, resolve first-match joins with
// duplicate build keys, probe. Results accumulate into each job's JoinAccum (which the caller zeroes).
int mj_launch_wave(const WaveDev &w, int num_sms, cudaStream_t st, uint32_t *launches);

}  // namespace hj
