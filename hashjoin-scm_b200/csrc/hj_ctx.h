// hj_ctx.h - the library context (hj_ctx_t), shared by the C ABI and the batch layer.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "../../include/hjscm.h"

namespace hj {
struct JoinAccum;
}

// A device-resident join as replayed from a CUDA graph: everything that its enqueued work depends on.
struct hj_graph_key {
    int algo = -1;
    const void *R = nullptr, *S = nullptr;
    size_t nR = 0, nS = 0;
    uint32_t flags = 0;
    int bits = 0, passes = 0, bits_pass1 = 0;
    double table_load = 0;
    bool seg = false;
    const char *arena = nullptr;
    size_t arena_bytes = 0;
    bool operator==(const hj_graph_key &o) const {
        return algo == o.algo && R == o.R && S == o.S && nR == o.nR && nS == o.nS && flags == o.flags &&
               bits == o.bits && passes == o.passes && bits_pass1 == o.bits_pass1 && table_load == o.table_load &&
               seg == o.seg && arena == o.arena && arena_bytes == o.arena_bytes;
    }
};

struct hj_graph_entry {
    hj_graph_key key;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;  // kernels in the graph
    uint64_t used = 0;      // last use (for eviction)
};

struct hj_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_h2d = nullptr, ev_start = nullptr, ev_mid = nullptr, ev_end = nullptr;
    cudaEvent_t ev_ret = nullptr;   // materialising joins: end of the retrieve phase
    cudaEvent_t ev_done = nullptr;  // watchdog: the result copy has landed
    cudaEvent_t ev_ph[HJ_PH_COUNT + 1] = {};
    char *arena = nullptr;
    size_t arena_bytes = 0;
    hj::JoinAccum *acc_host = nullptr;  // pinned
    hj_tuner_t tuner = {};              // autotuner state used by batches
    // Joins repeated on the same device buffers: the second consecutive identical call is captured into
    // a CUDA graph, later ones replay it (one launch instead of one per kernel, copy and event).
    std::vector<hj_graph_entry> graphs;
    hj_graph_key last_key;              // the previous join's key (a repeat triggers the capture)
    uint64_t graph_tick = 0;
    // phj_radix_lp: the last build relation whose unordered first run found a probe tuple with two
    // build matches; its next joins on this context run with ordered passes at once.
    const void *lp_ordered_R = nullptr;
    size_t lp_ordered_nR = 0;
    std::mutex mu;
};
