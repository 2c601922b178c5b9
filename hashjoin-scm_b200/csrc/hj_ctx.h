// hj_ctx.h - the library context (hj_ctx_t), shared by the C ABI and the batch layer.
#pragma once

#include <cuda_runtime.h>

#include <mutex>

#include "../../include/hjscm.h"

namespace hj {
struct JoinAccum;
}

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
    std::mutex mu;
};
