// hj_noalloc.cu - a non-partitioned join that allocates nothing.
//
// Some callers cannot allocate device memory: a host engine that has already reserved the GPU's memory
// for its own buffer pool and forbids other allocations, or a tight request loop that must not call the
// CUDA allocator (cudaMalloc and cudaFree synchronise the device and their latency is unbounded). For
// them hj_nphj_join_noalloc runs nphj_sc / nphj_lp with its hash table in a fixed device array that is
// part of the library image, so the only memory it touches besides the caller's inputs and output is
// that array.
//
// The array holds kNoallocSlots table slots (16 bytes each) plus the join's side record; every GPU that
// loads the library keeps it until the process exits. All calls share it and it keeps the last call's
// contents, so each call clears what must start empty (table, side record, result) on its stream, and
// calls whose work overlaps on the GPU (different streams, or different host threads) race.
#include <cuda.h>

#include <cstdio>
#include <mutex>

#include "hj_common.cuh"
#include "hj_internal.h"

namespace {

constexpr unsigned long long kNoallocSlots = 1ull << 20;                  // table slots (16 MiB)
constexpr unsigned long long kNoallocSide = 256;                          // side record after the slots
constexpr unsigned long long kNoallocBytes = kNoallocSlots * 16 + kNoallocSide;
constexpr double kNoallocLoad = 0.5;                                      // table load factor
// Largest build relation: the table must hold |R| / load slots (see nphj_scratch_bytes).
constexpr unsigned long long kNoallocMaxBuild = (unsigned long long)(kNoallocSlots * kNoallocLoad) - 2;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocBytes];

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[64] = {};
int g_noalloc_sms[64] = {};
unsigned long long g_noalloc_ctx[64] = {};

// Process-unique id of the CUDA context current on this thread (0 when none is current yet). The
// driver's entry points are fetched through the runtime, so the library needs no link to libcuda.
unsigned long long current_context_id() {
    using get_current_fn = CUresult (*)(CUcontext *);
    using get_id_fn = CUresult (*)(CUcontext, unsigned long long *);
    static get_current_fn get_current = nullptr;
    static get_id_fn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", reinterpret_cast<void **>(&get_current), cudaEnableDefault,
                                    &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
            get_current = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", reinterpret_cast<void **>(&get_id), cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess)
            get_id = nullptr;
        cudaGetLastError();
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch array on the current device. The name of the array in host code is
// only a host-side stand-in; kernels must be given this address instead. It is looked up on the first
// call per device and again whenever the device's context changed since (a cudaDeviceReset, or a new
// primary context, reloads the library's module, and the array may then sit elsewhere).
int noalloc_setup(int dev, void **ptr, int *sms) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    unsigned long long ctx = current_context_id();
    if (!g_noalloc_ptr[dev] || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // makes the device's context current
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "hj_nphj_join_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            cudaGetLastError();
            return HJ_E_DEVICE;
        }
        int n = 0;
        e = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return HJ_E_DEVICE;
        g_noalloc_ptr[dev] = p;
        g_noalloc_sms[dev] = n;
        g_noalloc_ctx[dev] = current_context_id();
    }
    *ptr = g_noalloc_ptr[dev];
    *sms = g_noalloc_sms[dev];
    return HJ_OK;
}

}  // namespace

static_assert(sizeof(hj_device_result_t) == sizeof(hj::JoinAccum), "device result mirrors the accumulator");

extern "C" int hj_nphj_join_noalloc(hj_algo_t algo, const hj_tuple_t *R_dev, size_t nR, const hj_tuple_t *S_dev,
                                    size_t nS, hj_device_result_t *out_dev, void *stream) {
    if (algo != HJ_ALGO_NPHJ_SC && algo != HJ_ALGO_NPHJ_LP) return HJ_E_INVAL;
    if (!out_dev || (nR && !R_dev) || (nS && !S_dev)) return HJ_E_INVAL;
    if (nR > kNoallocMaxBuild) {
        fprintf(stderr,
                "hj_nphj_join_noalloc: the build relation has %zu tuples; this entry point's fixed table "
                "holds at most %llu (use hj_join for larger joins)\n",
                nR, (unsigned long long)kNoallocMaxBuild);
        return HJ_E_INVAL;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HJ_E_DEVICE;
    void *scratch = nullptr;
    int sms = 0;
    int rc = noalloc_setup(dev, &scratch, &sms);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // The result starts at zero; the table and the side record are cleared by the join itself.
    if (cudaMemsetAsync(out_dev, 0, sizeof(hj_device_result_t), st) != cudaSuccess) return HJ_E_DEVICE;
    if (nR == 0 || nS == 0) return HJ_OK;
    return hj::nphj_enqueue(algo == HJ_ALGO_NPHJ_LP, false, reinterpret_cast<const ulonglong2 *>(R_dev), nR,
                            reinterpret_cast<const ulonglong2 *>(S_dev), nS, scratch, kNoallocBytes, kNoallocLoad,
                            reinterpret_cast<hj::JoinAccum *>(out_dev), st, nullptr, sms, nullptr, nullptr);
}
