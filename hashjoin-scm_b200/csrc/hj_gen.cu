// hj_gen.cu - parallel relation generators on the device (same bytes as hj_gen_fast_host).
#include <cmath>
#include <cstdio>
#include <vector>

#include "../host/hj_feistel.h"
#include "hj_common.cuh"

namespace {

__global__ void gen_fast_kernel(hj_feistel_t fr, hj_feistel_t fs, uint64_t distinct, int payload,
                                ulonglong2 *R, uint64_t nR, ulonglong2 *S, uint64_t nS) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nR; i += stride) {
        unsigned long long k, r;
        hj_fast_r_tuple(&fr, distinct, payload, i, (uint64_t *)&k, (uint64_t *)&r);
        R[i] = make_ulonglong2(k, r);
    }
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nS; j += stride) {
        unsigned long long k, r;
        hj_fast_s_tuple(&fs, distinct, payload, j, (uint64_t *)&k, (uint64_t *)&r);
        S[j] = make_ulonglong2(k, r);
    }
}

// Zipf sampling with the gen_zipf rule (src/inc/eth_genzipf.c:97-147) on a counter-based uniform
// stream: u = (mix64(seed, j) >> 11) * 2^-53 in [0, 1).
__global__ void gen_zipf_kernel(const double *lut, const uint64_t *alphabet, uint64_t n, uint64_t seed,
                                ulonglong2 *S, uint64_t nS) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nS; j += stride) {
        const double r = (double)(hj_mix64(seed + 0x9e3779b97f4a7c15ull * (j + 1)) >> 11) * 0x1.0p-53;
        uint64_t pos;
        if (lut[0] >= r) {
            pos = 0;
        } else {
            uint64_t left = 1, right = n;
            while (right - left > 1) {
                const uint64_t m = (left + right) / 2;
                if (lut[m] < r) left = m; else right = m;
            }
            pos = right < n ? right : n - 1;
        }
        S[j] = make_ulonglong2(alphabet[pos], j + 1);
    }
}

}  // namespace

extern "C" int hj_gen_fast_device(size_t nR, size_t nS, uint64_t seed, int payload, unsigned dup,
                                  hj_tuple_t *R_dev, hj_tuple_t *S_dev, void *stream) {
    if (nR == 0 || !R_dev || (nS && !S_dev)) return HJ_E_INVAL;
    if (dup == 0) dup = 1;
    hj_feistel_t fr, fs;
    hj_feistel_init(&fr, nR, HJ_GEN_SEED_R(seed));
    hj_feistel_init(&fs, nS ? nS : 1, HJ_GEN_SEED_S(seed));
    const uint64_t distinct = (nR + dup - 1) / dup;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    gen_fast_kernel<<<sms * 8, 256, 0, (cudaStream_t)stream>>>(
        fr, fs, distinct, dup > 1 ? 1 : payload, reinterpret_cast<ulonglong2 *>(R_dev), nR,
        reinterpret_cast<ulonglong2 *>(S_dev), nS);
    if (cudaGetLastError() != cudaSuccess) return HJ_E_DEVICE;
    return HJ_OK;
}

extern "C" int hj_gen_zipf_device(size_t nS, size_t nR, double zipf_factor, uint64_t seed,
                                  hj_tuple_t *S_dev, void *stream) {
    if (nR == 0 || !S_dev) return HJ_E_INVAL;
    // Alphabet: a seeded permutation of 1..nR; CDF table exactly as gen_zipf_lut
    // (src/inc/eth_genzipf.c:61-91).
    std::vector<uint64_t> alphabet(nR);
    std::vector<double> lut(nR);
    hj_feistel_t fa;
    hj_feistel_init(&fa, nR, seed ^ 0xa1fa0000ull);
    for (size_t i = 0; i < nR; i++) alphabet[i] = hj_feistel_perm(&fa, i) + 1;
    double scale = 0.0;
    for (size_t i = 1; i <= nR; i++) scale += 1.0 / pow((double)i, zipf_factor);
    double sum = 0.0;
    for (size_t i = 1; i <= nR; i++) {
        sum += 1.0 / pow((double)i, zipf_factor);
        lut[i - 1] = sum / scale;
    }
    cudaStream_t st = (cudaStream_t)stream;
    double *dlut = nullptr;
    uint64_t *dalpha = nullptr;
    if (cudaMalloc(&dlut, nR * sizeof(double)) != cudaSuccess) return HJ_E_OOM;
    if (cudaMalloc(&dalpha, nR * sizeof(uint64_t)) != cudaSuccess) {
        cudaFree(dlut);
        return HJ_E_OOM;
    }
    cudaMemcpyAsync(dlut, lut.data(), nR * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dalpha, alphabet.data(), nR * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    gen_zipf_kernel<<<sms * 8, 256, 0, st>>>(dlut, dalpha, nR, seed, reinterpret_cast<ulonglong2 *>(S_dev), nS);
    int rc = cudaGetLastError() == cudaSuccess ? HJ_OK : HJ_E_DEVICE;
    cudaStreamSynchronize(st);
    cudaFree(dlut);
    cudaFree(dalpha);
    return rc;
}
