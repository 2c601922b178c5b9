// hj_stream.cu - joins whose probe side is larger than the device memory hj_join needs.
//
// hj_join keeps both relations and two partition buffers in HBM (about 48 B per tuple for a two-pass
// radix join), so it stops at roughly a third of the device's memory. The reference's billion-scale
// workloads (2^30 x 2^34 tuples, 272 GB) exceed that many times over. A streamed join keeps the build
// relation R on the device and streams the probe relation S from host memory in chunks through two
// device buffers: the copy of chunk k+1 (its own stream) overlaps the join of chunk k. Every chunk is
// joined with all of R by the ordinary pipeline and the counts and checksums add up, so the result is
// hj_join's: every-match joins sum over chunks, and first-match joins pick per probe tuple the first R
// tuple in input order, which does not depend on how S is cut. Non-partitioned joins build their table
// from R once and only probe it per chunk.
//
// The overlap needs S in pinned (page-locked) host memory: cudaHostAlloc'd, or registered once by the
// caller with cudaHostRegister. From pageable memory the driver stages each chunk's copy through its own
// pinned buffers and the copies no longer run beside the joins (the result is the same). The join does
// not register S itself: pinning tens of GB takes longer than the copies it would speed up.
#include <chrono>
#include <cstdio>
#include <cstring>

#include "hj_common.cuh"
#include "hj_ctx.h"
#include "hj_internal.h"

namespace {

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

size_t stream_need(hj_algo_t algo, const hj_params_t &p, const hj::RadixGeom &g, size_t nR, size_t chunk,
                   int num_sms) {
    size_t need = 256 + a256(nR * 16) + 2 * a256(chunk * 16);
    if (hj::algo_is_phj(algo))
        need += hj::phj_scratch_bytes(g, nR, chunk, num_sms);
    else
        need += a256(hj::nphj_scratch_bytes(nR, p.table_load));
    return need;
}

}  // namespace

extern "C" int hj_join_streamed(hj_ctx_t *c, hj_algo_t algo, const hj_params_t *pin, const hj_tuple_t *R,
                                size_t nR, const hj_tuple_t *S, size_t nS, size_t chunk_tuples, hj_result_t *out) {
    if (!c || !out || (int)algo < 0 || algo >= HJ_ALGO_COUNT) return HJ_E_INVAL;
    memset(out, 0, sizeof(*out));
    if ((nR && !R) || (nS && !S)) return out->status = HJ_E_INVAL;
    if (nR >= (1ull << 32)) return out->status = HJ_E_INVAL;
    hj_params_t p;
    hj_params_init(&p);
    if (pin) p = *pin;
    if (p.num_radix_bits == 0) p.num_radix_bits = 14;
    if (p.num_passes == 0) p.num_passes = 2;
    if (!(p.table_load > 0.0)) p.table_load = 0.0;  // the size-dependent default
    if (p.device != c->device || p.inputs_on_device) return out->status = HJ_E_INVAL;  // host relations only
    hj::RadixGeom g = {};
    if (hj::algo_is_phj(algo)) {
        const int rc = hj::radix_geom(p.num_radix_bits, p.num_passes, &g, p.radix_bits_pass1);
        if (rc) return out->status = rc;
        out->physical_passes = g.passes;
    }
    if (nR == 0 || nS == 0) return out->status = HJ_OK;

    int dev_prev = -1;
    cudaGetDevice(&dev_prev);
    cudaSetDevice(c->device);
    struct Restore {
        int d;
        ~Restore() {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{dev_prev};
    std::lock_guard<std::mutex> lk(c->mu);

    // Chunk size: as asked, else the largest that fits the free memory (beyond the context's arena)
    // with R, two staging buffers and the pipeline's scratch, capped below 2^32 tuples.
    size_t chunk = chunk_tuples ? chunk_tuples : nS;
    if (chunk >= (1ull << 32)) chunk = (1ull << 32) - 1;
    if (!chunk_tuples) {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t avail = (size_t)(0.9 * (double)(free_b + c->arena_bytes));
        while (chunk > (1u << 20) && stream_need(algo, p, g, nR, chunk, c->num_sms) > avail) chunk /= 2;
    }
    if (chunk > nS) chunk = nS;
    const size_t need = stream_need(algo, p, g, nR, chunk, c->num_sms);
    if (c->arena_bytes < need) {
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) return out->status = HJ_E_DEVICE;
        if (c->arena) cudaFree(c->arena);
        c->arena = nullptr;
        c->arena_bytes = 0;
        if (cudaMalloc(&c->arena, need) != cudaSuccess) {
            cudaGetLastError();
            c->arena = nullptr;
            return out->status = HJ_E_OOM;
        }
        c->arena_bytes = need;
    }
    char *cur = c->arena;
    hj::JoinAccum *acc = reinterpret_cast<hj::JoinAccum *>(cur);
    cur += 256;
    ulonglong2 *dR = reinterpret_cast<ulonglong2 *>(cur);
    cur += a256(nR * 16);
    ulonglong2 *buf[2];
    buf[0] = reinterpret_cast<ulonglong2 *>(cur);
    cur += a256(chunk * 16);
    buf[1] = reinterpret_cast<ulonglong2 *>(cur);
    cur += a256(chunk * 16);
    char *scratch = cur;

    cudaStream_t st = c->stream, cs = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr}, t0 = nullptr, t1 = nullptr;
    int rc = HJ_OK;
    auto cleanup = [&]() {
        if (cs) cudaStreamSynchronize(cs);
        cudaStreamSynchronize(st);
        for (int b = 0; b < 2; b++) {
            if (copied[b]) cudaEventDestroy(copied[b]);
            if (consumed[b]) cudaEventDestroy(consumed[b]);
        }
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        if (cs) cudaStreamDestroy(cs);
    };
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&t0) != cudaSuccess ||
        cudaEventCreate(&t1) != cudaSuccess) {
        cleanup();
        return out->status = HJ_E_DEVICE;
    }
    for (int b = 0; b < 2; b++)
        if (cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&consumed[b], cudaEventDisableTiming) != cudaSuccess) {
            cleanup();
            return out->status = HJ_E_DEVICE;
        }
    // A join that a watchdog gave up on may still use the arena.
    cudaStreamWaitEvent(st, c->ev_done, 0);
    cudaEventRecord(t0, st);
    cudaMemsetAsync(acc, 0, sizeof(hj::JoinAccum), st);
    cudaMemcpyAsync(dR, R, nR * 16, cudaMemcpyHostToDevice, st);
    cudaEventRecord(consumed[0], st);  // the staging buffers are free once R is in
    cudaEventRecord(consumed[1], st);
    const size_t nchunks = (nS + chunk - 1) / chunk;
    uint32_t launches = 0;
    const bool nphj = !hj::algo_is_phj(algo);
    const size_t table_bytes = c->arena_bytes - (size_t)(scratch - c->arena);
    if (nphj) {
        // The table is built once, from R alone, while the first chunk is copied.
        uint32_t l = 0;
        rc = hj::nphj_enqueue(hj::algo_lp(algo), false, dR, nR, nullptr, 0, scratch, table_bytes, p.table_load, acc,
                              st, nullptr, c->num_sms, nullptr, &l, nullptr, hj::kNphjBuild);
        launches += l;
    }
    for (size_t k = 0; k < nchunks && !rc; k++) {
        const int b = (int)(k & 1);
        const size_t lo = k * chunk, len = nS - lo < chunk ? nS - lo : chunk;
        // copy stream: wait until the buffer's previous chunk has been joined, then fill it
        if (cudaStreamWaitEvent(cs, consumed[b], 0) != cudaSuccess ||
            cudaMemcpyAsync(buf[b], S + lo, len * 16, cudaMemcpyHostToDevice, cs) != cudaSuccess ||
            cudaEventRecord(copied[b], cs) != cudaSuccess) {
            rc = HJ_E_DEVICE;
            break;
        }
        // compute stream: join the chunk with all of R, into the same accumulators
        if (cudaStreamWaitEvent(st, copied[b], 0) != cudaSuccess) {
            rc = HJ_E_DEVICE;
            break;
        }
        uint32_t l = 0;
        if (hj::algo_is_phj(algo)) {
            hj::PhjScratch s;
            hj::phj_carve(g, nR, len, c->num_sms, scratch, &s);
            rc = hj::phj_enqueue(g, hj::algo_lp(algo), hj::algo_skip0(algo), dR, nR, buf[b], len, s, acc, st,
                                 nullptr, c->num_sms, nullptr, &l);
        } else {
            rc = hj::nphj_enqueue(hj::algo_lp(algo), false, dR, nR, buf[b], len, scratch, table_bytes, p.table_load,
                                  acc, st, nullptr, c->num_sms, nullptr, &l, nullptr, hj::kNphjProbe);
        }
        launches += l;
        if (!rc && cudaEventRecord(consumed[b], st) != cudaSuccess) rc = HJ_E_DEVICE;
    }
    cudaEventRecord(t1, st);
    cudaMemcpyAsync(c->acc_host, acc, sizeof(hj::JoinAccum), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess && !rc) rc = HJ_E_DEVICE;
    if (!rc) {
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        out->total = ms * 1e-3;  // copies included: the chunks' copies and joins overlap
        out->matched_cnt = c->acc_host->matched;
        out->checksum = c->acc_host->checksum;
        out->large_partitions = c->acc_host->large_parts;
        out->kernel_launches = launches;
        const unsigned e = c->acc_host->error;
        rc = !e ? HJ_OK : e & hj::kErrSpinLimit ? HJ_E_TIMEOUT : e & hj::kErrProbeLimit ? HJ_E_PROBE_LIMIT : HJ_E_OVERFLOW;
    }
    cleanup();
    return out->status = rc;
}
