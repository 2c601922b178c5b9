// hj_server.cu - a join server: requests arrive at any time, are admitted under an HBM budget as
// execution slots and memory free up, and run concurrently on the device.
//
// The reference has no serving mode (one join per process, src/main.c:429-448). Here:
//   - one device memory pool of the configured budget is allocated at creation; every admitted request
//     takes its scratch (and, for host inputs, the copies of its relations) from the pool with a
//     first-fit allocator and returns it on completion, so the server never calls the CUDA allocator
//     while serving;
//   - `slots` requests run at once, each on its own CUDA stream, so a request that arrives while others
//     are on the GPU is admitted as soon as a slot and its memory are free and its kernels overlap with
//     theirs; small requests run on high-priority streams, so their thread blocks are scheduled ahead of
//     the waiting blocks of a large join and their latency stays near their own run time;
//   - large requests size their persistent kernels for a share of the SMs (large_sm_share, 0.75 by
//     default), so the blocks of small requests find free SMs instead of waiting for a whole partition
//     pass of a large join to drain (stream priority orders pending blocks, it does not preempt);
//   - the dispatcher thread polls the slots' completion events without sleeping while any request is
//     on the GPU (a sleep of a few microseconds costs tens of microseconds of timer slack per request);
//   - admission is first come, first served, except that requests behind a head that does not fit yet
//     may go first while the head has waited less than a bound;
//   - each request runs the implementation the context's autotuner picks for its sizes (or the named
//     one) with the named algorithm's result semantics, so its result is the same alone and in the mix.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "hj_common.cuh"
#include "hj_ctx.h"
#include "hj_internal.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Request {
    uint64_t id;
    hj_algo_t algo;
    const hj_tuple_t *R, *S;
    size_t nR, nS;
    int on_device;
    int impl, bits, passes;
    size_t need;
    double submit_s, start_s;
    size_t off;
};

// First-fit allocator over [0, size) with coalescing of neighbours.
class Pool {
  public:
    void init(size_t size) {
        free_.clear();
        if (size) free_[0] = size;
        in_use_ = peak_ = 0;
    }
    bool alloc(size_t bytes, size_t *off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                const size_t rest = it->second - bytes;
                const size_t noff = it->first + bytes;
                free_.erase(it);
                if (rest) free_[noff] = rest;
                in_use_ += bytes;
                if (in_use_ > peak_) peak_ = in_use_;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        in_use_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t in_use() const { return in_use_; }
    size_t peak() const { return peak_; }

  private:
    std::map<size_t, size_t> free_;
    size_t in_use_ = 0, peak_ = 0;
};

struct Slot {
    cudaStream_t stream = nullptr;     // low priority: large requests
    cudaStream_t stream_hi = nullptr;  // high priority: small requests
    cudaStream_t cur = nullptr;        // the one the slot's request runs on
    cudaEvent_t done = nullptr;
    hj::JoinAccum *acc_host = nullptr;  // pinned
    bool busy = false;
    Request req;
};

constexpr double kSkipAheadSeconds = 0.05;  // a head that waited longer is not overtaken any more
constexpr int kSkipAheadWindow = 16;

}  // namespace

struct hj_server {
    hj_server_config_t cfg;
    hj_ctx *ctx = nullptr;  // tuner and device properties
    char *pool_mem = nullptr;
    size_t pool_bytes = 0;
    Pool pool;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_submit, cv_done;
    std::deque<Request> queue;
    std::atomic<int> pending{0};  // queued requests, readable without the lock
    std::deque<hj_server_completion_t> done;
    uint64_t next_id = 1, n_submitted = 0, n_admitted = 0, n_completed = 0;
    bool stop = false;
    std::thread worker;
};

namespace {

int request_need(hj_server *s, Request &r) {
    hj_params_t p;
    hj_params_init(&p);
    const bool phj_named = hj::algo_is_phj(r.algo);
    if (s->cfg.autotune) {
        hj_tuner_decide(s->ctx, r.nR, r.nS, &r.impl, &r.bits, &r.passes);
    } else {
        r.impl = phj_named ? 1 : 0;
        r.bits = 14;
        r.passes = 2;
    }
    size_t need = 256;
    if (!r.on_device) need += a256(r.nR * 16) + a256(r.nS * 16);
    if (r.impl == 0) {
        need += a256(hj::nphj_scratch_bytes(r.nR, 0.5));
    } else {
        hj::RadixGeom g;
        if (hj::radix_geom(r.bits, r.passes, &g)) return HJ_E_INVAL;
        need += hj::phj_scratch_bytes(g, r.nR, r.nS, s->ctx->num_sms);
    }
    r.need = a256(need);
    return HJ_OK;
}

// Enqueue one admitted request on a slot's stream; nothing here waits for the device.
int launch(hj_server *s, Slot &sl) {
    Request &r = sl.req;
    const bool small = (double)(r.nR + r.nS) <= s->cfg.small_request_tuples;
    cudaStream_t st = sl.cur = small ? sl.stream_hi : sl.stream;
    // Grids of a large request's persistent kernels scale with the SMs they are sized for.
    int sms = s->ctx->num_sms;
    if (!small && s->cfg.large_sm_share > 0.0 && s->cfg.large_sm_share < 1.0) {
        sms = (int)(s->ctx->num_sms * s->cfg.large_sm_share);
        if (sms < 1) sms = 1;
    }
    char *base = s->pool_mem + r.off;
    hj::JoinAccum *acc = reinterpret_cast<hj::JoinAccum *>(base);
    char *cur = base + 256;
    if (cudaMemsetAsync(acc, 0, sizeof(hj::JoinAccum), st) != cudaSuccess) return HJ_E_DEVICE;
    const ulonglong2 *R = reinterpret_cast<const ulonglong2 *>(r.R), *S = reinterpret_cast<const ulonglong2 *>(r.S);
    if (!r.on_device) {
        ulonglong2 *dr = reinterpret_cast<ulonglong2 *>(cur);
        cur += a256(r.nR * 16);
        ulonglong2 *ds = reinterpret_cast<ulonglong2 *>(cur);
        cur += a256(r.nS * 16);
        if (r.nR && cudaMemcpyAsync(dr, r.R, r.nR * 16, cudaMemcpyHostToDevice, st) != cudaSuccess) return HJ_E_DEVICE;
        if (r.nS && cudaMemcpyAsync(ds, r.S, r.nS * 16, cudaMemcpyHostToDevice, st) != cudaSuccess) return HJ_E_DEVICE;
        R = dr;
        S = ds;
    }
    const bool lp = hj::algo_lp(r.algo);
    const bool skip0 = hj::algo_skip0(r.algo);
    int rc = HJ_OK;
    if (r.nR && r.nS) {
        if (r.impl == 0) {
            const size_t tb = r.need - (size_t)(cur - base);
            rc = hj::nphj_enqueue(lp, skip0, R, r.nR, S, r.nS, cur, tb, 0.5, acc, st, nullptr, sms,
                                  nullptr, nullptr);
        } else {
            hj::RadixGeom g;
            hj::radix_geom(r.bits, r.passes, &g);
            hj::PhjScratch ps;
            hj::phj_carve(g, r.nR, r.nS, s->ctx->num_sms, cur, &ps);
            rc = hj::phj_enqueue(g, lp, skip0, R, r.nR, S, r.nS, ps, acc, st, nullptr, sms, nullptr,
                                 nullptr);
        }
    }
    if (rc) return rc;
    if (cudaMemcpyAsync(sl.acc_host, acc, sizeof(hj::JoinAccum), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return HJ_E_DEVICE;
    if (cudaEventRecord(sl.done, st) != cudaSuccess) return HJ_E_DEVICE;
    return HJ_OK;
}

// Record a finished request: its pool range and slot are returned in the same critical section that
// publishes the completion, so a caller that has polled every completion sees an idle server.
void complete(hj_server *s, Slot &sl, int status, const hj::JoinAccum *acc) {
    const Request &r = sl.req;
    hj_server_completion_t c;
    memset(&c, 0, sizeof(c));
    c.id = r.id;
    c.impl = r.impl;
    c.submit_s = r.submit_s;
    c.start_s = r.start_s;
    c.done_s = now_s();
    if (!status && acc) {
        c.matched_cnt = acc->matched;
        c.checksum = acc->checksum;
        const unsigned e = acc->error;
        status = e & hj::kErrSpinLimit ? HJ_E_TIMEOUT : e & hj::kErrProbeLimit ? HJ_E_PROBE_LIMIT : e ? HJ_E_OVERFLOW : 0;
    }
    c.status = status;
    std::lock_guard<std::mutex> lk(s->mu);
    s->pool.release(r.off, r.need);
    sl.busy = false;
    s->done.push_back(c);
    s->n_completed++;
    s->cv_done.notify_all();
}

void worker_main(hj_server *s) {
    cudaSetDevice(s->cfg.device);
    for (;;) {
        bool progressed = false;
        // 1. completions
        for (Slot &sl : s->slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaErrorNotReady) continue;
            complete(s, sl, q == cudaSuccess ? HJ_OK : HJ_E_DEVICE, sl.acc_host);
            progressed = true;
        }
        // 2. admission
        std::vector<Slot *> to_launch;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            const double t = now_s();
            int scanned = 0;
            for (auto it = s->queue.begin(); it != s->queue.end() && scanned < kSkipAheadWindow;) {
                Slot *free_slot = nullptr;
                for (Slot &sl : s->slots)
                    if (!sl.busy) {
                        free_slot = &sl;
                        break;
                    }
                if (!free_slot) break;
                size_t off = 0;
                if (s->pool.alloc(it->need, &off)) {
                    it->off = off;
                    it->start_s = t;
                    free_slot->req = *it;
                    free_slot->busy = true;
                    to_launch.push_back(free_slot);
                    it = s->queue.erase(it);
                    s->pending.fetch_sub(1, std::memory_order_release);
                    s->n_admitted++;
                    continue;
                }
                // The head does not fit yet: later requests may pass it only while it is young.
                if (it == s->queue.begin() && t - it->submit_s > kSkipAheadSeconds) break;
                ++it;
                scanned++;
            }
            if (to_launch.empty() && !progressed) {
                bool any_busy = false;
                for (Slot &sl : s->slots) any_busy = any_busy || sl.busy;
                if (s->stop && s->queue.empty() && !any_busy) return;
                if (!any_busy && s->queue.empty()) {
                    // Idle: spin briefly for the next submission, then block until one arrives.
                    lk.unlock();
                    const double t_spin = now_s() + 2e-4;
                    while (now_s() < t_spin && s->pending.load(std::memory_order_acquire) == 0)
                        std::this_thread::yield();
                    lk.lock();
                    if (s->queue.empty() && !s->stop)
                        s->cv_submit.wait_for(lk, std::chrono::milliseconds(2));
                }
            }
        }
        for (Slot *sl : to_launch) {
            const int rc = launch(s, *sl);
            if (rc) {
                cudaStreamSynchronize(sl->cur);
                complete(s, *sl, rc, nullptr);
            }
        }
        if (to_launch.empty() && !progressed) std::this_thread::yield();
    }
}

}  // namespace

extern "C" {

double hj_now(void) { return now_s(); }

int hj_server_config_init(hj_server_config_t *c) {
    if (!c) return HJ_E_INVAL;
    memset(c, 0, sizeof(*c));
    c->device = 0;
    c->slots = 8;
    c->hbm_budget_bytes = 150e9;
    c->autotune = 1;
    c->small_request_tuples = (double)(1u << 25);
    c->large_sm_share = 0.75;
    return HJ_OK;
}

int hj_server_create(const hj_server_config_t *cfg, hj_server_t **out) {
    if (!cfg || !out || cfg->slots < 1 || cfg->slots > 256 || !(cfg->hbm_budget_bytes > 0)) return HJ_E_INVAL;
    *out = nullptr;
    hj_server *s = new hj_server();
    s->cfg = *cfg;
    int rc = hj_ctx_create(cfg->device, &s->ctx);
    if (rc) {
        delete s;
        return rc;
    }
    if (cfg->tuner.partition_target > 0) s->ctx->tuner = cfg->tuner;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(cfg->device);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    size_t want = (size_t)cfg->hbm_budget_bytes;
    if (want > (size_t)(0.92 * (double)free_b)) want = (size_t)(0.92 * (double)free_b);
    want &= ~(size_t)255;
    if (cudaMalloc(&s->pool_mem, want) != cudaSuccess) {
        cudaGetLastError();
        hj_ctx_destroy(s->ctx);
        delete s;
        if (prev >= 0) cudaSetDevice(prev);
        return HJ_E_OOM;
    }
    s->pool_bytes = want;
    s->pool.init(want);
    hj::phj_prepare_device();
    int prio_lo = 0, prio_hi = 0;
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    s->slots.resize(cfg->slots);
    for (Slot &sl : s->slots) {
        if (cudaStreamCreateWithPriority(&sl.stream, cudaStreamNonBlocking, prio_lo) != cudaSuccess ||
            cudaStreamCreateWithPriority(&sl.stream_hi, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
            cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
            cudaMallocHost(&sl.acc_host, sizeof(hj::JoinAccum)) != cudaSuccess) {
            if (prev >= 0) cudaSetDevice(prev);
            hj_server_destroy(s);
            return HJ_E_DEVICE;
        }
    }
    s->worker = std::thread(worker_main, s);
    if (prev >= 0) cudaSetDevice(prev);
    *out = s;
    return HJ_OK;
}

int hj_server_submit(hj_server_t *s, hj_algo_t algo, const hj_tuple_t *R, size_t nR, const hj_tuple_t *S, size_t nS,
                     int inputs_on_device, uint64_t *id) {
    if (!s || (int)algo < 0 || algo >= HJ_ALGO_COUNT || (nR && !R) || (nS && !S)) return HJ_E_INVAL;
    if (nR >= (1ull << 32) || nS >= (1ull << 32)) return HJ_E_INVAL;
    Request r;
    memset(&r, 0, sizeof(r));
    r.algo = algo;
    r.R = R;
    r.S = S;
    r.nR = nR;
    r.nS = nS;
    r.on_device = inputs_on_device ? 1 : 0;
    r.submit_s = now_s();
    int rc = request_need(s, r);
    if (rc) return rc;
    if (r.need > s->pool_bytes) return HJ_E_BUDGET;
    std::lock_guard<std::mutex> lk(s->mu);
    r.id = s->next_id++;
    s->queue.push_back(r);
    s->pending.fetch_add(1, std::memory_order_release);
    s->n_submitted++;
    if (id) *id = r.id;
    s->cv_submit.notify_all();
    return HJ_OK;
}

int hj_server_poll(hj_server_t *s, hj_server_completion_t *out, int max, int *n, int wait_ms) {
    if (!s || !n || (max > 0 && !out)) return HJ_E_INVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return !s->done.empty(); });
    int k = 0;
    while (k < max && !s->done.empty()) {
        out[k++] = s->done.front();
        s->done.pop_front();
    }
    *n = k;
    return HJ_OK;
}

int hj_server_stats(hj_server_t *s, hj_server_stats_t *out) {
    if (!s || !out) return HJ_E_INVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    memset(out, 0, sizeof(*out));
    out->submitted = s->n_submitted;
    out->admitted = s->n_admitted;
    out->completed = s->n_completed;
    out->budget_bytes = (double)s->pool_bytes;
    out->in_use_bytes = (double)s->pool.in_use();
    out->peak_in_use_bytes = (double)s->pool.peak();
    out->queued = (int)s->queue.size();
    for (Slot &sl : s->slots) out->inflight += sl.busy;
    return HJ_OK;
}

int hj_server_destroy(hj_server_t *s) {
    if (!s) return HJ_E_INVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_submit.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(s->cfg.device);
    for (Slot &sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        if (sl.stream_hi) cudaStreamSynchronize(sl.stream_hi);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.acc_host) cudaFreeHost(sl.acc_host);
        if (sl.stream) cudaStreamDestroy(sl.stream);
        if (sl.stream_hi) cudaStreamDestroy(sl.stream_hi);
    }
    if (s->pool_mem) cudaFree(s->pool_mem);
    if (s->ctx) hj_ctx_destroy(s->ctx);
    if (prev >= 0) cudaSetDevice(prev);
    delete s;
    return HJ_OK;
}

}  // extern "C"
