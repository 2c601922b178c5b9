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
//     one) with the named algorithm's result semantics, so its result is the same alone and in the mix;
//   - continuous batching: requests that run as non-partitioned joins (the small ones) do not take
//     slots. At each dispatch the queued ones are coalesced into a wave (hj_wave.cuh): one descriptor
//     copy, one multi-join build and one multi-join probe launch over all of them, on a high-priority
//     stream, with the wave's tables, descriptors and results in one block of the pool. Two wave lanes
//     let a wave be formed and launched while the previous one runs; requests that arrive meanwhile
//     join the next wave, so waves grow with the load and a request's cost is no longer a launch
//     sequence of its own.
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
#include "hj_wave.cuh"

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

// Continuous batching.
constexpr int kWaveLanes = 2;               // waves on the GPU at once
constexpr double kServerWaveTableBytes = 1e9;  // table bytes of one wave unless the config's tuner says
constexpr double kServerNphjTableBytes = 16e6; // largest non-partitioned table unless the config's tuner says
constexpr int kWaveMaxRequestsCap = 1024;   // the multi-join kernels stage count + 1 prefix sums in shared memory
constexpr unsigned kWaveMaxChunks = 1u << 15;  // build chunks (and probe chunks) of one wave

// Byte layout of one wave's pool block (every region 256-byte aligned):
//   [results: JoinAccum x n][descriptors: MJob x n | r_flat | s_flat | t_flat | build chunks | probe
//   chunks][side records: MSide x n][tables][device copies of host relations]
// The descriptor region is written into pinned host memory first and copied with one transfer.
struct WaveLayout {
    size_t desc_off, desc_bytes;
    size_t jobs_rel, rf_rel, sf_rel, tf_rel, rc_rel, sc_rel;  // offsets inside the descriptor region
    size_t sides_off, tables_off, copies_off, total;
    unsigned n_r_chunks, n_s_chunks;
    unsigned r_piece, s_piece;  // chunk lengths of the build and probe relations (mj_piece)
};

struct WaveLane {
    cudaStream_t stream = nullptr;  // high priority
    cudaEvent_t done = nullptr;
    char *stage = nullptr;            // pinned: the descriptor image of the wave in flight
    hj::JoinAccum *acc_host = nullptr;  // pinned: its results
    bool busy = false;
    std::vector<Request> reqs;
    WaveLayout lay;
    size_t off = 0;
    uint64_t wave_id = 0;
};

unsigned ceil_div(size_t a, unsigned b) { return (unsigned)((a + b - 1) / b); }

// Bytes of the descriptor region for n jobs with the given chunk counts (its largest value bounds the
// pinned staging buffer of a lane).
size_t wave_desc_bytes(size_t n, size_t nrc, size_t nsc, WaveLayout *L) {
    size_t o = 0;
    if (L) L->jobs_rel = o;
    o += a256(sizeof(hj::MJob) * n);
    if (L) L->rf_rel = o;
    o += a256(8 * (n + 1));
    if (L) L->sf_rel = o;
    o += a256(8 * (n + 1));
    if (L) L->tf_rel = o;
    o += a256(8 * (n + 1));
    if (L) L->rc_rel = o;
    o += a256(sizeof(hj::MChunk) * (nrc ? nrc : 1));
    if (L) L->sc_rel = o;
    o += a256(sizeof(hj::MChunk) * (nsc ? nsc : 1));
    return o;
}

void wave_layout(const std::vector<Request> &reqs, int num_sms, WaveLayout *L) {
    const size_t n = reqs.size();
    size_t nrc = 0, nsc = 0, table_bytes = 0, copy_bytes = 0;
    unsigned long long tr = 0, ts = 0;
    for (const Request &r : reqs) {
        tr += r.nR;
        ts += r.nS;
    }
    L->r_piece = hj::mj_piece(tr, hj::kBuildChunk, num_sms);
    L->s_piece = hj::mj_piece(ts, hj::kProbeChunkMJ, num_sms);
    for (const Request &r : reqs) {
        nrc += ceil_div(r.nR, L->r_piece);
        nsc += ceil_div(r.nS, L->s_piece);
        table_bytes += hj::mj_slots(r.nR) * 16;
        if (!r.on_device) copy_bytes += a256(r.nR * 16) + a256(r.nS * 16);
    }
    L->n_r_chunks = (unsigned)nrc;
    L->n_s_chunks = (unsigned)nsc;
    L->desc_off = a256(sizeof(hj::JoinAccum) * n);
    L->desc_bytes = wave_desc_bytes(n, nrc, nsc, L);
    L->sides_off = L->desc_off + L->desc_bytes;
    L->tables_off = L->sides_off + a256(sizeof(hj::MSide) * n);
    L->copies_off = L->tables_off + a256(table_bytes);
    L->total = L->copies_off + copy_bytes;
}

}  // namespace

struct hj_server {
    hj_server_config_t cfg;
    hj_ctx *ctx = nullptr;  // tuner and device properties
    char *pool_mem = nullptr;
    size_t pool_bytes = 0;
    Pool pool;
    std::vector<Slot> slots;
    WaveLane lanes[kWaveLanes];
    size_t stage_bytes = 0;
    uint64_t n_waves = 0, n_wave_requests = 0;
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

bool wave_eligible(const hj_server *s, const Request &r) { return s->cfg.waves && r.impl == 0 && r.nR && r.nS; }

// Requests above small_request_tuples run on low-priority streams with kernels sized for a share of the SMs.
bool is_large(const hj_server *s, const Request &r) { return (double)(r.nR + r.nS) > s->cfg.small_request_tuples; }

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
        if (wave_eligible(s, r)) {  // it will run in a wave: a wave of this request alone must fit
            WaveLayout lay;
            wave_layout(std::vector<Request>(1, r), s->ctx->num_sms, &lay);
            if (lay.total > need) need = lay.total;
        }
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

hj_server_completion_t make_completion(const Request &r, int status, const hj::JoinAccum *acc, double t) {
    hj_server_completion_t c;
    memset(&c, 0, sizeof(c));
    c.id = r.id;
    c.impl = r.impl;
    c.submit_s = r.submit_s;
    c.start_s = r.start_s;
    c.done_s = t;
    if (!status && acc) {
        c.matched_cnt = acc->matched;
        c.checksum = acc->checksum;
        const unsigned e = acc->error;
        status = e & hj::kErrSpinLimit ? HJ_E_TIMEOUT : e & hj::kErrProbeLimit ? HJ_E_PROBE_LIMIT : e ? HJ_E_OVERFLOW : 0;
    }
    c.status = status;
    return c;
}

// Record a finished request: its pool range and slot are returned in the same critical section that
// publishes the completion, so a caller that has polled every completion sees an idle server.
void complete(hj_server *s, Slot &sl, int status, const hj::JoinAccum *acc) {
    const hj_server_completion_t c = make_completion(sl.req, status, acc, now_s());
    std::lock_guard<std::mutex> lk(s->mu);
    s->pool.release(sl.req.off, sl.req.need);
    sl.busy = false;
    s->done.push_back(c);
    s->n_completed++;
    s->cv_done.notify_all();
}

// Record every request of a finished wave and return the wave's block and lane, in one critical section.
void complete_wave(hj_server *s, WaveLane &L, int status) {
    const double t = now_s();
    std::vector<hj_server_completion_t> cs;
    cs.reserve(L.reqs.size());
    for (size_t q = 0; q < L.reqs.size(); q++) {
        hj_server_completion_t c = make_completion(L.reqs[q], status, status ? nullptr : &L.acc_host[q], t);
        c.wave = L.wave_id;
        c.wave_size = (int)L.reqs.size();
        cs.push_back(c);
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->pool.release(L.off, L.lay.total);
    L.busy = false;
    L.reqs.clear();
    for (const hj_server_completion_t &c : cs) s->done.push_back(c);
    s->n_completed += cs.size();
    s->cv_done.notify_all();
}

// Enqueue one admitted wave on its lane's stream: host relations are copied into the block, the
// descriptor image (built here in the lane's pinned buffer) goes over in one copy, then the wave's
// kernels run and the results come back into pinned memory; nothing here waits for the device.
int launch_wave(hj_server *s, WaveLane &L) {
    const int n = (int)L.reqs.size();
    const WaveLayout &lay = L.lay;
    cudaStream_t st = L.stream;
    char *base = s->pool_mem + L.off;
    hj::JoinAccum *accs = reinterpret_cast<hj::JoinAccum *>(base);
    char *desc_dev = base + lay.desc_off;
    hj::MSide *sides = reinterpret_cast<hj::MSide *>(base + lay.sides_off);
    char *tp = base + lay.tables_off;
    char *cp = base + lay.copies_off;
    char *img = L.stage;
    hj::MJob *mj = reinterpret_cast<hj::MJob *>(img + lay.jobs_rel);
    unsigned long long *rf = reinterpret_cast<unsigned long long *>(img + lay.rf_rel);
    unsigned long long *sf = reinterpret_cast<unsigned long long *>(img + lay.sf_rel);
    unsigned long long *tf = reinterpret_cast<unsigned long long *>(img + lay.tf_rel);
    hj::MChunk *rc = reinterpret_cast<hj::MChunk *>(img + lay.rc_rel);
    hj::MChunk *sc = reinterpret_cast<hj::MChunk *>(img + lay.sc_rel);
    rf[0] = sf[0] = tf[0] = 0;
    unsigned nrc = 0, nsc = 0;
    bool any_lp = false;
    for (int q = 0; q < n; q++) {
        const Request &r = L.reqs[q];
        const hj::tuple_v *R = reinterpret_cast<const hj::tuple_v *>(r.R);
        const hj::tuple_v *S = reinterpret_cast<const hj::tuple_v *>(r.S);
        if (!r.on_device) {
            if (cudaMemcpyAsync(cp, r.R, r.nR * 16, cudaMemcpyHostToDevice, st) != cudaSuccess) return HJ_E_DEVICE;
            R = reinterpret_cast<const hj::tuple_v *>(cp);
            cp += a256(r.nR * 16);
            if (cudaMemcpyAsync(cp, r.S, r.nS * 16, cudaMemcpyHostToDevice, st) != cudaSuccess) return HJ_E_DEVICE;
            S = reinterpret_cast<const hj::tuple_v *>(cp);
            cp += a256(r.nS * 16);
        }
        hj::MJob &m = mj[q];
        m.R = R;
        m.S = S;
        m.nR = r.nR;
        m.nS = r.nS;
        m.cap = hj::mj_slots(r.nR);
        m.table = reinterpret_cast<hj::tuple_v *>(tp);
        tp += m.cap * 16;
        m.side = sides + q;
        m.acc = accs + q;
        m.lp = hj::algo_lp(r.algo) ? 1u : 0u;
        m.skip0 = hj::algo_skip0(r.algo) ? 1u : 0u;
        any_lp = any_lp || m.lp;
        for (size_t b = 0; b < r.nR; b += lay.r_piece, nrc++) {
            rc[nrc].job = (unsigned)q;
            rc[nrc].begin = b;
            rc[nrc].len = (unsigned)(r.nR - b < lay.r_piece ? r.nR - b : lay.r_piece);
        }
        for (size_t b = 0; b < r.nS; b += lay.s_piece, nsc++) {
            sc[nsc].job = (unsigned)q;
            sc[nsc].begin = b;
            sc[nsc].len = (unsigned)(r.nS - b < lay.s_piece ? r.nS - b : lay.s_piece);
        }
        rf[q + 1] = rf[q] + r.nR;
        sf[q + 1] = sf[q] + r.nS;
        tf[q + 1] = tf[q] + m.cap;
    }
    if (nrc != lay.n_r_chunks || nsc != lay.n_s_chunks) return HJ_E_INVAL;
    if (cudaMemcpyAsync(desc_dev, img, lay.desc_bytes, cudaMemcpyHostToDevice, st) != cudaSuccess) return HJ_E_DEVICE;
    if (cudaMemsetAsync(accs, 0, sizeof(hj::JoinAccum) * n, st) != cudaSuccess) return HJ_E_DEVICE;
    hj::WaveDev w;
    w.jobs = reinterpret_cast<const hj::MJob *>(desc_dev + lay.jobs_rel);
    w.count = n;
    w.r_chunks = reinterpret_cast<const hj::MChunk *>(desc_dev + lay.rc_rel);
    w.s_chunks = reinterpret_cast<const hj::MChunk *>(desc_dev + lay.sc_rel);
    w.n_r_chunks = (int)nrc;
    w.n_s_chunks = (int)nsc;
    w.r_flat = reinterpret_cast<const unsigned long long *>(desc_dev + lay.rf_rel);
    w.t_flat = reinterpret_cast<const unsigned long long *>(desc_dev + lay.tf_rel);
    w.total_r = rf[n];
    w.total_t = tf[n];
    w.any_lp = any_lp;
    w.tables = base + lay.tables_off;
    w.sides = sides;
    const int rcode = hj::mj_launch_wave(w, s->ctx->num_sms, st, nullptr);
    if (rcode) return rcode;
    if (cudaMemcpyAsync(L.acc_host, accs, sizeof(hj::JoinAccum) * n, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return HJ_E_DEVICE;
    if (cudaEventRecord(L.done, st) != cudaSuccess) return HJ_E_DEVICE;
    return HJ_OK;
}


void worker_main(hj_server *s) {
    cudaSetDevice(s->cfg.device);
    const int wave_max = s->cfg.wave_max_requests;
    const double wave_tables = s->ctx->tuner.wave_table_bytes > 0 ? s->ctx->tuner.wave_table_bytes : 64e6;
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
        for (WaveLane &L : s->lanes) {
            if (!L.busy) continue;
            const cudaError_t q = cudaEventQuery(L.done);
            if (q == cudaErrorNotReady) continue;
            complete_wave(s, L, q == cudaSuccess ? HJ_OK : HJ_E_DEVICE);
            progressed = true;
        }
        // 2. admission: slots for partitioned requests, one new wave for the non-partitioned ones
        std::vector<Slot *> to_launch;
        WaveLane *wave_lane = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            const double t = now_s();
            WaveLane *free_lane = nullptr;
            if (s->cfg.waves)
                for (WaveLane &L : s->lanes)
                    if (!L.busy) {
                        free_lane = &L;
                        break;
                    }
            std::vector<Request> wave;
            size_t w_nrc = 0, w_nsc = 0;
            double w_tables = 0;
            int scanned = 0;
            bool blocked_seen = false;
            int large_busy = 0;
            for (Slot &sl : s->slots) large_busy += sl.busy && is_large(s, sl.req);
            for (auto it = s->queue.begin(); it != s->queue.end() && scanned < kSkipAheadWindow;) {
                if (wave_eligible(s, *it)) {
                    if (free_lane && (int)wave.size() < wave_max) {
                        const size_t nrc = ceil_div(it->nR, hj::kBuildChunk), nsc = ceil_div(it->nS, hj::kProbeChunkMJ);
                        const double tb = (double)hj::mj_slots(it->nR) * 16.0;
                        if (w_nrc + nrc <= kWaveMaxChunks && w_nsc + nsc <= kWaveMaxChunks &&
                            (wave.empty() || w_tables + tb <= wave_tables)) {
                            wave.push_back(*it);
                            w_nrc += nrc;
                            w_nsc += nsc;
                            w_tables += tb;
                            ++it;
                            continue;
                        }
                    }
                    // It waits for the next wave (a free lane), not for memory that a slot request
                    // behind it could take: it neither blocks those nor counts toward the window.
                    ++it;
                    continue;
                } else if (s->cfg.max_large_inflight > 0 && is_large(s, *it) &&
                           large_busy >= s->cfg.max_large_inflight) {
                    // Waits for the large request on the GPU to finish; like a request waiting for a
                    // wave, it holds nothing back from the requests behind it.
                    ++it;
                    continue;
                } else {
                    Slot *free_slot = nullptr;
                    for (Slot &sl : s->slots)
                        if (!sl.busy) {
                            free_slot = &sl;
                            break;
                        }
                    size_t off = 0;
                    if (free_slot && s->pool.alloc(it->need, &off)) {
                        large_busy += is_large(s, *it);
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
                }
                // This request cannot start now. The oldest such request blocks everything behind it
                // once it has waited longer than the skip-ahead bound.
                if (!blocked_seen && t - it->submit_s > kSkipAheadSeconds) break;
                blocked_seen = true;
                ++it;
                scanned++;
            }
            if (!wave.empty()) {
                // The wave's block must fit the pool now; under memory pressure the wave shrinks (the
                // requests left out stay queued, in order).
                WaveLayout lay;
                wave_layout(wave, s->ctx->num_sms, &lay);
                size_t off = 0;
                bool got = false;
                for (;;) {
                    got = lay.desc_bytes <= s->stage_bytes && s->pool.alloc(lay.total, &off);
                    if (got || wave.size() == 1) break;
                    wave.resize(wave.size() / 2);
                    wave_layout(wave, s->ctx->num_sms, &lay);
                }
                if (got) {
                    // Take the wave's requests out of the queue (they are in queue order).
                    size_t k = 0;
                    for (auto it = s->queue.begin(); it != s->queue.end() && k < wave.size();) {
                        if (it->id == wave[k].id) {
                            it = s->queue.erase(it);
                            k++;
                        } else {
                            ++it;
                        }
                    }
                    for (Request &r : wave) r.start_s = t;
                    s->pending.fetch_sub((int)wave.size(), std::memory_order_release);
                    s->n_admitted += wave.size();
                    s->n_waves++;
                    s->n_wave_requests += wave.size();
                    free_lane->reqs.swap(wave);
                    free_lane->lay = lay;
                    free_lane->off = off;
                    free_lane->wave_id = s->n_waves;
                    free_lane->busy = true;
                    wave_lane = free_lane;
                }
            }
            if (to_launch.empty() && !wave_lane && !progressed) {
                bool any_busy = false;
                for (Slot &sl : s->slots) any_busy = any_busy || sl.busy;
                for (WaveLane &L : s->lanes) any_busy = any_busy || L.busy;
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
        if (wave_lane) {
            const int rc = launch_wave(s, *wave_lane);
            if (rc) {
                cudaStreamSynchronize(wave_lane->stream);
                complete_wave(s, *wave_lane, rc);
            }
        }
        for (Slot *sl : to_launch) {
            const int rc = launch(s, *sl);
            if (rc) {
                cudaStreamSynchronize(sl->cur);
                complete(s, *sl, rc, nullptr);
            }
        }
        if (to_launch.empty() && !wave_lane && !progressed) std::this_thread::yield();
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
    c->waves = 1;
    c->wave_max_requests = 512;
    c->max_large_inflight = 0;
    return HJ_OK;
}

int hj_server_create(const hj_server_config_t *cfg, hj_server_t **out) {
    if (!cfg || !out || cfg->slots < 1 || cfg->slots > 256 || !(cfg->hbm_budget_bytes > 0)) return HJ_E_INVAL;
    if (cfg->waves && (cfg->wave_max_requests < 1 || cfg->wave_max_requests > kWaveMaxRequestsCap)) return HJ_E_INVAL;
    if (cfg->max_large_inflight < 0) return HJ_E_INVAL;
    *out = nullptr;
    hj_server *s = new hj_server();
    s->cfg = *cfg;
    int rc = hj_ctx_create(cfg->device, &s->ctx);
    if (rc) {
        delete s;
        return rc;
    }
    if (cfg->tuner.partition_target > 0) {
        s->ctx->tuner = cfg->tuner;
    } else {
        // Waves of served requests are sized for throughput, not for L2: a request's table averages
        // ~16 MB on the served workload, so an L2-sized budget would cap waves at a few requests. Joins
        // whose table would exceed 16 MB run partitioned (on slots): the budget batches tune to.
        s->ctx->tuner.wave_table_bytes = kServerWaveTableBytes;
        s->ctx->tuner.nphj_max_table_bytes = kServerNphjTableBytes;
    }
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
    if (cfg->waves) {
        s->stage_bytes = wave_desc_bytes((size_t)cfg->wave_max_requests, kWaveMaxChunks, kWaveMaxChunks, nullptr);
        for (WaveLane &L : s->lanes) {
            if (cudaStreamCreateWithPriority(&L.stream, cudaStreamNonBlocking, prio_hi) != cudaSuccess ||
                cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming) != cudaSuccess ||
                cudaMallocHost(&L.stage, s->stage_bytes) != cudaSuccess ||
                cudaMallocHost(&L.acc_host, sizeof(hj::JoinAccum) * cfg->wave_max_requests) != cudaSuccess) {
                if (prev >= 0) cudaSetDevice(prev);
                hj_server_destroy(s);
                return HJ_E_DEVICE;
            }
            L.reqs.reserve(cfg->wave_max_requests);
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
    for (WaveLane &L : s->lanes) out->inflight += L.busy ? (int)L.reqs.size() : 0;
    out->waves = s->n_waves;
    out->wave_requests = s->n_wave_requests;
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
    for (WaveLane &L : s->lanes) {
        if (L.stream) cudaStreamSynchronize(L.stream);
        if (L.done) cudaEventDestroy(L.done);
        if (L.stage) cudaFreeHost(L.stage);
        if (L.acc_host) cudaFreeHost(L.acc_host);
        if (L.stream) cudaStreamDestroy(L.stream);
    }
    if (s->pool_mem) cudaFree(s->pool_mem);
    if (s->ctx) hj_ctx_destroy(s->ctx);
    if (prev >= 0) cudaSetDevice(prev);
    delete s;
    return HJ_OK;
}

}  // extern "C"
