// hj_api.cu - the C ABI: contexts, scratch arena, and the synchronous join entry points.
//
// The reference's join_init_run (src/algo/phj.c:1875-2512) and nphj_sc/nphj_lp
// (src/algo/nphj.c:677-1037, 1487-...) each allocate their buffers, spawn thread pools, join and free
// everything per call. Here a context keeps a stream, events and a grow-only device arena; a join
// carves its scratch out of the arena and enqueues the whole kernel pipeline on one stream, reading
// back only the 64-byte accumulator at the end.
#include <cstdio>
#include <chrono>
#include <cstring>
#include <thread>
#include <mutex>

#include "hj_common.cuh"
#include "hj_ctx.h"
#include "hj_internal.h"

using hj::JoinAccum;

#define CU_OR(call, code)                                                                   \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            fprintf(stderr, "hjscm: %s failed: %s\n", #call, cudaGetErrorString(e_));       \
            return (code);                                                                  \
        }                                                                                   \
    } while (0)

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

std::mutex g_default_mu;
hj_ctx *g_default[64] = {};

constexpr size_t kAccBytes = 256;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

void resolve_params(const hj_params_t *p, hj_params_t *out) {
    hj_params_init(out);
    if (p) *out = *p;
    if (out->num_radix_bits == 0) out->num_radix_bits = 14;
    if (out->num_passes == 0) out->num_passes = 2;
    if (!(out->table_load > 0.0)) out->table_load = 0.0;  // the size-dependent default (nphj_default_load)
}

bool is_phj(hj_algo_t a) { return hj::algo_is_phj(a); }

// Segment mode for a radix join (see HJ_F_SEGMENTS): by size unless a flag decides.
bool want_seg(hj_algo_t algo, const hj_params_t &p, const hj::RadixGeom &g, size_t nR, size_t nS) {
    if (!is_phj(algo) || (p.flags & HJ_F_EXACT)) return false;
    if (p.flags & HJ_F_SEGMENTS) return hj::phj_seg_applies(g, hj::algo_lp(algo), 1ull << 40, 0);
    return hj::phj_seg_applies(g, hj::algo_lp(algo), nR, nS);
}

int scratch_need(hj_algo_t algo, const hj_params_t &p, size_t nR, size_t nS, bool host_inputs, int num_sms,
                 size_t *bytes, bool seg) {
    size_t need = kAccBytes;
    if (host_inputs) need += align256(nR * 16) + align256(nS * 16);
    if (is_phj(algo)) {
        hj::RadixGeom g;
        int rc = hj::radix_geom(p.num_radix_bits, p.num_passes, &g, p.radix_bits_pass1);
        if (rc) return rc;
        need += hj::phj_scratch_bytes(g, nR, nS, num_sms, seg);
    } else {
        need += align256(hj::nphj_scratch_bytes(nR, p.table_load));
    }
    *bytes = need;
    return HJ_OK;
}

// Drop the context's join graphs (they address the arena).
void drop_graphs(hj_ctx *c) {
    for (hj_graph_entry &e : c->graphs)
        if (e.exec) cudaGraphExecDestroy(e.exec);
    c->graphs.clear();
    c->last_key = hj_graph_key();
}

constexpr size_t kMaxJoinGraphs = 4;

hj_graph_entry *find_graph(hj_ctx *c, const hj_graph_key &k) {
    for (hj_graph_entry &e : c->graphs)
        if (e.key == k) {
            e.used = ++c->graph_tick;
            return &e;
        }
    return nullptr;
}

int ensure_arena(hj_ctx *c, size_t bytes) {
    if (c->arena_bytes >= bytes) return HJ_OK;
    CU_OR(cudaStreamSynchronize(c->stream), HJ_E_DEVICE);
    drop_graphs(c);
    if (c->arena) cudaFree(c->arena);
    c->arena = nullptr;
    c->arena_bytes = 0;
    if (cudaMalloc(&c->arena, bytes) != cudaSuccess) {
        cudaGetLastError();
        c->arena = nullptr;
        return HJ_E_OOM;
    }
    c->arena_bytes = bytes;
    return HJ_OK;
}

int map_error_bits(unsigned bits) {
    if (!bits) return HJ_OK;
    if (bits & hj::kErrSpinLimit) return HJ_E_TIMEOUT;
    if (bits & hj::kErrProbeLimit) return HJ_E_PROBE_LIMIT;
    if (bits & hj::kErrOutput) return HJ_E_CAPACITY;
    if (bits & hj::kErrRowId) return HJ_E_ROWID;
    return HJ_E_OVERFLOW;
}

}  // namespace

extern "C" {

void hj_params_init(hj_params_t *p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->num_radix_bits = 14;
    p->num_passes = 2;
    p->table_load = 0.0;
}

const char *hj_status_str(int s) {
    switch (s) {
        case HJ_OK: return "ok";
        case HJ_E_INVAL: return "invalid argument";
        case HJ_E_OOM: return "out of memory";
        case HJ_E_DEVICE: return "CUDA error";
        case HJ_E_PROBE_LIMIT: return "table walk exceeded capacity";
        case HJ_E_TIMEOUT: return "bounded wait gave up";
        case HJ_E_NOT_FOUND: return "unknown algorithm";
        case HJ_E_IO: return "i/o error";
        case HJ_E_OVERFLOW: return "device bound check fired";
        case HJ_E_BUDGET: return "over the HBM budget";
        case HJ_E_CAPACITY: return "the pair buffer is too small (matched_cnt = pairs needed)";
        case HJ_E_ROWID: return "a matched row id is not a 1-based position of its relation";
        default: return "unknown status";
    }
}

static const char *const k_algo_names[HJ_ALGO_COUNT] = {"nphj_sc",      "nphj_lp",      "phj_radix_bc", "phj_radix_lp",
                                                        "phj_radix_sc", "phj_radix_hr", "phj_radix_hro"};

const char *hj_algo_name(hj_algo_t a) {
    return ((int)a >= 0 && a < HJ_ALGO_COUNT) ? k_algo_names[a] : "?";
}

int hj_algo_from_name(const char *name, hj_algo_t *algo) {
    if (!name || !algo) return HJ_E_INVAL;
    for (int i = 0; i < HJ_ALGO_COUNT; i++)
        if (strcmp(name, k_algo_names[i]) == 0) {
            *algo = (hj_algo_t)i;
            return HJ_OK;
        }
    // Bandwidth-regulated variants compute identical results (src/algo/phj_bw_reg.c:2874-2893); the
    // asymmetric-radix variants too (the bit split is hj_params_t.radix_bits_pass1).
    static const char *const prefixes[] = {"phj_radix_bw_reg_", "phj_asymm_radix_bw_reg_", "phj_asymm_radix_"};
    for (const char *pre : prefixes) {
        const size_t n = strlen(pre);
        if (strncmp(name, pre, n) != 0) continue;
        const char *suf = name + n;
        static const char *const sufs[] = {"bc", "lp", "sc", "hr", "hro"};
        static const hj_algo_t algs[] = {HJ_ALGO_PHJ_RADIX_BC, HJ_ALGO_PHJ_RADIX_LP, HJ_ALGO_PHJ_RADIX_SC,
                                         HJ_ALGO_PHJ_RADIX_HR, HJ_ALGO_PHJ_RADIX_HRO};
        for (int i = 0; i < 5; i++)
            if (strcmp(suf, sufs[i]) == 0) {
                // The reference has no phj_asymm_radix_lp (src/main.c:80-82, 114-116, 128, 138).
                if (i == 1 && pre[4] == 'a') return HJ_E_NOT_FOUND;
                *algo = algs[i];
                return HJ_OK;
            }
    }
    return HJ_E_NOT_FOUND;
}

int hj_ctx_create(int device, hj_ctx_t **out) {
    if (!out) return HJ_E_INVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return HJ_E_DEVICE;
    }
    DeviceGuard g(device);
    hj_ctx *c = new hj_ctx();
    c->device = device;
    CU_OR(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device), HJ_E_DEVICE);
    CU_OR(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), HJ_E_DEVICE);
    CU_OR(cudaEventCreate(&c->ev_h2d), HJ_E_DEVICE);
    CU_OR(cudaEventCreate(&c->ev_start), HJ_E_DEVICE);
    CU_OR(cudaEventCreate(&c->ev_mid), HJ_E_DEVICE);
    CU_OR(cudaEventCreate(&c->ev_end), HJ_E_DEVICE);
    CU_OR(cudaEventCreate(&c->ev_ret), HJ_E_DEVICE);
    CU_OR(cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming), HJ_E_DEVICE);
    for (int i = 0; i <= HJ_PH_COUNT; i++) CU_OR(cudaEventCreate(&c->ev_ph[i]), HJ_E_DEVICE);
    CU_OR(cudaMallocHost(&c->acc_host, sizeof(JoinAccum)), HJ_E_OOM);
    c->tuner.nphj_max_table_bytes = 64e6;
    c->tuner.wave_table_bytes = 64e6;
    c->tuner.partition_target = 6144;
    c->tuner.calibrated = 0;
    *out = c;
    return HJ_OK;
}

int hj_ctx_destroy(hj_ctx_t *c) {
    if (!c) return HJ_E_INVAL;
    {
        DeviceGuard g(c->device);
        std::lock_guard<std::mutex> lk(c->mu);
        if (c->stream) cudaStreamSynchronize(c->stream);
        drop_graphs(c);
        if (c->arena) cudaFree(c->arena);
        if (c->acc_host) cudaFreeHost(c->acc_host);
        cudaEventDestroy(c->ev_h2d);
        cudaEventDestroy(c->ev_start);
        cudaEventDestroy(c->ev_mid);
        if (c->ev_ret) cudaEventDestroy(c->ev_ret);
        if (c->ev_done) cudaEventDestroy(c->ev_done);
        cudaEventDestroy(c->ev_end);
        for (int i = 0; i <= HJ_PH_COUNT; i++) cudaEventDestroy(c->ev_ph[i]);
        if (c->stream) cudaStreamDestroy(c->stream);
    }
    delete c;
    return HJ_OK;
}

size_t hj_ctx_scratch_bytes(const hj_ctx_t *c) { return c ? c->arena_bytes : 0; }

int hj_ctx_reserve(hj_ctx_t *c, hj_algo_t algo, const hj_params_t *pin, size_t nR, size_t nS) {
    if (!c || (int)algo < 0 || algo >= HJ_ALGO_COUNT) return HJ_E_INVAL;
    hj_params_t p;
    resolve_params(pin, &p);
    size_t need = 0;
    bool seg = false;
    if (is_phj(algo)) {
        hj::RadixGeom geom;
        const int rc = hj::radix_geom(p.num_radix_bits, p.num_passes, &geom, p.radix_bits_pass1);
        if (rc) return rc;
        seg = want_seg(algo, p, geom, nR, nS);
    }
    int rc = scratch_need(algo, p, nR, nS, !p.inputs_on_device, c->num_sms, &need, seg);
    if (rc) return rc;
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    rc = ensure_arena(c, need);
    if (rc == HJ_E_OOM && seg) {
        rc = scratch_need(algo, p, nR, nS, !p.inputs_on_device, c->num_sms, &need, false);
        if (!rc) rc = ensure_arena(c, need);
    }
    return rc;
}

int hj_join_ctx(hj_ctx_t *c, hj_algo_t algo, const hj_params_t *pin, const hj_tuple_t *R, size_t nR,
                const hj_tuple_t *S, size_t nS, hj_result_t *out) {
    if (!c || !out || (int)algo < 0 || algo >= HJ_ALGO_COUNT) return HJ_E_INVAL;
    memset(out, 0, sizeof(*out));
    if ((nR && !R) || (nS && !S)) return out->status = HJ_E_INVAL;
    hj_params_t p;
    resolve_params(pin, &p);
    if (p.device != c->device) return out->status = HJ_E_INVAL;
    hj::RadixGeom geom = {};
    if (is_phj(algo)) {
        int rc = hj::radix_geom(p.num_radix_bits, p.num_passes, &geom, p.radix_bits_pass1);
        if (rc) return out->status = rc;
        out->physical_passes = geom.passes;
    }
    if (nR == 0 || nS == 0) return out->status = HJ_OK;  // no join task (src/algo/phj.c:1290)

    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    const bool host_in = !p.inputs_on_device;
    size_t need = 0;
    bool seg = want_seg(algo, p, geom, nR, nS);
    int rc = scratch_need(algo, p, nR, nS, host_in, c->num_sms, &need, seg);
    if (rc) return out->status = rc;
    rc = ensure_arena(c, need);
    if (rc == HJ_E_OOM && seg) {  // the exact-offset pipeline needs less memory
        seg = false;
        rc = scratch_need(algo, p, nR, nS, host_in, c->num_sms, &need, false);
        if (!rc) rc = ensure_arena(c, need);
    }
    if (rc) return out->status = rc;
    cudaStream_t st = p.stream ? (cudaStream_t)p.stream : c->stream;
    // A join that a watchdog gave up on may still run; its arena use must end before this one starts.
    CU_OR(cudaStreamWaitEvent(st, c->ev_done, 0), out->status = HJ_E_DEVICE);
    const bool timing = !(p.flags & HJ_F_NO_TIMING);
    const bool phases = (p.flags & HJ_F_PHASE_TIMES) != 0;
    cudaEvent_t *ph = phases ? c->ev_ph : nullptr;
    uint32_t launches = 0;

    char *cur = c->arena;
    JoinAccum *acc = reinterpret_cast<JoinAccum *>(cur);
    cur += kAccBytes;
    const ulonglong2 *dR = reinterpret_cast<const ulonglong2 *>(R);
    const ulonglong2 *dS = reinterpret_cast<const ulonglong2 *>(S);
    if (host_in) {
        ulonglong2 *r = reinterpret_cast<ulonglong2 *>(cur);
        cur += align256(nR * 16);
        ulonglong2 *s = reinterpret_cast<ulonglong2 *>(cur);
        cur += align256(nS * 16);
        if (timing) CU_OR(cudaEventRecord(c->ev_h2d, st), out->status = HJ_E_DEVICE);
        CU_OR(cudaMemcpyAsync(r, R, nR * 16, cudaMemcpyHostToDevice, st), out->status = HJ_E_DEVICE);
        CU_OR(cudaMemcpyAsync(s, S, nS * 16, cudaMemcpyHostToDevice, st), out->status = HJ_E_DEVICE);
        dR = r;
        dS = s;
    }
    // phj_radix_lp: first with unordered partition passes (phj_radix_bc's ranks), then, only if a probe
    // tuple matched two build tuples (the first match then depends on the order inside a partition),
    // again with ordered ones. The second run needs the first one's flag on the host, so these joins
    // are not captured into a graph; a build relation that needed it runs ordered at once next time.
    const bool lp_try = is_phj(algo) && hj::algo_lp(algo) && !(p.flags & (HJ_F_ORDERED | HJ_F_TEST_STALL)) &&
                        p.watchdog_ms <= 0 && !(c->lp_ordered_R == (const void *)R && c->lp_ordered_nR == nR);
    const bool lp_ordered = is_phj(algo) && hj::algo_lp(algo) && !lp_try;
    bool lp_rerun = false;
    // Everything from the result reset to the result copy; a repeated device-resident join replays it
    // from a CUDA graph (the key holds every input of the enqueued work).
    auto enqueue = [&]() -> int {
        if (cudaMemsetAsync(acc, 0, sizeof(JoinAccum), st) != cudaSuccess) return HJ_E_DEVICE;
        if (timing && hj::record_event(c->ev_start, st) != cudaSuccess) return HJ_E_DEVICE;
        int erc;
        if (is_phj(algo)) {
            hj::PhjScratch s;
            hj::phj_carve(geom, nR, nS, c->num_sms, cur, &s, seg);
            const int tf = ((p.flags & HJ_F_TEST_STALL) ? 1 : 0) | ((p.flags & HJ_F_WIDE) ? 2 : 0) |
                           ((p.flags & HJ_F_WORDS) ? 4 : 0);
            uint32_t first = 0;
            if (lp_try) {
                erc = hj::phj_enqueue(geom, true, hj::algo_skip0(algo), dR, nR, dS, nS, s, acc, st,
                                      timing ? c->ev_mid : nullptr, c->num_sms, ph, &first, nullptr, tf, false);
                if (erc) return erc;
                if (cudaMemcpyAsync(c->acc_host, acc, sizeof(JoinAccum), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess)
                    return HJ_E_DEVICE;
                lp_rerun = c->acc_host->dup_flag != 0;
                if (lp_rerun && cudaMemsetAsync(acc, 0, sizeof(JoinAccum), st) != cudaSuccess) return HJ_E_DEVICE;
            }
            if (!lp_try || lp_rerun)
                erc = hj::phj_enqueue(geom, hj::algo_lp(algo), hj::algo_skip0(algo), dR, nR, dS, nS, s, acc, st,
                                      timing ? c->ev_mid : nullptr, c->num_sms, ph, &launches, nullptr, tf);
            launches += first;
        } else {
            const size_t tb = c->arena_bytes - (size_t)(cur - c->arena);
            erc = hj::nphj_enqueue(hj::algo_lp(algo), false, dR, nR, dS, nS, cur, tb, p.table_load, acc, st,
                                   timing ? c->ev_mid : nullptr, c->num_sms, ph, &launches);
        }
        if (erc) return erc;
        if (timing && hj::record_event(c->ev_end, st) != cudaSuccess) return HJ_E_DEVICE;
        if (cudaMemcpyAsync(c->acc_host, acc, sizeof(JoinAccum), cudaMemcpyDeviceToHost, st) != cudaSuccess)
            return HJ_E_DEVICE;
        return HJ_OK;
    };
    hj_graph_key key;
    const bool graphable = !host_in && st == c->stream && !(p.flags & HJ_F_TEST_STALL) && !lp_try;
    if (graphable) {
        key.algo = (int)algo;
        key.R = R;
        key.S = S;
        key.nR = nR;
        key.nS = nS;
        key.flags = p.flags;
        key.bits = p.num_radix_bits;
        key.passes = p.num_passes;
        key.bits_pass1 = p.radix_bits_pass1;
        key.table_load = p.table_load;
        key.seg = seg;
        key.arena = c->arena;
        key.arena_bytes = c->arena_bytes;
    }
    if (hj_graph_entry *ge = graphable ? find_graph(c, key) : nullptr) {
        CU_OR(cudaGraphLaunch(ge->exec, st), out->status = HJ_E_DEVICE);
        launches = ge->launches;
    } else if (graphable && key == c->last_key) {
        // Second identical call in a row: capture, instantiate, launch; keep the graph. If the capture
        // or the instantiation fails, the join runs its kernels directly instead.
        bool ran = false;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            const int crc = enqueue();
            cudaGraph_t graph = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(st, &graph);
            cudaGraphExec_t exec = nullptr;
            if (!crc && ce == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess &&
                cudaGraphLaunch(exec, st) == cudaSuccess) {
                if (c->graphs.size() >= kMaxJoinGraphs) {
                    size_t lru = 0;
                    for (size_t i = 1; i < c->graphs.size(); i++)
                        if (c->graphs[i].used < c->graphs[lru].used) lru = i;
                    cudaGraphExecDestroy(c->graphs[lru].exec);
                    c->graphs.erase(c->graphs.begin() + (long)lru);
                }
                hj_graph_entry e;
                e.key = key;
                e.exec = exec;
                e.launches = launches;
                e.used = ++c->graph_tick;
                c->graphs.push_back(e);
                ran = true;
            } else if (exec) {
                cudaGraphExecDestroy(exec);
            }
            if (graph) cudaGraphDestroy(graph);
            if (crc && crc != HJ_E_DEVICE) {  // an argument the enqueue rejects: the same without a graph
                cudaGetLastError();
                return out->status = crc;
            }
        }
        cudaGetLastError();
        if (!ran) {
            launches = 0;
            rc = enqueue();
            if (rc) {
                cudaStreamSynchronize(st);
                return out->status = rc;
            }
        }
    } else {
        rc = enqueue();
        if (rc) {
            cudaStreamSynchronize(st);
            return out->status = rc;
        }
    }
    if (graphable) c->last_key = key;
    if (p.watchdog_ms > 0) {
        // Host watchdog: poll the join's completion against a deadline instead of blocking.
        CU_OR(cudaEventRecord(c->ev_done, st), out->status = HJ_E_DEVICE);
        const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(p.watchdog_ms);
        for (;;) {
            const cudaError_t q = cudaEventQuery(c->ev_done);
            if (q == cudaSuccess) break;
            if (q != cudaErrorNotReady) return out->status = HJ_E_DEVICE;
            if (std::chrono::steady_clock::now() > deadline) return out->status = HJ_E_TIMEOUT;
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    } else {
        CU_OR(cudaStreamSynchronize(st), out->status = HJ_E_DEVICE);
    }
    out->matched_cnt = c->acc_host->matched;
    out->checksum = c->acc_host->checksum;
    out->large_partitions = c->acc_host->large_parts;
    out->flags = (uint32_t)c->acc_host->flags;
    if (lp_ordered || lp_rerun) out->flags |= HJ_RES_ORDERED_PASSES;
    if (lp_rerun) {
        c->lp_ordered_R = R;
        c->lp_ordered_nR = nR;
    }
    if (timing) {
        float a = 0, b = 0, h = 0;
        cudaEventElapsedTime(&a, c->ev_start, c->ev_mid);
        cudaEventElapsedTime(&b, c->ev_mid, c->ev_end);
        if (host_in) cudaEventElapsedTime(&h, c->ev_h2d, c->ev_start);
        out->buildpart = a * 1e-3;
        out->probejoin = b * 1e-3;
        out->total = out->buildpart + out->probejoin;
        out->h2d = h * 1e-3;
    }
    if (phases) {
        for (int i = 0; i < HJ_PH_COUNT; i++) {
            float ms = 0;
            int from = 0, to = 0;
            if (hj::phj_phase_span(seg, i, &from, &to)) cudaEventElapsedTime(&ms, c->ev_ph[from], c->ev_ph[to]);
            out->phase[i] = ms * 1e-3;
        }
    }
    out->kernel_launches = launches;
    out->status = map_error_bits(c->acc_host->error);
    return out->status;
}

// Materialising joins (the reference's ptr_* joins, src/algo/ptr_phj.c, ptr_nphj.c): the join writes
// one (r.row_id, s.row_id) pair per match, and a retrieve phase recomputes the checksum by gathering
// R[r_row_id - 1].row_id + S[s_row_id - 1].row_id (src/inc/utils.c:712-724).
static int join_mat(hj_ctx *c, hj_algo_t algo, const hj_params_t &p, const hj_tuple_t *R, size_t nR,
                    const hj_tuple_t *S, size_t nS, hj_pair_t *user_pairs, size_t user_cap,
                    unsigned long long cap_guess, hj_result_t *out) {
    hj::RadixGeom geom = {};
    if (is_phj(algo)) {
        int rc = hj::radix_geom(p.num_radix_bits, p.num_passes, &geom, p.radix_bits_pass1);
        if (rc) return out->status = rc;
        out->physical_passes = geom.passes;
    }
    if (nR == 0 || nS == 0) return out->status = HJ_OK;
    const bool host_in = !p.inputs_on_device;
    // Pairs land in the caller's device buffer, or in the arena (library-owned, or staged for a host
    // buffer).
    const bool pairs_in_arena = !user_pairs || host_in;
    const unsigned long long cap = user_pairs ? (unsigned long long)user_cap : cap_guess;
    bool seg = want_seg(algo, p, geom, nR, nS);
    auto need_of = [&](bool sg) {
        size_t need = kAccBytes;
        if (host_in) need += align256(nR * 16) + align256(nS * 16);
        if (is_phj(algo))
            need += hj::phj_scratch_bytes(geom, nR, nS, c->num_sms, sg);
        else
            need += align256(hj::nphj_scratch_bytes(nR, p.table_load, true));
        if (pairs_in_arena) need += align256(cap * 16);
        return need;
    };
    int rc = ensure_arena(c, need_of(seg));
    if (rc == HJ_E_OOM && seg) {
        seg = false;
        rc = ensure_arena(c, need_of(false));
    }
    if (rc) return out->status = rc;
    cudaStream_t st = p.stream ? (cudaStream_t)p.stream : c->stream;
    CU_OR(cudaStreamWaitEvent(st, c->ev_done, 0), out->status = HJ_E_DEVICE);
    const bool timing = !(p.flags & HJ_F_NO_TIMING);
    uint32_t launches = 0;

    char *cur = c->arena;
    JoinAccum *acc = reinterpret_cast<JoinAccum *>(cur);
    cur += kAccBytes;
    const ulonglong2 *dR = reinterpret_cast<const ulonglong2 *>(R);
    const ulonglong2 *dS = reinterpret_cast<const ulonglong2 *>(S);
    if (host_in) {
        ulonglong2 *r = reinterpret_cast<ulonglong2 *>(cur);
        cur += align256(nR * 16);
        ulonglong2 *s = reinterpret_cast<ulonglong2 *>(cur);
        cur += align256(nS * 16);
        if (timing) CU_OR(cudaEventRecord(c->ev_h2d, st), out->status = HJ_E_DEVICE);
        CU_OR(cudaMemcpyAsync(r, R, nR * 16, cudaMemcpyHostToDevice, st), out->status = HJ_E_DEVICE);
        CU_OR(cudaMemcpyAsync(s, S, nS * 16, cudaMemcpyHostToDevice, st), out->status = HJ_E_DEVICE);
        dR = r;
        dS = s;
    }
    hj::MatOut mat;
    mat.cap = cap;
    if (pairs_in_arena) {
        mat.pairs = reinterpret_cast<ulonglong2 *>(cur);
        cur += align256(cap * 16);
    } else {
        mat.pairs = reinterpret_cast<ulonglong2 *>(user_pairs);
    }
    CU_OR(cudaMemsetAsync(acc, 0, sizeof(JoinAccum), st), out->status = HJ_E_DEVICE);
    if (timing) CU_OR(cudaEventRecord(c->ev_start, st), out->status = HJ_E_DEVICE);
    if (is_phj(algo)) {
        hj::PhjScratch s;
        hj::phj_carve(geom, nR, nS, c->num_sms, cur, &s, seg);
        rc = hj::phj_enqueue(geom, hj::algo_lp(algo), hj::algo_skip0(algo), dR, nR, dS, nS, s, acc, st,
                             timing ? c->ev_mid : nullptr, c->num_sms, nullptr, &launches, &mat);
    } else {
        const size_t tb = c->arena_bytes - (size_t)(cur - c->arena);
        rc = hj::nphj_enqueue(hj::algo_lp(algo), false, dR, nR, dS, nS, cur, tb, p.table_load, acc, st,
                              timing ? c->ev_mid : nullptr, c->num_sms, nullptr, &launches, &mat);
    }
    if (!rc) {
        if (timing) CU_OR(cudaEventRecord(c->ev_end, st), out->status = HJ_E_DEVICE);
        rc = hj::mat_retrieve_enqueue(mat.pairs, &acc->pairs, cap, dR, nR, dS, nS, acc, st, c->num_sms);
        launches++;
    }
    if (rc) {
        cudaStreamSynchronize(st);
        return out->status = rc;
    }
    if (timing) CU_OR(cudaEventRecord(c->ev_ret, st), out->status = HJ_E_DEVICE);
    CU_OR(cudaMemcpyAsync(c->acc_host, acc, sizeof(JoinAccum), cudaMemcpyDeviceToHost, st),
          out->status = HJ_E_DEVICE);
    CU_OR(cudaStreamSynchronize(st), out->status = HJ_E_DEVICE);
    const unsigned long long n = c->acc_host->pairs;
    if (user_pairs && host_in && n)
        CU_OR(cudaMemcpy(user_pairs, mat.pairs, (size_t)(n < cap ? n : cap) * 16, cudaMemcpyDeviceToHost),
              out->status = HJ_E_DEVICE);
    out->matched_cnt = n;
    out->checksum = c->acc_host->checksum;
    out->large_partitions = c->acc_host->large_parts;
    out->flags = (uint32_t)c->acc_host->flags;
    if (timing) {
        float a = 0, b = 0, r = 0, h = 0;
        cudaEventElapsedTime(&a, c->ev_start, c->ev_mid);
        cudaEventElapsedTime(&b, c->ev_mid, c->ev_end);
        cudaEventElapsedTime(&r, c->ev_end, c->ev_ret);
        if (host_in) cudaEventElapsedTime(&h, c->ev_h2d, c->ev_start);
        out->buildpart = a * 1e-3;
        out->probejoin = b * 1e-3;
        out->retrieve = r * 1e-3;
        // The reference's ptr joins time partition/build + join/probe + retrieve (ptr_phj.c:3094-3096).
        out->total = out->buildpart + out->probejoin + out->retrieve;
        out->h2d = h * 1e-3;
    }
    out->kernel_launches = launches;
    out->status = map_error_bits(c->acc_host->error);
    return out->status;
}

int hj_join_mat_ctx(hj_ctx_t *c, hj_algo_t algo, const hj_params_t *pin, const hj_tuple_t *R, size_t nR,
                    const hj_tuple_t *S, size_t nS, hj_pair_t *pairs, size_t pair_cap, hj_result_t *out) {
    if (!c || !out || (int)algo < 0 || algo >= HJ_ALGO_COUNT) return HJ_E_INVAL;
    memset(out, 0, sizeof(*out));
    if ((nR && !R) || (nS && !S) || (pair_cap && !pairs)) return out->status = HJ_E_INVAL;
    hj_params_t p;
    resolve_params(pin, &p);
    if (p.device != c->device) return out->status = HJ_E_INVAL;
    DeviceGuard g(c->device);
    std::lock_guard<std::mutex> lk(c->mu);
    if (pairs) return join_mat(c, algo, p, R, nR, S, nS, pairs, pair_cap, 0, out);
    // Library-owned pairs: first-match joins write at most |S| pairs; for the others |S| is the
    // guess (exact for PK-FK joins), and one rerun with the exact count follows when it was short.
    int rc = join_mat(c, algo, p, R, nR, S, nS, nullptr, 0, nS ? nS : 1, out);
    if (rc == HJ_E_CAPACITY) {
        const unsigned long long need = out->matched_cnt;
        memset(out, 0, sizeof(*out));
        rc = join_mat(c, algo, p, R, nR, S, nS, nullptr, 0, need, out);
    }
    return rc;
}

int hj_join_mat(hj_algo_t algo, const hj_params_t *pin, const hj_tuple_t *R, size_t nR, const hj_tuple_t *S,
                size_t nS, hj_pair_t *pairs, size_t pair_cap, hj_result_t *out) {
    hj_params_t p;
    resolve_params(pin, &p);
    if (p.device < 0 || p.device >= 64) return HJ_E_INVAL;
    hj_ctx *c;
    {
        std::lock_guard<std::mutex> lk(g_default_mu);
        if (!g_default[p.device]) {
            int rc = hj_ctx_create(p.device, &g_default[p.device]);
            if (rc) return rc;
        }
        c = g_default[p.device];
    }
    return hj_join_mat_ctx(c, algo, &p, R, nR, S, nS, pairs, pair_cap, out);
}

int hj_join(hj_algo_t algo, const hj_params_t *pin, const hj_tuple_t *R, size_t nR, const hj_tuple_t *S,
            size_t nS, hj_result_t *out) {
    hj_params_t p;
    resolve_params(pin, &p);
    if (p.device < 0 || p.device >= 64) return HJ_E_INVAL;
    hj_ctx *c;
    {
        std::lock_guard<std::mutex> lk(g_default_mu);
        if (!g_default[p.device]) {
            int rc = hj_ctx_create(p.device, &g_default[p.device]);
            if (rc) return rc;
        }
        c = g_default[p.device];
    }
    return hj_join_ctx(c, algo, &p, R, nR, S, nS, out);
}

}  // extern "C"
