// hj_batch.cu - many independent joins as one captured launch sequence, with an autotuner.
//
// The reference runs one join per process invocation (src/main.c:429-448). A batch here takes N joins of
// uneven sizes on device-resident relations and
//   1. decides per join how to run it (the autotuner): joins whose global hash table (32 B per build
//      tuple at load 0.5) fits the table budget run as non-partitioned joins; larger ones run the
//      radix-partitioned pipeline with radix bits chosen so build partitions hold about
//      `partition_target` tuples (two passes above 8 bits). The join's result semantics - every match
//      (nphj_sc, phj_radix_bc/sc/hr/hro), first match (nphj_lp), first match with key 0 never matching
//      (phj_radix_lp) - are kept whichever implementation runs, so results equal the named algorithm's.
//      With HJ_F_TUNE the budget is chosen by timing the batch's own graph under several budgets; a
//      calibrated cost model (hj_tuner_calibrate) serves single joins;
//   2. packs the non-partitioned joins into waves whose tables together stay within the wave budget,
//      and runs each wave as one set of multi-join kernels over a flattened index space (build over all
//      build tuples of the wave, then probe over all probe tuples), so the tables are still in L2 when
//      probed;
//   3. enqueues the partitioned joins on up to kPhjLanes streams forked from the first (each with its own
//      scratch area; largest joins first, each on the least loaded stream), so they overlap the waves
//      and each other;
//   4. captures the whole sequence in a CUDA graph once (parallel branches), so a run is one graph
//      launch.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../host/hj_feistel.h"
#include "hj_common.cuh"
#include "hj_ctx.h"
#include "hj_internal.h"
#include "hj_nphj.cuh"
#include "hj_wave.cuh"

namespace hj {

constexpr unsigned long long kMjEmpty = ~0ull;

// Largest j with flat[j] <= g (flat[0] = 0, non-decreasing; empty jobs are skipped over).
__device__ __forceinline__ int mj_find(const unsigned long long *flat, int njobs, unsigned long long g) {
    int lo = 0, hi = njobs;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (flat[mid] <= g) lo = mid; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void mj_load_flat(unsigned long long *sflat, const unsigned long long *flat, int njobs) {
    for (int j = threadIdx.x; j <= njobs; j += blockDim.x) sflat[j] = flat[j];
    __syncthreads();
}

// Each block takes one contiguous range of the flattened index space, so a thread stays on one job for
// many iterations.
__device__ __forceinline__ void mj_range(unsigned long long total, unsigned long long *lo, unsigned long long *hi) {
    const unsigned long long chunk = (total + gridDim.x - 1) / gridDim.x;
    *lo = blockIdx.x * chunk;
    *hi = *lo + chunk < total ? *lo + chunk : total;
}

__device__ __forceinline__ void mj_insert(const MJob &J, const tuple_v t, unsigned long long i) {
    if (J.skip0 && t.x == 0) return;
    if (t.x == kMjEmpty) {
        if (atomicAdd(&J.side->cnt, 1ull) >= 1ull) atomicOr(&J.side->dup, 1u);
        atomicAdd(&J.side->sum, (unsigned long long)t.y);
        atomicMax(&J.side->notpos, ~i);
        return;
    }
    unsigned long long h = table_hash(t.x, J.cap);
    for (unsigned long long steps = 0;; steps++) {
        const unsigned long long cur = atomicCAS(&J.table[h].x, kMjEmpty, (unsigned long long)t.x);
        if (cur == kMjEmpty) {
            J.table[h].y = t.y;
            return;
        }
        if (cur == t.x && !J.side->dup) atomicOr(&J.side->dup, 1u);
        if (++h == J.cap) h = 0;
        if (steps + 1 >= J.cap) {
            set_error(&J.acc->error, kErrProbeLimit);
            return;
        }
    }
}

__global__ void mj_build(const MJob *__restrict__ jobs, const MChunk *__restrict__ chunks, int nchunks) {
    constexpr int U = 4;
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const MChunk ch = chunks[c];
        const MJob J = jobs[ch.job];
        for (unsigned e0 = threadIdx.x; e0 < ch.len; e0 += U * blockDim.x) {
            tuple_v t[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const unsigned e = e0 + u * blockDim.x;
                t[u] = e < ch.len ? ld_stream(J.R + ch.begin + e) : make_ulonglong2(0, 0);
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const unsigned e = e0 + u * blockDim.x;
                if (e < ch.len) mj_insert(J, t[u], ch.begin + e);
            }
        }
    }
}

// First-match joins with duplicate build keys: rebuild the job's table with one slot per key holding
// the smallest build position, then replace positions by row ids.
__global__ void mj_lp_refill(const MJob *__restrict__ jobs, int njobs, const unsigned long long *__restrict__ t_flat,
                             unsigned long long total) {
    extern __shared__ unsigned long long sflat[];
    mj_load_flat(sflat, t_flat, njobs);
    unsigned long long lo, hi;
    mj_range(total, &lo, &hi);
    int j = -1;
    unsigned long long jbeg = 0, jend = 0;
    bool act = false;
    tuple_v *table = nullptr;
    for (unsigned long long g = lo + threadIdx.x; g < hi; g += blockDim.x) {
        if (j < 0 || g >= jend || g < jbeg) {
            j = mj_find(sflat, njobs, g);
            jbeg = sflat[j];
            jend = sflat[j + 1];
            act = jobs[j].lp && *reinterpret_cast<volatile unsigned int *>(&jobs[j].side->dup);
            table = jobs[j].table;
        }
        if (act) table[g - jbeg] = make_ulonglong2(kMjEmpty, kMjEmpty);
    }
}

__global__ void mj_lp_dedup(const MJob *__restrict__ jobs, int njobs, const unsigned long long *__restrict__ r_flat,
                            unsigned long long total) {
    extern __shared__ unsigned long long sflat[];
    mj_load_flat(sflat, r_flat, njobs);
    unsigned long long lo, hi;
    mj_range(total, &lo, &hi);
    int j = -1;
    unsigned long long jbeg = 0, jend = 0;
    MJob J;
    bool act = false;
    for (unsigned long long g = lo + threadIdx.x; g < hi; g += blockDim.x) {
        if (j < 0 || g >= jend || g < jbeg) {
            j = mj_find(sflat, njobs, g);
            J = jobs[j];
            jbeg = sflat[j];
            jend = sflat[j + 1];
            act = J.lp && *reinterpret_cast<volatile unsigned int *>(&J.side->dup);
        }
        if (!act) continue;
        const unsigned long long i = g - jbeg;
        const unsigned long long k = J.R[i].x;
        if (k == kMjEmpty || (J.skip0 && k == 0)) continue;
        unsigned long long h = table_hash(k, J.cap);
        for (unsigned long long steps = 0;; steps++) {
            unsigned long long *kp = &J.table[h].x;
            unsigned long long cur = *reinterpret_cast<volatile unsigned long long *>(kp);
            if (cur == kMjEmpty) cur = atomicCAS(kp, kMjEmpty, k);
            if (cur == kMjEmpty || cur == k) {
                atomicMin(&J.table[h].y, i);
                break;
            }
            if (++h == J.cap) h = 0;
            if (steps + 1 >= J.cap) {
                set_error(&J.acc->error, kErrProbeLimit);
                break;
            }
        }
    }
}

__global__ void mj_lp_resolve(const MJob *__restrict__ jobs, int njobs, const unsigned long long *__restrict__ t_flat,
                              unsigned long long total) {
    extern __shared__ unsigned long long sflat[];
    mj_load_flat(sflat, t_flat, njobs);
    unsigned long long lo, hi;
    mj_range(total, &lo, &hi);
    int j = -1;
    unsigned long long jbeg = 0, jend = 0;
    MJob J;
    bool act = false;
    for (unsigned long long g = lo + threadIdx.x; g < hi; g += blockDim.x) {
        if (j < 0 || g >= jend || g < jbeg) {
            j = mj_find(sflat, njobs, g);
            J = jobs[j];
            jbeg = sflat[j];
            jend = sflat[j + 1];
            act = J.lp && *reinterpret_cast<volatile unsigned int *>(&J.side->dup);
        }
        if (!act) continue;
        const tuple_v e = J.table[g - jbeg];
        if (e.x != kMjEmpty) {
            if (e.y < J.nR)
                J.table[g - jbeg].y = J.R[e.y].y;
            else
                set_error(&J.acc->error, kErrBounds);
        }
    }
}

__global__ void __launch_bounds__(256, 8) mj_probe(const MJob *__restrict__ jobs, const MChunk *__restrict__ chunks,
                                                  int nchunks) {
    __shared__ unsigned long long red[64];
    constexpr int U = 2;
    for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
        const MChunk ch = chunks[c];
        const MJob J = jobs[ch.job];
        ProbeArgs P;
        P.table = J.table;
        P.cap = J.cap;
        P.lp = J.lp != 0;
        P.skip0 = J.skip0 != 0;
        P.first_only = P.lp || *reinterpret_cast<volatile unsigned int *>(&J.side->dup) == 0;
        P.side_cnt = J.side->cnt;
        P.side_sum = J.side->sum;
        P.side_first_rid = P.side_cnt ? J.R[~J.side->notpos].y : 0;
        P.err = &J.acc->error;
        unsigned long long cnt = 0, sum = 0;
        for (unsigned e0 = threadIdx.x; e0 < ch.len; e0 += U * blockDim.x) {
            tuple_v sv[U];
            bool valid[U];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const unsigned e = e0 + u * blockDim.x;
                valid[u] = e < ch.len;
                sv[u] = valid[u] ? ld_stream(J.S + ch.begin + e) : make_ulonglong2(0, 0);
            }
            probe_group<U>(P, sv, valid, cnt, sum);
        }
        block_sum2_to(cnt, sum, red, &J.acc->matched, &J.acc->checksum);
    }
}

int mj_launch_wave(const WaveDev &w, int num_sms, cudaStream_t st, uint32_t *launches) {
    if (w.count <= 0) return HJ_OK;
    if (w.total_t && cudaMemsetAsync(w.tables, 0xff, w.total_t * 16, st) != cudaSuccess) return HJ_E_DEVICE;
    if (cudaMemsetAsync(w.sides, 0, sizeof(MSide) * w.count, st) != cudaSuccess) return HJ_E_DEVICE;
    const size_t sm = sizeof(unsigned long long) * (w.count + 1);
    const int grid = num_sms * 8;
    uint32_t l = 0;
    if (w.n_r_chunks) {
        mj_build<<<w.n_r_chunks < grid ? w.n_r_chunks : grid, 256, 0, st>>>(w.jobs, w.r_chunks, w.n_r_chunks);
        l++;
    }
    if (w.any_lp && w.total_r) {
        mj_lp_refill<<<grid, 256, sm, st>>>(w.jobs, w.count, w.t_flat, w.total_t);
        mj_lp_dedup<<<grid, 256, sm, st>>>(w.jobs, w.count, w.r_flat, w.total_r);
        mj_lp_resolve<<<grid, 256, sm, st>>>(w.jobs, w.count, w.t_flat, w.total_t);
        l += 3;
    }
    if (w.n_s_chunks) {
        mj_probe<<<w.n_s_chunks < grid ? w.n_s_chunks : grid, 256, 0, st>>>(w.jobs, w.s_chunks, w.n_s_chunks);
        l++;
    }
    if (launches) *launches += l;
    return cudaGetLastError() == cudaSuccess ? HJ_OK : HJ_E_DEVICE;
}

}  // namespace hj

using hj::JoinAccum;

// ------------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------------
namespace {

constexpr int kImplNphj = 0, kImplPhj = 1;

struct Wave {
    int first, count;                 // range in the wave-ordered job list
    ulonglong2 *tables;               // the wave's tables, back to back
    hj::MSide *sides;                 // followed by one side record per job
    unsigned long long total_r, total_s, total_t;
    hj::MJob *jobs_dev;
    unsigned long long *r_flat, *s_flat, *t_flat;  // device, count + 1 each
    hj::MChunk *r_chunks, *s_chunks;                // device work items of the build and probe kernels
    int n_r_chunks, n_s_chunks;
    bool any_lp;
};

using hj::kBuildChunk;
using hj::kProbeChunkMJ;

void make_chunks(std::vector<hj::MChunk> &out, unsigned job, unsigned long long n, unsigned piece) {
    for (unsigned long long b = 0; b < n; b += piece) {
        hj::MChunk c;
        c.job = job;
        c.begin = b;
        c.len = (unsigned)(n - b < piece ? n - b : piece);
        out.push_back(c);
    }
}

size_t a256(size_t x) { return (x + 255) & ~(size_t)255; }

bool sem_lp(hj_algo_t a) { return hj::algo_lp(a); }
bool sem_skip0(hj_algo_t a) { return hj::algo_skip0(a); }

unsigned long long nphj_slots(size_t nR) { return hj::mj_slots(nR); }

}  // namespace

// Partitioned joins of a batch run on up to this many parallel branches (streams forked from the batch's
// stream, each with its own scratch), so that small pipelines overlap instead of running one after
// another; the largest joins are placed first, each on the branch with the fewest tuples so far. Fewer
// branches when their scratch would take more than a quarter of the free device memory. (512 joins:
// 40.4 ms on one branch, 33.7 on four, 33.0 on eight.)
constexpr int kPhjLanes = 8;

struct hj_batch {
    hj_ctx *ctx = nullptr;
    int njobs = 0;
    std::vector<hj_batch_job_t> jobs;
    std::vector<int> impl, bits, passes;
    std::vector<Wave> waves;
    std::vector<int> phj_jobs;
    char *mem = nullptr;
    size_t mem_bytes = 0;
    JoinAccum *accs = nullptr;      // device, one per job
    JoinAccum *accs_host = nullptr; // pinned
    char *phj_scratch = nullptr;                  // phj_lanes areas of phj_lane_bytes
    size_t phj_lane_bytes = 0;
    int phj_lanes = 1;
    cudaStream_t stream = nullptr;
    cudaStream_t stream_phj[kPhjLanes] = {};      // partitioned joins, forked from `stream`
    cudaEvent_t ev_fork = nullptr, ev_join[kPhjLanes] = {};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool use_graph = true;
    uint32_t launches = 0;
};

namespace {

// Calibrated cost of each implementation for a join of (nR, nS), from the level of the nearest build
// size (log scale). Returns false when the tuner has no cost model.
bool model_prefers_nphj(const hj_tuner_t &t, size_t nR, size_t nS, bool *nphj) {
    if (!t.calibrated) return false;
    int best = -1;
    double bd = 1e300;
    for (int i = 0; i < HJ_TUNER_LEVELS; i++) {
        if (!(t.level_nR[i] > 0) || !(t.phj[i] > 0)) continue;
        const double d = std::fabs(std::log2((double)(nR ? nR : 1)) - std::log2(t.level_nR[i]));
        if (d < bd) {
            bd = d;
            best = i;
        }
    }
    if (best < 0) return false;
    const double tn = (double)nR * t.nphj_build[best] + (double)nS * t.nphj_probe[best];
    const double tp = t.phj_fixed + (double)(nR + nS) * t.phj[best];
    *nphj = tn <= tp;
    return true;
}

void decide(const hj_ctx *c, size_t nR, size_t nS, int *impl, int *bits, int *passes) {
    const hj_tuner_t &t = c->tuner;
    const bool fits = (double)nphj_slots(nR) * 16.0 <= t.nphj_max_table_bytes;
    bool use_nphj = fits;
    bool pref = false;
    if (fits && model_prefers_nphj(t, nR, nS, &pref)) use_nphj = pref;
    if (use_nphj) {
        *impl = kImplNphj;
        *bits = 0;
        *passes = 0;
        return;
    }
    int b = 1;
    while (b < 15 && (double)nR / (double)(1ull << b) > (double)t.partition_target) b++;
    *impl = kImplPhj;
    *bits = b;
    *passes = b > 8 ? 2 : 1;
}

#define BCU(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "hjscm batch: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
            return HJ_E_DEVICE;                                                        \
        }                                                                              \
    } while (0)

int enqueue_batch(hj_batch *b) {
    const int sms = b->ctx->num_sms;
    cudaStream_t st = b->stream;
    BCU(cudaMemsetAsync(b->accs, 0, sizeof(JoinAccum) * b->njobs, st));
    uint32_t launches = 0;
    // The partitioned joins run on streams forked here and joined at the end: they share nothing with
    // the waves of non-partitioned joins or with each other, and their kernels fill the SMs that a
    // wave's small kernels, or a small pipeline's, leave idle (in the captured graph these become
    // parallel branches).
    const bool fork = !b->phj_jobs.empty();
    const int lanes = fork ? b->phj_lanes : 0;
    if (fork) {
        BCU(cudaEventRecord(b->ev_fork, st));
        for (int l = 0; l < lanes; l++) BCU(cudaStreamWaitEvent(b->stream_phj[l], b->ev_fork, 0));
    }
    for (const Wave &w : b->waves) {
        if (w.total_r == 0 && w.total_s == 0) continue;
        hj::WaveDev wd;
        wd.jobs = w.jobs_dev;
        wd.count = w.count;
        wd.r_chunks = w.r_chunks;
        wd.s_chunks = w.s_chunks;
        wd.n_r_chunks = w.n_r_chunks;
        wd.n_s_chunks = w.n_s_chunks;
        wd.r_flat = w.r_flat;
        wd.t_flat = w.t_flat;
        wd.total_r = w.total_r;
        wd.total_t = w.total_t;
        wd.any_lp = w.any_lp;
        wd.tables = w.tables;
        wd.sides = w.sides;
        const int rc = hj::mj_launch_wave(wd, sms, st, &launches);
        if (rc) return rc;
    }
    std::vector<int> order(b->phj_jobs);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return b->jobs[x].nR + b->jobs[x].nS > b->jobs[y].nR + b->jobs[y].nS;
    });
    unsigned long long load[kPhjLanes] = {};
    for (int j : order) {
        const hj_batch_job_t &J = b->jobs[j];
        if (J.nR == 0 || J.nS == 0) continue;
        int l = 0;
        for (int q = 1; q < lanes; q++)
            if (load[q] < load[l]) l = q;
        load[l] += J.nR + J.nS;
        hj::RadixGeom g;
        if (hj::radix_geom(b->bits[j], b->passes[j], &g)) return HJ_E_INVAL;
        hj::PhjScratch s;
        hj::phj_carve(g, J.nR, J.nS, sms, b->phj_scratch + (size_t)l * b->phj_lane_bytes, &s);
        uint32_t nl = 0;
        int rc = hj::phj_enqueue(g, sem_lp(J.algo), sem_skip0(J.algo), reinterpret_cast<const ulonglong2 *>(J.R), J.nR,
                                 reinterpret_cast<const ulonglong2 *>(J.S), J.nS, s, b->accs + j, b->stream_phj[l],
                                 nullptr, sms, nullptr, &nl);
        if (rc) return rc;
        launches += nl;
    }
    for (int l = 0; l < lanes; l++) {
        BCU(cudaEventRecord(b->ev_join[l], b->stream_phj[l]));
        BCU(cudaStreamWaitEvent(st, b->ev_join[l], 0));
    }
    b->launches = launches;
    return HJ_OK;
}

}  // namespace

extern "C" {

int hj_tuner_get(hj_ctx_t *c, hj_tuner_t *out) {
    if (!c || !out) return HJ_E_INVAL;
    *out = c->tuner;
    return HJ_OK;
}

int hj_tuner_set(hj_ctx_t *c, const hj_tuner_t *in) {
    if (!c || !in || !(in->nphj_max_table_bytes >= 0) || in->partition_target < 64) return HJ_E_INVAL;
    c->tuner = *in;
    return HJ_OK;
}

int hj_tuner_decide(hj_ctx_t *c, size_t nR, size_t nS, int *impl, int *bits, int *passes) {
    if (!c || !impl || !bits || !passes) return HJ_E_INVAL;
    decide(c, nR, nS, impl, bits, passes);
    return HJ_OK;
}

static int plan_one(hj_ctx_t *c, const hj_batch_job_t *jobs, int njobs, const hj_params_t *p, hj_batch_t **out);

// Empirical tuning of a batch (HJ_F_TUNE): plan it under a few table budgets around the current one,
// time each plan's graph, keep the fastest and leave its budget in the context's tuner. Timings of
// single joins in isolation do not predict a batch well (waves share tables' L2 room, partitioned
// joins overlap the waves on their own branch), the batch itself does.
int hj_batch_plan(hj_ctx_t *c, const hj_batch_job_t *jobs, int njobs, const hj_params_t *p, hj_batch_t **out) {
    if (!c || !out) return HJ_E_INVAL;
    if (!(p && (p->flags & HJ_F_TUNE))) return plan_one(c, jobs, njobs, p, out);
    *out = nullptr;
    const hj_tuner_t saved = c->tuner;
    const double base = saved.nphj_max_table_bytes > 0 ? saved.nphj_max_table_bytes : 64e6;
    const double scales[] = {1.0 / 32, 1.0 / 16, 0.125, 0.25, 0.5, 1.0, 2.0, 4.0};
    hj_batch_t *best = nullptr;
    double best_s = 1e300, best_budget = base;
    std::vector<int> last_impl;
    for (double sc : scales) {
        hj_tuner_t t = saved;
        t.nphj_max_table_bytes = base * sc;
        t.calibrated = 0;  // the table-budget rule
        c->tuner = t;
        hj_batch_t *b = nullptr;
        int rc = plan_one(c, jobs, njobs, p, &b);
        if (rc) {
            c->tuner = saved;
            if (best) hj_batch_destroy(best);
            return rc;
        }
        if (best && b->impl == last_impl) {  // same decisions as the previous budget: nothing to time
            hj_batch_destroy(b);
            continue;
        }
        last_impl = b->impl;
        double s = 1e300;
        for (int rep = 0; rep < 3 && !rc; rep++) {
            hj_batch_stats_t st;
            rc = hj_batch_run(b, nullptr, &st);
            if (!rc && rep > 0) s = std::min(s, st.seconds);
        }
        if (rc) {
            hj_batch_destroy(b);
            c->tuner = saved;
            if (best) hj_batch_destroy(best);
            return rc;
        }
        if (s < best_s) {
            if (best) hj_batch_destroy(best);
            best = b;
            best_s = s;
            best_budget = t.nphj_max_table_bytes;
        } else {
            hj_batch_destroy(b);
        }
    }
    c->tuner = saved;
    c->tuner.nphj_max_table_bytes = best_budget;
    c->tuner.calibrated = 0;
    *out = best;
    return HJ_OK;
}

static int plan_one(hj_ctx_t *c, const hj_batch_job_t *jobs, int njobs, const hj_params_t *p, hj_batch_t **out) {
    if (!c || !out || njobs < 0 || (njobs && !jobs)) return HJ_E_INVAL;
    *out = nullptr;
    for (int j = 0; j < njobs; j++) {
        if ((int)jobs[j].algo < 0 || jobs[j].algo >= HJ_ALGO_COUNT) return HJ_E_INVAL;
        if ((jobs[j].nR && !jobs[j].R) || (jobs[j].nS && !jobs[j].S)) return HJ_E_INVAL;
        if (jobs[j].nR >= (1ull << 32) || jobs[j].nS >= (1ull << 32)) return HJ_E_INVAL;
    }
    hj_batch *b = new hj_batch();
    b->ctx = c;
    b->njobs = njobs;
    b->jobs.assign(jobs, jobs + njobs);
    b->impl.resize(njobs);
    b->bits.resize(njobs);
    b->passes.resize(njobs);
    b->use_graph = !(p && (p->flags & HJ_F_NO_GRAPH));
    for (int j = 0; j < njobs; j++) decide(c, jobs[j].nR, jobs[j].nS, &b->impl[j], &b->bits[j], &b->passes[j]);

    // Waves of non-partitioned joins, packed in job order up to the table budget.
    const double budget = c->tuner.wave_table_bytes > 0 ? c->tuner.wave_table_bytes : 64e6;
    std::vector<int> order;
    std::vector<std::pair<int, int>> wave_ranges;  // [first, count) into order
    double acc = 0;
    int wfirst = 0;
    for (int j = 0; j < njobs; j++) {
        if (b->impl[j] != kImplNphj) {
            b->phj_jobs.push_back(j);
            continue;
        }
        const double tb = (double)nphj_slots(jobs[j].nR) * 16.0;
        if ((int)order.size() > wfirst && (acc + tb > budget || (int)order.size() - wfirst >= 1024)) {
            wave_ranges.push_back({wfirst, (int)order.size() - wfirst});
            wfirst = (int)order.size();
            acc = 0;
        }
        order.push_back(j);
        acc += tb;
    }
    if ((int)order.size() > wfirst) wave_ranges.push_back({wfirst, (int)order.size() - wfirst});

    // Device memory of the batch: results, wave tables (the largest wave), wave descriptors, and the
    // scratch of the largest partitioned join.
    size_t max_wave_tables = 0, desc_bytes = 0;
    for (auto &wr : wave_ranges) {
        size_t t = 0;
        for (int q = 0; q < wr.second; q++) t += nphj_slots(jobs[order[wr.first + q]].nR) * 16;
        t += sizeof(hj::MSide) * wr.second;
        max_wave_tables = std::max(max_wave_tables, a256(t));
        size_t nrc = 0, nsc = 0;
        for (int q = 0; q < wr.second; q++) {
            nrc += (jobs[order[wr.first + q]].nR + kBuildChunk - 1) / kBuildChunk;
            nsc += (jobs[order[wr.first + q]].nS + kProbeChunkMJ - 1) / kProbeChunkMJ;
        }
        desc_bytes += a256(sizeof(hj::MJob) * wr.second) + 3 * a256(8 * (wr.second + 1)) +
                      a256(sizeof(hj::MChunk) * (nrc + 1)) + a256(sizeof(hj::MChunk) * (nsc + 1));
    }
    size_t phj_bytes = 0;
    for (int j : b->phj_jobs) {
        hj::RadixGeom g;
        if (hj::radix_geom(b->bits[j], b->passes[j], &g)) {
            delete b;
            return HJ_E_INVAL;
        }
        phj_bytes = std::max(phj_bytes, hj::phj_scratch_bytes(g, jobs[j].nR, jobs[j].nS, c->num_sms));
    }
    const size_t acc_bytes = a256(sizeof(JoinAccum) * (njobs ? njobs : 1));
    // All waves share one table area (they run one after another); descriptors are per wave.
    b->phj_lane_bytes = a256(phj_bytes);
    {
        size_t free_b = 0, total_b = 0;
        int dev_now = -1;
        cudaGetDevice(&dev_now);
        cudaSetDevice(c->device);
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            free_b = 0;
        }
        if (dev_now >= 0) cudaSetDevice(dev_now);
        size_t lanes = std::min<size_t>(kPhjLanes, b->phj_jobs.size() ? b->phj_jobs.size() : 1);
        while (lanes > 1 && lanes * b->phj_lane_bytes > free_b / 4) lanes--;
        b->phj_lanes = (int)lanes;
    }
    b->mem_bytes = acc_bytes + max_wave_tables + desc_bytes + (size_t)b->phj_lanes * b->phj_lane_bytes;
    int dev_prev = -1;
    cudaGetDevice(&dev_prev);
    cudaSetDevice(c->device);
    auto fail = [&](int rc) {
        hj_batch_destroy(b);
        if (dev_prev >= 0) cudaSetDevice(dev_prev);
        return rc;
    };
    if (cudaMalloc(&b->mem, b->mem_bytes ? b->mem_bytes : 256) != cudaSuccess) {
        cudaGetLastError();
        b->mem = nullptr;
        return fail(HJ_E_OOM);
    }
    if (cudaMallocHost(&b->accs_host, sizeof(JoinAccum) * (njobs ? njobs : 1)) != cudaSuccess) return fail(HJ_E_OOM);
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess)
        return fail(HJ_E_DEVICE);
    for (int l = 0; l < kPhjLanes; l++)
        if (cudaStreamCreateWithFlags(&b->stream_phj[l], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_join[l], cudaEventDisableTiming) != cudaSuccess)
            return fail(HJ_E_DEVICE);
    if (cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) return fail(HJ_E_DEVICE);
    char *cur = b->mem;
    b->accs = reinterpret_cast<JoinAccum *>(cur);
    cur += acc_bytes;
    char *tables = cur;
    cur += max_wave_tables;
    for (auto &wr : wave_ranges) {
        Wave w;
        w.first = wr.first;
        w.count = wr.second;
        std::vector<hj::MJob> mj(w.count);
        std::vector<unsigned long long> rf(w.count + 1, 0), sf(w.count + 1, 0), tf(w.count + 1, 0);
        std::vector<hj::MChunk> rch, sch;
        char *tp = tables;
        size_t slots_total = 0;
        for (int q = 0; q < w.count; q++) slots_total += nphj_slots(jobs[order[w.first + q]].nR);
        hj::MSide *sides = reinterpret_cast<hj::MSide *>(tables + slots_total * 16);
        w.any_lp = false;
        for (int q = 0; q < w.count; q++) {
            const int j = order[w.first + q];
            const hj_batch_job_t &J = jobs[j];
            hj::MJob m;
            m.R = reinterpret_cast<const ulonglong2 *>(J.R);
            m.S = reinterpret_cast<const ulonglong2 *>(J.S);
            m.nR = J.nR;
            m.nS = J.nS;
            m.cap = nphj_slots(J.nR);
            m.table = reinterpret_cast<ulonglong2 *>(tp);
            tp += m.cap * 16;
            m.side = sides + q;
            m.acc = b->accs + j;
            m.lp = sem_lp(J.algo) ? 1u : 0u;
            m.skip0 = sem_skip0(J.algo) ? 1u : 0u;
            w.any_lp = w.any_lp || m.lp;
            mj[q] = m;
            make_chunks(rch, (unsigned)q, J.nR, kBuildChunk);
            make_chunks(sch, (unsigned)q, J.nS, kProbeChunkMJ);
            rf[q + 1] = rf[q] + J.nR;
            sf[q + 1] = sf[q] + J.nS;
            tf[q + 1] = tf[q] + m.cap;
        }
        w.tables = reinterpret_cast<ulonglong2 *>(tables);
        w.sides = sides;
        w.total_r = rf[w.count];
        w.total_s = sf[w.count];
        w.total_t = tf[w.count];
        w.jobs_dev = reinterpret_cast<hj::MJob *>(cur);
        cur += a256(sizeof(hj::MJob) * w.count);
        w.r_flat = reinterpret_cast<unsigned long long *>(cur);
        cur += a256(8 * (w.count + 1));
        w.s_flat = reinterpret_cast<unsigned long long *>(cur);
        cur += a256(8 * (w.count + 1));
        w.t_flat = reinterpret_cast<unsigned long long *>(cur);
        cur += a256(8 * (w.count + 1));
        w.n_r_chunks = (int)rch.size();
        w.n_s_chunks = (int)sch.size();
        w.r_chunks = reinterpret_cast<hj::MChunk *>(cur);
        cur += a256(sizeof(hj::MChunk) * (rch.size() + 1));
        w.s_chunks = reinterpret_cast<hj::MChunk *>(cur);
        cur += a256(sizeof(hj::MChunk) * (sch.size() + 1));
        if ((rch.size() && cudaMemcpy(w.r_chunks, rch.data(), sizeof(hj::MChunk) * rch.size(), cudaMemcpyHostToDevice) != cudaSuccess) ||
            (sch.size() && cudaMemcpy(w.s_chunks, sch.data(), sizeof(hj::MChunk) * sch.size(), cudaMemcpyHostToDevice) != cudaSuccess))
            return fail(HJ_E_DEVICE);
        if (cudaMemcpy(w.jobs_dev, mj.data(), sizeof(hj::MJob) * w.count, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(w.r_flat, rf.data(), 8 * (w.count + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(w.s_flat, sf.data(), 8 * (w.count + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(w.t_flat, tf.data(), 8 * (w.count + 1), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(HJ_E_DEVICE);
        b->waves.push_back(w);
    }
    b->phj_scratch = cur;
    if (hj::phj_prepare_device()) return fail(HJ_E_DEVICE);
    if (b->use_graph) {
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return fail(HJ_E_DEVICE);
        int rc = enqueue_batch(b);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return fail(rc);
        }
        if (e != cudaSuccess) return fail(HJ_E_DEVICE);
        b->graph = g;
        if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) return fail(HJ_E_DEVICE);
    }
    if (dev_prev >= 0) cudaSetDevice(dev_prev);
    *out = b;
    return HJ_OK;
}

int hj_batch_run(hj_batch_t *b, hj_batch_result_t *results, hj_batch_stats_t *stats) {
    if (!b) return HJ_E_INVAL;
    int dev_prev = -1;
    cudaGetDevice(&dev_prev);
    cudaSetDevice(b->ctx->device);
    int rc = HJ_OK;
    cudaEventRecord(b->e0, b->stream);
    if (b->use_graph) {
        if (cudaGraphLaunch(b->exec, b->stream) != cudaSuccess) rc = HJ_E_DEVICE;
    } else {
        rc = enqueue_batch(b);
    }
    cudaEventRecord(b->e1, b->stream);
    if (!rc && b->njobs)
        if (cudaMemcpyAsync(b->accs_host, b->accs, sizeof(JoinAccum) * b->njobs, cudaMemcpyDeviceToHost, b->stream) !=
            cudaSuccess)
            rc = HJ_E_DEVICE;
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) rc = HJ_E_DEVICE;
    float ms = 0;
    cudaEventElapsedTime(&ms, b->e0, b->e1);
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->seconds = ms * 1e-3;
        stats->kernel_launches = b->launches;
        stats->waves = (int)b->waves.size();
        for (int j = 0; j < b->njobs; j++) stats->nphj_jobs += b->impl[j] == kImplNphj;
        stats->phj_jobs = b->njobs - stats->nphj_jobs;
    }
    for (int j = 0; results && j < b->njobs; j++) {
        hj_batch_result_t &r = results[j];
        r.matched_cnt = rc ? 0 : b->accs_host[j].matched;
        r.checksum = rc ? 0 : b->accs_host[j].checksum;
        const unsigned e = rc ? 0 : b->accs_host[j].error;
        r.status = rc ? rc : (e & hj::kErrSpinLimit ? HJ_E_TIMEOUT : e & hj::kErrProbeLimit ? HJ_E_PROBE_LIMIT : e ? HJ_E_OVERFLOW : HJ_OK);
        r.impl = b->impl[j];
        r.num_radix_bits = b->bits[j];
        r.num_passes = b->passes[j];
    }
    if (dev_prev >= 0) cudaSetDevice(dev_prev);
    return rc;
}

int hj_batch_destroy(hj_batch_t *b) {
    if (!b) return HJ_E_INVAL;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->mem) cudaFree(b->mem);
    if (b->accs_host) cudaFreeHost(b->accs_host);
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (int l = 0; l < kPhjLanes; l++) {
        if (b->stream_phj[l]) cudaStreamDestroy(b->stream_phj[l]);
        if (b->ev_join[l]) cudaEventDestroy(b->ev_join[l]);
    }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    delete b;
    return HJ_OK;
}

int hj_join_batch(hj_ctx_t *c, const hj_batch_job_t *jobs, int njobs, const hj_params_t *p,
                  hj_batch_result_t *results, hj_batch_stats_t *stats) {
    hj_batch_t *b = nullptr;
    int rc = hj_batch_plan(c, jobs, njobs, p, &b);
    if (rc) return rc;
    rc = hj_batch_run(b, results, stats);
    hj_batch_destroy(b);
    return rc;
}

// Calibration: time both implementations on PK-FK joins of growing build size (|S| = 8 |R|) and set
// the table budget to the largest build whose non-partitioned join was faster.
int hj_tuner_calibrate(hj_ctx_t *c, double *report, int report_len) {
    if (!c) return HJ_E_INVAL;
    int dev_prev = -1;
    cudaGetDevice(&dev_prev);
    cudaSetDevice(c->device);
    const int logs[] = {16, 18, 19, 20, 21, 22, 23, 24};
    const int nl = (int)(sizeof(logs) / sizeof(logs[0]));
    const size_t maxR = 1ull << logs[nl - 1], maxS = 8 * maxR;
    hj_tuple_t *R = nullptr, *S = nullptr;
    if (cudaMalloc(&R, maxR * 16) != cudaSuccess || cudaMalloc(&S, maxS * 16) != cudaSuccess) {
        cudaGetLastError();
        if (R) cudaFree(R);
        if (dev_prev >= 0) cudaSetDevice(dev_prev);
        return HJ_E_OOM;
    }
    hj_tuner_t saved = c->tuner;
    hj_tuner_t model = saved;
    int rc = HJ_OK;
    for (int q = 0; q < nl && !rc; q++) {
        const size_t nR = 1ull << logs[q], nS = 8 * nR;
        hj_gen_fast_device(nR, nS, 777 + q, 0, 1, R, S, nullptr);
        cudaDeviceSynchronize();
        double t[2] = {1e30, 1e30}, tb = 1e30, tpr = 1e30;
        for (int impl = 0; impl < 2 && !rc; impl++) {
            hj_params_t p;
            hj_params_init(&p);
            p.device = c->device;
            p.inputs_on_device = 1;
            hj_algo_t algo = HJ_ALGO_NPHJ_SC;
            if (impl == 1) {
                int im, b, ps;
                hj_tuner_t forced = saved;
                forced.nphj_max_table_bytes = 0;
                c->tuner = forced;
                decide(c, nR, nS, &im, &b, &ps);
                c->tuner = saved;
                p.num_radix_bits = b;
                p.num_passes = ps;
                algo = HJ_ALGO_PHJ_RADIX_BC;
            }
            for (int rep = 0; rep < 4; rep++) {
                hj_result_t r;
                rc = hj_join_ctx(c, algo, &p, R, nR, S, nS, &r);
                if (rc) break;
                if (rep > 0 && r.total < t[impl]) {
                    t[impl] = r.total;
                    if (impl == 0) {
                        tb = r.buildpart;
                        tpr = r.probejoin;
                    }
                }
            }
        }
        if (q < HJ_TUNER_LEVELS && !rc) {
            model.level_nR[q] = (double)nR;
            model.nphj_build[q] = tb / (double)nR;
            model.nphj_probe[q] = tpr / (double)nS;
            model.phj[q] = t[1];  // whole time for now: split into fixed + per tuple below
        }
        if (report && 3 * q + 2 < report_len) {
            report[3 * q] = (double)nR;
            report[3 * q + 1] = t[0];
            report[3 * q + 2] = t[1];
        }
    }
    cudaFree(R);
    cudaFree(S);
    if (!rc) {
        // Partitioned joins: the smallest size is dominated by the fixed cost; take as fixed cost what
        // it took beyond the per-tuple rate of the largest size, and charge the rest per tuple.
        const int last = std::min(nl, HJ_TUNER_LEVELS) - 1;
        const double n0 = model.level_nR[0] * 9.0, nl_t = model.level_nR[last] * 9.0;
        const double rate = model.phj[last] / nl_t;
        double fixed = model.phj[0] - n0 * rate;
        if (fixed < 0) fixed = 0;
        model.phj_fixed = fixed;
        for (int q = 0; q <= last; q++) {
            const double n = model.level_nR[q] * 9.0;
            const double per = (model.phj[q] - fixed) / n;
            model.phj[q] = per > 0.25 * rate ? per : 0.25 * rate;
        }
        // The cost model decides per join; the table budget only bounds it to the sizes measured.
        model.nphj_max_table_bytes = (double)nphj_slots(maxR) * 16.0;
        model.calibrated = 1;
        c->tuner = model;
    }
    if (dev_prev >= 0) cudaSetDevice(dev_prev);
    return rc;
}

}  // extern "C"
