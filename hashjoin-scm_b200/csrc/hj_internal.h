// hj_internal.h - host-side interfaces between the C ABI layer and the kernel launchers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/hjscm.h"

namespace hj {

struct JoinAccum;
struct MatOut;

// Geometry of the radix plan: total bits B split into physical passes of <= 8 bits each
// (src/algo/params.h:34-35: FANOUT_PASS1 = 1 << (B/P), FANOUT_PASS2 = 1 << (B - B/P)).
struct RadixGeom {
    int bits;       // B
    int passes;     // physical passes (1 or 2)
    int b1, b2;     // bits of pass 1 / pass 2 (b2 = 0 for one pass)
    int F1, F2;     // fanouts (F2 = 1 for one pass)
    int nparts() const { return 1 << bits; }
};

// Record `ev` on `st`. While the stream is being captured into a CUDA graph the record becomes an
// event-record node (recorded at every launch of the graph, so its timings stay readable); a plain
// cudaEventRecord there would only order the capture.
inline cudaError_t record_event(cudaEvent_t ev, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusActive)
        return cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal);
    return cudaEventRecord(ev, st);
}

// b1_req > 0 asks for that many pass-1 bits (clamped so that both passes have 1..8 bits).
int radix_geom(int bits, int passes, RadixGeom *g, int b1_req = 0);

// Result semantics of an algorithm: radix-partitioned or not; first match per probe tuple (lp) or
// every match; build key 0 never matches (the phj_radix_lp empty-slot rule, src/algo/phj.c:614).
inline bool algo_is_phj(hj_algo_t a) { return a >= HJ_ALGO_PHJ_RADIX_BC && a < HJ_ALGO_COUNT; }
inline bool algo_lp(hj_algo_t a) { return a == HJ_ALGO_NPHJ_LP || a == HJ_ALGO_PHJ_RADIX_LP; }
inline bool algo_skip0(hj_algo_t a) { return a == HJ_ALGO_PHJ_RADIX_LP; }

// Tile and work-item constants shared by the plan and the kernels.
constexpr int kScatterThreads = 256;
constexpr int kScatterItems = 8;
constexpr int kScatterBufs = 2;       // tile buffers per CTA (2: double-buffered TMA loads)
constexpr int kScatterCtasPerSm = 3;  // resident scatter CTAs per SM (registers and shared memory)
constexpr int kScatterWordCtasPerSm = 2;  // pass 2 over 8-byte words: 16 words per thread, up to 128 registers
constexpr int kTile = kScatterThreads * kScatterItems;  // tuples per partition tile
constexpr int kJoinThreads = 1024;
constexpr int kSmemCap = 10240;        // largest build partition joined in shared memory
constexpr int kProbeChunk = 1 << 16;   // S tuples per join work item

// Device scratch layout of one partitioned join, carved out of a context arena.
struct PhjScratch {
    uint64_t chunk;          // tuples per input chunk
    uint32_t cR, cS;         // chunks of R and of S
    uint64_t sub;            // tuples per sub-chunk (pass-1 work item)
    uint32_t spc;            // sub-chunks per chunk
    uint32_t *chunk_hist;    // [chunk][2^B] joint digit histogram of each chunk
    uint32_t *prefix;        // [chunk][2^B] exclusive prefix over the chunks of the same relation
    uint32_t *total;         // [2][2^B]
    uint64_t *start;         // [2][2^B + 1] final partition starts
    uint64_t *unit_off;      // [chunk][F1] start of (chunk, d1) in the pass-1 output
    uint32_t *unit_cnt;      // [chunk][F1] its size
    uint32_t *subhist;       // [chunk][spc][F1] pass-1 digit histogram of each sub-chunk, then its start
                             // within (chunk, d1)
    uint32_t *counters;      // work-item counters, totals, error word (memset per join)
    void *items;             // join work items
    size_t max_items;
    void *large;             // large-partition descriptors
    size_t max_large;
    uint32_t *large_table;   // head/next chains for large partitions (>= 12 B per R tuple)
    size_t large_table_words;
    ulonglong2 *tmp1;        // pass-1 output [nR + nS]; segment storage [max_segs * kTile] in segment mode
    ulonglong2 *tmp2;        // pass-2 output [nR + nS] (== tmp1 for one pass)
    // Segment mode (phj_seg_applies): pass 1 writes chains of kTile-tuple segments and counts the
    // histograms itself, so no histogram pass reads the relations first. "Chunks" are then the pass-1
    // CTAs: cR = cS = seg_grid.
    bool seg;
    uint32_t seg_grid;       // pass-1 CTAs
    uint32_t max_segs;       // segments that tmp1 holds
    uint32_t it_tiles;       // tiles per pass-1 work item
    uint32_t *seg_head;      // [2 * seg_grid][F1] first segment of (CTA, relation, pass-1 digit)
    uint32_t *seg_next;      // [max_segs] next segment of the same chain
};

// Segment mode applies to the joins that count every match (the order of tuples within a partition
// does not matter), two physical passes, at most 14 radix bits, and relations large enough that the
// histogram read it saves outweighs the memory it reserves (one partly filled segment per CTA,
// relation and pass-1 digit).
bool phj_seg_applies(const RadixGeom &g, bool lp, size_t nR, size_t nS);

// Kernel attributes (dynamic shared memory limits) for the current device; phj_enqueue calls it too,
// but callers that capture a stream into a graph call it before the capture.
int phj_prepare_device();

// seg: lay the scratch out for segment mode (callers pass phj_seg_applies(...) or false).
size_t phj_scratch_bytes(const RadixGeom &g, size_t nR, size_t nS, int num_sms, bool seg = false);
void phj_carve(const RadixGeom &g, size_t nR, size_t nS, int num_sms, char *base, PhjScratch *s, bool seg = false);

// Result semantics: lp = first match per probe tuple (lowest build position) instead of all matches;
// skip0 = build tuples with key 0 never match (the phj_radix_lp empty-slot rule, src/algo/phj.c:614).
// Enqueue a full partitioned join on `st`; matches/checksum accumulate into acc (zeroed by caller).
// ev_mid, if non-null, is recorded between the partition phase and the join phase.
// ph, if non-null, holds HJ_PH_COUNT + 1 events recorded at the phase boundaries (in segment mode,
// see phj_phase_span, in a different order); *launches receives the number of kernels enqueued.
// A scratch carved for segment mode runs in segment mode, else the exact-offset pipeline.
// mat, if non-null, makes the join write one (r.row_id, s.row_id) pair per match into mat->pairs
// (slots counted in acc->pairs) instead of summing row ids. test_flags bit 0: the partition pass's
// first CTA withholds one tile load, so its bounded wait expires (failure-detection tests); bit 1:
// 16-byte tuples in every pass; bit 2: 8-byte words in every pass the widths allow.
// ordered (first-match joins, lp): true keeps each final build partition in input order (stable ranks),
// so the lowest position among equal keys is the first in input order. false ranks the build relation
// as the all-matches joins do; the result is then right unless a probe tuple matched two build tuples,
// which the joins record in acc->dup_flag: the caller then runs the join again with ordered = true.
int phj_enqueue(const RadixGeom &g, bool lp, bool skip0, const ulonglong2 *R, size_t nR, const ulonglong2 *S,
                size_t nS, const PhjScratch &s, JoinAccum *acc, cudaStream_t st, cudaEvent_t ev_mid,
                int num_sms, cudaEvent_t *ph, uint32_t *launches, const MatOut *mat = nullptr,
                int test_flags = 0, bool ordered = true);

// The events of phase slot i (HJ_PH_*) that phj_enqueue recorded: elapsed(ph[*from], ph[*to]);
// false for a slot that the mode does not time (segment mode has no histogram pass).
inline bool phj_phase_span(bool seg_mode, int i, int *from, int *to) {
    if (!seg_mode) {
        *from = i;
        *to = i + 1;
        return true;
    }
    // Segment mode records: start, pass 1, plan, pass 2, joins, large joins.
    static const int kFrom[HJ_PH_COUNT] = {-1, 1, 0, 2, 3, 4};
    if (i < 0 || i >= HJ_PH_COUNT || kFrom[i] < 0) return false;
    *from = kFrom[i];
    *to = kFrom[i] + 1;
    return true;
}

// Non-partitioned joins on a global open-addressing table.
// mat: as for phj_enqueue; a materialising join needs nphj_scratch_bytes(nR, load, true).
size_t nphj_scratch_bytes(size_t nR, double load, bool mat = false);
// The load factor a table_load of 0 (or outside (0.05, 0.95)) selects for a build relation of nR tuples.
double nphj_default_load(size_t nR);
// Shared-memory attributes of the non-partitioned join's kernels on the current device (idempotent;
// call before capturing nphj_enqueue in a graph).
int nphj_prepare_device();
// phases: kNphjBuild and/or kNphjProbe. A probe-only call probes the table an earlier build-only call
// on the same table memory (same R, nR, table, table_bytes, load) left there; its results add to acc.
constexpr int kNphjBuild = 1, kNphjProbe = 2;
int nphj_enqueue(bool lp, bool skip0, const ulonglong2 *R, size_t nR, const ulonglong2 *S, size_t nS, void *table,
                 size_t table_bytes, double load, JoinAccum *acc, cudaStream_t st, cudaEvent_t ev_mid,
                 int num_sms, cudaEvent_t *ph, uint32_t *launches, const MatOut *mat = nullptr,
                 int phases = kNphjBuild | kNphjProbe);

// Checksum of materialised pairs as the reference's retrieve phase computes it: the wrapping sum of
// R[r_row_id - 1].row_id + S[s_row_id - 1].row_id over the first n pairs (into acc->checksum).
int mat_retrieve_enqueue(const ulonglong2 *pairs, const unsigned long long *n_dev, unsigned long long cap,
                         const ulonglong2 *R, size_t nR, const ulonglong2 *S, size_t nS, JoinAccum *acc,
                         cudaStream_t st, int num_sms);

}  // namespace hj
