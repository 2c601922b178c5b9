/*
 * hjscm.h - C ABI of the B200-native equi-join hot path.
 *
 * The library joins two relations of 16-byte tuples {uint64 key, uint64 row_id} on the key and
 * reports the two numbers every join of the reference reports: the match count and the wrapping
 * 64-bit sum of (r.row_id + s.row_id) over all matches. Four join algorithms are provided under the
 * reference's --algo names:
 *
 *   nphj_sc        non-partitioned join, separate-chaining table, every match counted
 *                  (replaces src/algo/nphj.c:677 nphj_sc)
 *   nphj_lp        non-partitioned join, linear-probing table, first match per probe tuple
 *                  (replaces src/algo/nphj.c:1487 nphj_lp)
 *   phj_radix_bc   radix-partitioned join, bucket-chain partition tables, every match counted
 *                  (replaces src/algo/phj.c:2515 phj_radix_bc -> join_init_run(..., bc_join))
 *   phj_radix_lp   radix-partitioned join, linear-probing partition tables, first match per probe
 *                  (replaces src/algo/phj.c phj_radix_lp -> join_init_run(..., lp_join))
 *
 * phj_radix_sc, phj_radix_hr and phj_radix_hro differ from phj_radix_bc only in the layout of the
 * in-partition table on the CPU (separate-chaining buckets, src/algo/phj.c:683; a histogram-sorted copy
 * of R_p scanned per bucket, phj.c:784; the same scanned with AVX-512, phj.c:881). All three count every
 * match, so their results equal phj_radix_bc's and they run its partition join here.
 * The phj_asymm_radix_* names (src/algo/phj_asymm_radix.c) split the radix bits unevenly between the
 * two passes (hj_params_t.radix_bits_pass1); the partitions, hence the results, do not depend on the
 * split. The bandwidth-regulated names phj_radix_bw_reg_* / phj_asymm_radix_bw_reg_* compute the same
 * results as their unregulated counterparts (src/algo/phj_bw_reg.c:2874-2893).
 *
 * All entry points return an int status (HJ_OK or an HJ_E_* code) instead of exiting, and no entry
 * point frees memory it does not own.
 */
#ifndef HJSCM_H
#define HJSCM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 16-byte tuple, byte-identical to the reference's tuple_t (src/inc/store.h:87-96) at the default
 * TUPLE_T_SIZE of 16: {size_t key; size_t row_id;} packed and 16-byte aligned. */
typedef struct {
    uint64_t key;
    uint64_t row_id;
} hj_tuple_t;

/* Materialised result pair, byte-identical to row_id_pair_t (src/inc/store.h:99-102). */
typedef struct {
    uint64_t r_row_id;
    uint64_t s_row_id;
} hj_pair_t;

typedef enum {
    HJ_ALGO_NPHJ_SC = 0,
    HJ_ALGO_NPHJ_LP = 1,
    HJ_ALGO_PHJ_RADIX_BC = 2,
    HJ_ALGO_PHJ_RADIX_LP = 3,
    HJ_ALGO_PHJ_RADIX_SC = 4,  /* src/algo/phj.c:2523 phj_radix_sc -> sc_join (phj.c:683) */
    HJ_ALGO_PHJ_RADIX_HR = 5,  /* src/algo/phj.c:2527 phj_radix_hr -> hr_join (phj.c:784) */
    HJ_ALGO_PHJ_RADIX_HRO = 6, /* src/algo/phj.c:2532 phj_radix_hro -> hro_join (phj.c:881) */
    HJ_ALGO_COUNT = 7
} hj_algo_t;

/* Status codes. The reference exit()s on every failure (src/main.c:215-218, src/inc/utils.c:501-518). */
enum {
    HJ_OK = 0,
    HJ_E_INVAL = 1,       /* bad argument: unknown algo, unsupported radix bits, NULL pointer ... */
    HJ_E_OOM = 2,         /* device or pinned-host allocation failed */
    HJ_E_DEVICE = 3,      /* a CUDA call failed */
    HJ_E_PROBE_LIMIT = 4, /* a table walk exceeded the table's capacity (full table, absent key) */
    HJ_E_TIMEOUT = 5,     /* a bounded device wait gave up, or the host watchdog expired */
    HJ_E_NOT_FOUND = 6,   /* unknown --algo name */
    HJ_E_IO = 7,          /* a relation file could not be read */
    HJ_E_OVERFLOW = 8,    /* a device-side bound check fired (internal error, results invalid) */
    HJ_E_BUDGET = 9,      /* a request does not fit the serving HBM budget */
    HJ_E_CAPACITY = 10,   /* materialising join: the pair buffer is too small; matched_cnt = pairs needed */
    HJ_E_ROWID = 11       /* materialising join: a matched row id is not a 1-based position of its
                             relation, so the retrieve phase cannot gather it */
};

/* Runtime knobs. The reference fixes these at compile time with -D (CMakeLists.txt:51-373,
 * src/algo/params.h:14-35); here they are per call. */
typedef struct {
    int num_radix_bits;   /* NUM_RADIX_BITS, 1..16; 0 selects 14 */
    int num_passes;       /* NUM_PASSES, 1 or 2; 0 selects 2 */
    int device;           /* CUDA device ordinal */
    int inputs_on_device; /* 1: R and S are device pointers; 0: host pointers (copied inside) */
    void *stream;         /* cudaStream_t to run on; NULL selects the context's own stream */
    uint32_t flags;       /* HJ_F_* bits */
    double table_load;    /* NPHJ global table load factor; 0 selects 0.4 for build relations of up to
                             5 M tuples (about L2-sized tables, where shorter probe chains pay) and 0.5
                             above */
    int radix_bits_pass1; /* two passes: bits of pass 1 (NUM_RADIX_BITS_PASS1 of phj_asymm_radix,
                             src/algo/phj_asymm_radix.h:10-19); 0 selects bits / 2. Clamped to the
                             split where each pass has 1..8 bits. */
    int watchdog_ms;      /* > 0: hj_join / hj_join_ctx return HJ_E_TIMEOUT if the join has not finished
                             after this many milliseconds (its kernels keep running; later calls on the
                             context queue behind them). 0: wait as long as it takes. */
} hj_params_t;

#define HJ_F_NO_TIMING   0x1u /* skip the per-phase CUDA events (buildpart/probejoin stay 0) */
#define HJ_F_PINNED_HOST 0x2u /* host inputs are already page-locked */
#define HJ_F_PHASE_TIMES 0x4u /* also time each kernel group (fills hj_result_t.phase) */
/* Radix joins (two passes, <= 14 bits) from 2^27 tuples run in segment mode: pass 1 writes chains of
 * fixed-size segments and counts the histograms itself, so no histogram pass reads the relations first
 * (if the larger scratch does not fit, the exact-offset pipeline runs). First-match joins (lp) keep each
 * build partition in input order there too: every pass-1 CTA takes a contiguous range of the build
 * relation and ranks it stably. These flags pick the pipeline regardless of size; results are the same. */
#define HJ_F_SEGMENTS    0x20u /* segment mode whenever the algorithm allows it */
#define HJ_F_EXACT       0x40u /* always the histogram pass and exact pass-1 offsets */
/* Radix joins store a tuple as one 8-byte word in the partitions when the widths allow (see
 * HJ_RES_COMPACT_PARTITIONS): the final partitions, and the pass-1 output of segment mode, and of the
 * exact-offset pipeline when its pass-2 units average a full 4096-word tile (smaller units run faster on
 * tuples). HJ_F_WIDE keeps 16-byte tuples in every pass instead; HJ_F_WORDS stores words in every pass
 * whenever the widths allow, whatever the unit sizes. Results are the same. */
#define HJ_F_WIDE        0x80u
#define HJ_F_WORDS       0x200u
/* Test hook for failure detection: the first partition pass of a radix join withholds one tile load,
 * so a bounded device wait (2 s) expires and the join returns HJ_E_TIMEOUT; the context stays usable. */
#define HJ_F_TEST_STALL  0x100u
/* phj_radix_lp keeps the first match in input order among equal build keys. It first runs with the
 * partition passes of phj_radix_bc (no order kept), and the joins note whether any probe tuple matched
 * two build tuples; only then is the first match order-dependent, and the join runs again with ordered
 * passes (each build partition in input order, stable ranks). The context remembers the last build
 * relation (pointer and size) that needed this; its next joins there run ordered at once. Both runs
 * together are one join: one result, and its times include both. Such joins are not replayed from a
 * CUDA graph. HJ_F_ORDERED runs the ordered passes at once. */
#define HJ_F_ORDERED     0x400u

/* hj_result_t.phase[] slots (seconds), filled with HJ_F_PHASE_TIMES. PHJ: histogram, plan, partition
 * pass 1, partition pass 2, shared-memory partition joins, global-memory (large) partition joins
 * (segment mode: no histogram pass, so that slot is 0 and pass 1 includes the counting).
 * NPHJ: build, -, -, -, probe, -. */
enum { HJ_PH_HIST = 0, HJ_PH_PLAN = 1, HJ_PH_PASS1 = 2, HJ_PH_PASS2 = 3, HJ_PH_JOIN = 4, HJ_PH_LARGE = 5,
       HJ_PH_COUNT = 6 };

/* Result of one join. matched_cnt/checksum are the reference's two printed values
 * (`matched_cnt: %zu\tcheck_sum: %zu`, src/algo/phj.c:2206); the times follow its timekeeper_t
 * (src/inc/store.h:74-78): buildpart = partition (PHJ) or build (NPHJ) phase, probejoin = join or
 * probe phase, total = their sum, all in seconds measured with CUDA events on the join's stream. */
typedef struct {
    uint64_t matched_cnt;
    uint64_t checksum;
    double buildpart;
    double probejoin;
    double total;
    double h2d;       /* seconds spent copying host inputs to the device (0 for device inputs) */
    int status;
    int physical_passes; /* partition passes the device ran (PHJ only) */
    uint64_t large_partitions; /* partitions joined through the global-memory path (PHJ only) */
    double phase[HJ_PH_COUNT]; /* per-kernel-group seconds (HJ_F_PHASE_TIMES) */
    uint32_t kernel_launches;  /* kernels this join launched */
    uint32_t flags;            /* HJ_RES_* bits */
    double retrieve;           /* materialising joins: seconds of the retrieve phase (included in total) */
} hj_result_t;

/* hj_result_t.flags: the last partition pass stored the final partitions as 8-byte words
 * (key >> radix bits) << 32 | row id, which the joins read (radix joins without per-match output and
 * without the key-0 rule, when every build key >> radix bits is below 2^31 and every row id below 2^32). */
#define HJ_RES_COMPACT_PARTITIONS 0x1u
/* hj_result_t.flags: segment mode stored the pass-1 chains as 8-byte words (key >> pass-1 bits) << 32 |
 * row id as well (every build key >> pass-1 bits below 2^31, every row id below 2^32), so pass 1 wrote
 * 8 bytes per tuple and pass 2 read 8. */
#define HJ_RES_WORD_PASS1 0x2u
/* hj_result_t.flags: phj_radix_lp ran with ordered partition passes (see HJ_F_ORDERED): asked for, a
 * probe tuple with two build matches in the first run, or an earlier join of the same build relation. */
#define HJ_RES_ORDERED_PASSES 0x4u

typedef struct hj_ctx hj_ctx_t;

/* Fill p with the defaults (14 radix bits, 2 passes, device 0, host inputs). */
void hj_params_init(hj_params_t *p);

/* Human-readable name of a status code. */
const char *hj_status_str(int status);

/* --algo name -> algorithm, the lookup of src/main.c:202-220 (exact strcmp over the algos[] table
 * of src/main.c:72-143, restricted to the names this library implements). */
int hj_algo_from_name(const char *name, hj_algo_t *algo);
const char *hj_algo_name(hj_algo_t algo);

/* Contexts own a CUDA stream, events and a grow-only device scratch arena; joins on one context are
 * serialised, joins on different contexts may run concurrently. */
int hj_ctx_create(int device, hj_ctx_t **out);
int hj_ctx_destroy(hj_ctx_t *ctx);
/* Pre-size the scratch arena for a join of the given shape, so that later joins allocate nothing. */
int hj_ctx_reserve(hj_ctx_t *ctx, hj_algo_t algo, const hj_params_t *p, size_t nR, size_t nS);
/* Bytes of device scratch the context currently holds. */
size_t hj_ctx_scratch_bytes(const hj_ctx_t *ctx);

/* One join, synchronous: returns after the result is on the host. Replaces the body of
 * join_init_run (src/algo/phj.c:1875-2512) and nphj_sc/nphj_lp (src/algo/nphj.c:677,1487) minus
 * their file loading. R and S are caller-owned and never modified. */
int hj_join_ctx(hj_ctx_t *ctx, hj_algo_t algo, const hj_params_t *p,
                const hj_tuple_t *R, size_t nR, const hj_tuple_t *S, size_t nS, hj_result_t *out);

/* hj_join_ctx on a per-device default context (created on first use, guarded by a mutex). */
int hj_join(hj_algo_t algo, const hj_params_t *p,
            const hj_tuple_t *R, size_t nR, const hj_tuple_t *S, size_t nS, hj_result_t *out);

/* Materialising join: the reference's ptr_* joins (src/algo/ptr_phj.c:3100-3114 ptr_phj_radix_bc/lp/
 * sc/hr, src/algo/ptr_nphj.c ptr_nphj_sc/lp). The join writes one hj_pair_t {r.row_id, s.row_id} per
 * match (one per matched probe tuple for the lp algorithms), then a retrieve phase recomputes the
 * checksum as the wrapping sum of R[r_row_id - 1].row_id + S[s_row_id - 1].row_id
 * (src/inc/utils.c:712-724), so row ids must be 1-based positions (the reference's payload_gen_*
 * data; otherwise HJ_E_ROWID). out->total = buildpart + probejoin + retrieve, as the reference times
 * its ptr joins (src/algo/ptr_phj.c:3094-3096).
 *   pairs: NULL keeps the pairs in library scratch (only the count and checksum come back); else
 *   the caller's buffer of pair_cap pairs, in device memory when p->inputs_on_device, else in host
 *   memory (copied back after the join). Pair order is unspecified. If pair_cap is too small the call
 *   returns HJ_E_CAPACITY with out->matched_cnt = the pairs needed. */
int hj_join_mat_ctx(hj_ctx_t *ctx, hj_algo_t algo, const hj_params_t *p, const hj_tuple_t *R, size_t nR,
                    const hj_tuple_t *S, size_t nS, hj_pair_t *pairs, size_t pair_cap, hj_result_t *out);
int hj_join_mat(hj_algo_t algo, const hj_params_t *p, const hj_tuple_t *R, size_t nR, const hj_tuple_t *S,
                size_t nS, hj_pair_t *pairs, size_t pair_cap, hj_result_t *out);

/* Streamed join for relations beyond what hj_join holds in device memory (both relations plus two
 * partition buffers): the build relation R is copied to the device once, the probe relation S streams
 * from host memory in chunks of chunk_tuples (0: the largest that fits) through two device buffers, so
 * the copy of one chunk overlaps the join of the previous one; each chunk is joined with all of R and
 * the counts and checksums add up to hj_join's result. R and S are host pointers (pinned memory copies
 * at full link speed), p->inputs_on_device must be 0. out->total covers the copies and the joins. This
 * is the device-side counterpart of the reference's billion-scale workloads (2^30 x 2^34 tuples,
 * config/billion-data), whose probe side no single device holds. */
int hj_join_streamed(hj_ctx_t *ctx, hj_algo_t algo, const hj_params_t *p, const hj_tuple_t *R, size_t nR,
                     const hj_tuple_t *S, size_t nS, size_t chunk_tuples, hj_result_t *out);

/* ----------------------------------------------------------------------------------------------
 * Data generation. The seeded generators replay the reference's src/gen.c exactly (glibc srand/rand,
 * Knuth shuffle), so the relations are byte-identical to the .bin files bin/gen writes.
 * payload = 0: row_id = key (gen_pkfk_uniform, src/gen.c:199-223);
 * payload = 1: row_id = 1-based position (payload_gen_pkfk_uniform, src/gen.c:258-283).
 * Reference constraints kept: nS must be a multiple of nR and nR*16 a multiple of 4096
 * (src/gen.c:178-179 copy FK blocks of 4096 bytes), else HJ_E_INVAL.
 * -------------------------------------------------------------------------------------------- */
int hj_gen_pkfk_uniform(size_t nR, size_t nS, unsigned seed, int payload, hj_tuple_t *R, hj_tuple_t *S);
/* gen_dup_uniform (src/gen.c:286-331): R keys uniform in [1, nR] from a Park-Miller stream, S = FK
 * copies of R, both shuffled. */
int hj_gen_dup_uniform(size_t nR, size_t nS, unsigned seed, hj_tuple_t *R, hj_tuple_t *S);
/* gen_fk_zipfian_eth -> gen_zipf (src/gen.c:375-391, src/inc/eth_genzipf.c:31-147): S keys Zipf over
 * an alphabet of nR keys with the given zipf factor, row_id = position. The reference passes
 * 1 + theta as the factor; this function takes the factor itself. */
int hj_gen_zipf(size_t nS, size_t nR, double zipf_factor, unsigned seed, hj_tuple_t *S);

/* Parallel seeded generators with the reference's value distributions, for sizes where the
 * sequential shuffle is too slow. Keys of R are a seeded permutation of 1..nR (a Feistel bijection
 * with cycle walking); S holds each of R's keys nS/nR times (+1 for the first nS%nR keys of a second
 * bijection) in seeded order. row_id follows `payload` as above. dup > 1 makes R keys repeat: R holds
 * keys 1..ceil(nR/dup) (the FK side draws from those); payload is forced to positions then.
 * The host version runs on `threads` threads (0 = all cores); the device version runs on `stream`
 * and writes device pointers. Both produce identical bytes. */
int hj_gen_fast_host(size_t nR, size_t nS, uint64_t seed, int payload, unsigned dup, int threads,
                     hj_tuple_t *R, hj_tuple_t *S);
int hj_gen_fast_device(size_t nR, size_t nS, uint64_t seed, int payload, unsigned dup,
                       hj_tuple_t *R_dev, hj_tuple_t *S_dev, void *stream);
/* Zipf FK keys over an alphabet of nR keys drawn with a counter-based uniform stream on the device
 * (same alphabet permutation / CDF-table / binary-search rule as gen_zipf); row_id = position. */
int hj_gen_zipf_device(size_t nS, size_t nR, double zipf_factor, uint64_t seed,
                       hj_tuple_t *S_dev, void *stream);

/* Closed-form result of a PK-FK join on hj_gen_pkfk_uniform / hj_gen_fast_* data with payload 0 and
 * nS a multiple of nR: matched = nS, checksum = m*n*(n+1) mod 2^64 with m = nS/nR. */
void hj_pkfk_closed_form(size_t nR, size_t nS, uint64_t *matched, uint64_t *checksum);

/* ----------------------------------------------------------------------------------------------
 * Batched joins: many independent joins of uneven sizes as one captured launch sequence. The
 * reference runs one join per invocation (src/main.c:429-448); this layer has no counterpart there.
 * An autotuner decides per join between the non-partitioned join (global table) and the
 * radix-partitioned pipeline with its own radix bits; results always equal the named algorithm's.
 * -------------------------------------------------------------------------------------------- */
#define HJ_F_NO_GRAPH 0x8u /* batches: launch the kernels one by one instead of one captured graph */
#define HJ_F_TUNE 0x10u    /* batches: plan under a few table budgets around the tuner's, time each plan
                              on the device (the joins run), keep the fastest and its budget */

#define HJ_TUNER_LEVELS 8

typedef struct {
    double nphj_max_table_bytes; /* joins whose global table (32 B per build tuple) fits run as nphj */
    double wave_table_bytes;     /* table bytes per wave of non-partitioned joins (a share of L2) */
    int partition_target;        /* partitioned joins: radix bits so build partitions hold ~this many */
    int calibrated;              /* 1 after hj_tuner_calibrate: the cost model below decides */
    /* Cost model measured by hj_tuner_calibrate at |R| = level_nR[i] (|S| = 8|R|): seconds per build
     * tuple and per probe tuple of the non-partitioned join, seconds per tuple of the partitioned one
     * beyond its fixed cost phj_fixed (the pipeline's ten-odd kernels). A join of (nR, nS) takes the
     * level of its build size and runs non-partitioned when
     * nR * nphj_build + nS * nphj_probe <= phj_fixed + (nR + nS) * phj (and its table fits
     * nphj_max_table_bytes). */
    double level_nR[HJ_TUNER_LEVELS];
    double nphj_build[HJ_TUNER_LEVELS], nphj_probe[HJ_TUNER_LEVELS], phj[HJ_TUNER_LEVELS];
    double phj_fixed;
} hj_tuner_t;

typedef struct {
    hj_algo_t algo;              /* result semantics: the reference algorithm the join stands for */
    const hj_tuple_t *R;         /* device pointers */
    size_t nR;
    const hj_tuple_t *S;
    size_t nS;
} hj_batch_job_t;

typedef struct {
    uint64_t matched_cnt;
    uint64_t checksum;
    int status;                  /* HJ_OK or an HJ_E_* code for this join */
    int impl;                    /* what ran: 0 = non-partitioned table, 1 = radix-partitioned */
    int num_radix_bits;          /* radix-partitioned joins: bits and passes chosen */
    int num_passes;
} hj_batch_result_t;

typedef struct {
    double seconds;              /* device time of the whole batch (CUDA events) */
    uint32_t kernel_launches;    /* kernels the batch launches */
    int waves;                   /* waves of non-partitioned joins */
    int nphj_jobs, phj_jobs;
} hj_batch_stats_t;

typedef struct hj_batch hj_batch_t;

int hj_tuner_get(hj_ctx_t *ctx, hj_tuner_t *out);
int hj_tuner_set(hj_ctx_t *ctx, const hj_tuner_t *in);
/* Decision for one join of the given sizes (impl 0/1 as in hj_batch_result_t). */
int hj_tuner_decide(hj_ctx_t *ctx, size_t nR, size_t nS, int *impl, int *bits, int *passes);
/* For single joins (hj_tuner_decide, the server): time both implementations on PK-FK joins with
 * |S| = 8|R|, |R| = 2^16..2^24: fills the cost model
 * (per-tuple build and probe costs of the non-partitioned join, per-tuple cost of the partitioned one)
 * and sets the table budget to the largest table measured. report (optional) receives triples
 * (|R|, seconds non-partitioned, seconds partitioned). Allocates temporary device memory. */
int hj_tuner_calibrate(hj_ctx_t *ctx, double *report, int report_len);
/* Plan a batch: decisions, device memory for all of it, and (unless HJ_F_NO_GRAPH) the captured
 * graph. The relations must stay valid and unchanged in place until hj_batch_destroy. */
int hj_batch_plan(hj_ctx_t *ctx, const hj_batch_job_t *jobs, int njobs, const hj_params_t *p, hj_batch_t **out);
/* Run a planned batch (one graph launch), wait, and fill one result per job. */
int hj_batch_run(hj_batch_t *b, hj_batch_result_t *results, hj_batch_stats_t *stats);
int hj_batch_destroy(hj_batch_t *b);
/* plan + run + destroy */
int hj_join_batch(hj_ctx_t *ctx, const hj_batch_job_t *jobs, int njobs, const hj_params_t *p,
                  hj_batch_result_t *results, hj_batch_stats_t *stats);

/* ----------------------------------------------------------------------------------------------
 * Allocation-free join. This entry point has no counterpart in the reference, whose joins allocate
 * their tables per call (src/algo/nphj.c:745-757).
 *
 * Some callers cannot allocate device memory: a host engine that has already reserved the GPU's memory
 * for its own buffer pool, or a request loop that must not call the CUDA allocator (cudaMalloc and
 * cudaFree synchronise the device and have unbounded latency). hj_nphj_join_noalloc runs nphj_sc or
 * nphj_lp on device-resident relations with its hash table in a fixed 16 MiB array that is part of the
 * library image (every GPU that loads the library holds it until the process exits); it calls no
 * allocator. Limits and rules:
 *   - nR (build side) <= 524286 tuples; larger builds return HJ_E_INVAL with a message on stderr.
 *   - R_dev, S_dev: device pointers; out_dev: a caller-owned device hj_device_result_t, zeroed and then
 *     filled on `stream` (cudaStream_t, NULL = legacy default stream); the call only enqueues work.
 *   - The first call on a device looks up the array's device address (once per device, with that device
 *     current); make that first call before any stream capture.
 *   - All calls share the one array and each clears it on its stream; calls whose GPU work overlaps
 *     (different streams or host threads) race and must be serialised by the caller.
 *   - After the stream completes, out_dev->error_bits != 0 means the result is invalid (1: a probe
 *     walked the whole table, 4: an index fell outside its buffer).
 * -------------------------------------------------------------------------------------------- */
typedef struct {
    uint64_t matched_cnt;
    uint64_t checksum;
    uint32_t error_bits;
    uint32_t reserved0;
    uint64_t reserved[5];
} hj_device_result_t;

int hj_nphj_join_noalloc(hj_algo_t algo, const hj_tuple_t *R_dev, size_t nR, const hj_tuple_t *S_dev,
                         size_t nS, hj_device_result_t *out_dev, void *stream);

/* ----------------------------------------------------------------------------------------------
 * Sharded joins over several GPUs (one process per GPU). The reference runs on one machine's threads
 * and has no counterpart; its co-partitions are independent (src/algo/phj.c:1257-1311), so a join
 * shards by key with one exchange step. hj_shard_route groups the n tuples of in_dev (device) by owner
 * rank, owner = mulhi(mix64(key ^ 0x5ca1ab1e5eed0001), nshards) with mix64 the splitmix64 output mix,
 * into out_dev (n tuples, device), stably (input order kept within each owner's range), and writes
 * the owners' tuple counts to counts_dev (nshards u64, device). All work is enqueued on `stream`;
 * scratch_dev (device) holds hj_shard_route_scratch_bytes(n, nshards) bytes. nshards: 1..32.
 * The exchange itself (all-to-all of counts, then of tuples) and the sum of the local results are
 * collective calls of the caller's communication library (the Python layer uses torch.distributed).
 * -------------------------------------------------------------------------------------------- */
size_t hj_shard_route_scratch_bytes(size_t n, int nshards);
int hj_shard_route(const hj_tuple_t *in_dev, size_t n, int nshards, hj_tuple_t *out_dev, uint64_t *counts_dev,
                   void *scratch_dev, size_t scratch_bytes, void *stream);

/* ----------------------------------------------------------------------------------------------
 * Join server: requests arrive at any time and are served concurrently under an HBM budget. The
 * reference runs one join per process (src/main.c:429-448); this layer has no counterpart there.
 *   - hj_server_create allocates one device pool of hbm_budget_bytes (capped at 92% of the free device
 *     memory) and `slots` CUDA streams; serving then calls no CUDA allocator.
 *   - hj_server_submit queues a join and returns at once. Each admitted request takes its scratch (and
 *     the device copies of host relations) from the pool and returns it on completion; a request is
 *     admitted when a slot and its memory are free, first come first served, except that later requests
 *     may pass a head that does not fit yet while the head has waited less than 50 ms. A request that
 *     can never fit the pool is refused at submission with HJ_E_BUDGET.
 *   - The relations (host or device, as inputs_on_device says) must stay valid and unchanged until the
 *     request's completion has been polled.
 *   - Each request runs the implementation the autotuner picks for its sizes (or, with autotune = 0,
 *     the named algorithm at 14 radix bits / 2 passes) with the named algorithm's result semantics, so
 *     its result is the same as hj_join's, alone or in any mix.
 *   - Continuous batching (waves = 1, the default): requests that run as non-partitioned joins are not
 *     given slots of their own. At each dispatch, the ones queued (up to wave_max_requests, their
 *     tables within the tuner's wave_table_bytes) are coalesced into one wave - one multi-join build
 *     and one multi-join probe launch over all of them, on a high-priority stream - whose memory is one
 *     block of the pool. Two waves can be on the GPU at once; requests that arrive while they run form
 *     the next wave. Partitioned (large) requests keep their slots and overlap the waves.
 * -------------------------------------------------------------------------------------------- */
typedef struct {
    int device;
    int slots;                   /* requests on the GPU at once (1..256), one stream each */
    double hbm_budget_bytes;     /* device pool size */
    int autotune;                /* 1: per-request implementation from the tuner (default) */
    hj_tuner_t tuner;            /* used when tuner.partition_target > 0, else the context defaults */
    double small_request_tuples; /* requests with |R| + |S| <= this run on high-priority streams */
    double large_sm_share;       /* larger requests launch their kernels sized for this share of the SMs
                                    (0..1], leaving room for small requests' blocks; 1 = all SMs */
    int waves;                   /* 1: coalesce non-partitioned requests into waves (default); 0: one slot
                                    per request */
    int wave_max_requests;       /* requests per wave (1..1024; default 512) */
    int max_large_inflight;      /* larger requests on the GPU at once; 0 = no limit (default) */
} hj_server_config_t;

typedef struct {
    uint64_t id;
    uint64_t matched_cnt;
    uint64_t checksum;
    int status;                  /* HJ_OK or an HJ_E_* code */
    int impl;                    /* 0 = non-partitioned table, 1 = radix-partitioned */
    double submit_s, start_s, done_s; /* hj_now() clock: submission, admission, completion seen */
    uint64_t wave;               /* 0: ran on a slot of its own; else the id (1, 2, ...) of its wave */
    int wave_size;               /* requests in that wave */
    int reserved;
} hj_server_completion_t;

typedef struct {
    uint64_t submitted, admitted, completed;
    double budget_bytes, in_use_bytes, peak_in_use_bytes;
    int queued, inflight;        /* inflight: requests on slots and in waves */
    uint64_t waves, wave_requests; /* waves launched and the requests they carried */
} hj_server_stats_t;

typedef struct hj_server hj_server_t;

/* Monotonic clock in seconds, the one completions are stamped with. */
double hj_now(void);
/* Defaults: device 0, 8 slots, 150e9 bytes, autotune (non-partitioned joins up to 16 MB tables), small
 * requests up to 2^25 tuples, large requests on 0.75 of the SMs, waves of up to 512 requests and 1e9
 * bytes of tables. */
int hj_server_config_init(hj_server_config_t *cfg);
int hj_server_create(const hj_server_config_t *cfg, hj_server_t **out);
int hj_server_submit(hj_server_t *srv, hj_algo_t algo, const hj_tuple_t *R, size_t nR, const hj_tuple_t *S,
                     size_t nS, int inputs_on_device, uint64_t *id);
/* Up to max completions into out (*n of them); waits up to wait_ms for the first when none is ready. */
int hj_server_poll(hj_server_t *srv, hj_server_completion_t *out, int max, int *n, int wait_ms);
int hj_server_stats(hj_server_t *srv, hj_server_stats_t *out);
/* Serves what is queued, waits for it, and frees everything; completions not polled are dropped. */
int hj_server_destroy(hj_server_t *srv);

#ifdef __cplusplus
}
#endif

#endif /* HJSCM_H */
