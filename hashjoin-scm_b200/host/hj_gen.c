/*
 * hj_gen.c - relation generators.
 *
 * 1. Exact replays of the reference's bin/gen (src/gen.c), so that a seed gives byte-identical
 *    relations. The reference calls srand(seed) before each dataset and draws with glibc rand()
 *    (src/gen.c:70-92, 144). Here the same stream comes from a private glibc random_r state of the
 *    default 128-byte (TYPE_3) size seeded through initstate_r, which is the generator srand/rand use;
 *    the process-wide rand() state is left alone.
 * 2. Parallel generators with the same value distributions (hj_feistel.h), for full-size runs.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../../include/hjscm.h"
#include "hj_feistel.h"

typedef struct {
    struct random_data rd;
    char state[128];
} hj_rng_t;

static void rng_seed(hj_rng_t *g, unsigned seed) {
    memset(g, 0, sizeof(*g));
    initstate_r(seed, g->state, sizeof(g->state), &g->rd);
}

static int rng_next(hj_rng_t *g) {
    int32_t r;
    random_r(&g->rd, &r);
    return (int)r;
}

/* knuth_shuffle (src/gen.c:161-171): for i in 0..n-1, j = rand() % n, swap(t[i], t[j]). */
static void knuth_shuffle(hj_rng_t *g, hj_tuple_t *t, size_t n) {
    for (size_t i = 0; i < n; i++) {
        size_t j = (size_t)rng_next(g) % n;
        hj_tuple_t tmp = t[j];
        t[j] = t[i];
        t[i] = tmp;
    }
}

/* gen_fk_from_pk (src/gen.c:174-196): nS/nR back-to-back copies of the shuffled PK array, then one
 * shuffle of the whole FK array. */
static void fk_from_pk(hj_rng_t *g, const hj_tuple_t *R, size_t nR, hj_tuple_t *S, size_t nS) {
    for (size_t c = 0; c < nS / nR; c++) memcpy(S + c * nR, R, nR * sizeof(hj_tuple_t));
    knuth_shuffle(g, S, nS);
}

static int exact_sizes_ok(size_t nR, size_t nS) {
    /* The reference copies in 4096-byte blocks (src/gen.c:179), so nR*16 must be a multiple of 4096,
     * and copies ceil(nS/nR) times into an nS buffer (src/gen.c:178), so nS must be a multiple of nR. */
    if (nR == 0 || nS == 0) return 0;
    if ((nR * sizeof(hj_tuple_t)) % 4096 != 0) return 0;
    if (nS % nR != 0) return 0;
    return 1;
}

int hj_gen_pkfk_uniform(size_t nR, size_t nS, unsigned seed, int payload, hj_tuple_t *R, hj_tuple_t *S) {
    if (!R || !S || !exact_sizes_ok(nR, nS)) return HJ_E_INVAL;
    hj_rng_t g;
    rng_seed(&g, seed);
    /* gen_pkfk_uniform (src/gen.c:199-223) / payload_gen_pkfk_uniform (src/gen.c:258-283) */
    for (size_t i = 0; i < nR; i++) {
        R[i].key = i + 1;
        R[i].row_id = i + 1;
    }
    knuth_shuffle(&g, R, nR);
    fk_from_pk(&g, R, nR, S, nS);
    if (payload) {
        /* payload_gen_fk_from_pk sets S row ids to positions (src/gen.c:243-245), then the caller sets
         * R row ids to positions (src/gen.c:276-278); keys are unaffected. */
        for (size_t j = 0; j < nS; j++) S[j].row_id = j + 1;
        for (size_t i = 0; i < nR; i++) R[i].row_id = i + 1;
    }
    return HJ_OK;
}

int hj_gen_dup_uniform(size_t nR, size_t nS, unsigned seed, hj_tuple_t *R, hj_tuple_t *S) {
    if (!R || !S || !exact_sizes_ok(nR, nS)) return HJ_E_INVAL;
    hj_rng_t g;
    rng_seed(&g, seed);
    /* gen_dup_uniform (src/gen.c:286-331): a Park-Miller minimal-standard stream (16807, 2^31-1 via
     * Schrage's method) seeded by rand() % RAND_MAX, mapped by rounding onto [min_key, max_key]. */
    const int i4_huge = 2147483647;
    int uni = rng_next(&g) % RAND_MAX;
    const uint64_t min_key = 1, max_key = nR;
    for (size_t i = 0; i < nR; i++) {
        int k = uni / 127773;
        uni = 16807 * (uni - k * 127773) - k * 2836;
        if (uni < 0) uni += i4_huge;
        double r = (double)uni * 4.656612875E-10;
        r = (1.0 - r) * ((double)min_key - 0.5) + r * ((double)max_key + 0.5);
        uint64_t key = (uint64_t)(int)round(r);
        if (key < min_key) key = min_key;
        if (key > max_key) key = max_key;
        R[i].key = key;
        R[i].row_id = i + 1;
    }
    knuth_shuffle(&g, R, nR);
    fk_from_pk(&g, R, nR, S, nS);
    return HJ_OK;
}

int hj_gen_zipf(size_t nS, size_t nR, double zipf_factor, unsigned seed, hj_tuple_t *S) {
    if (!S || nR == 0) return HJ_E_INVAL;
    hj_rng_t g;
    rng_seed(&g, seed);
    /* gen_alphabet (src/inc/eth_genzipf.c:31-54): 1..n permuted by kdx = idx * rand() / RAND_MAX
     * from the top index down. */
    uint64_t *alphabet = (uint64_t *)malloc(nR * sizeof(uint64_t));
    double *lut = (double *)malloc(nR * sizeof(double));
    if (!alphabet || !lut) {
        free(alphabet);
        free(lut);
        return HJ_E_OOM;
    }
    for (size_t i = 0; i < nR; i++) alphabet[i] = i + 1;
    for (size_t i = nR - 1; i > 0; i--) {
        size_t k = (size_t)i * (size_t)rng_next(&g) / RAND_MAX;
        uint64_t t = alphabet[i];
        alphabet[i] = alphabet[k];
        alphabet[k] = t;
    }
    /* gen_zipf_lut (src/inc/eth_genzipf.c:61-91): cumulative 1/i^f normalised by the same sum. */
    double scale = 0.0;
    for (size_t i = 1; i <= nR; i++) scale += 1.0 / pow((double)i, zipf_factor);
    double sum = 0.0;
    for (size_t i = 1; i <= nR; i++) {
        sum += 1.0 / pow((double)i, zipf_factor);
        lut[i - 1] = sum / scale;
    }
    /* gen_zipf (src/inc/eth_genzipf.c:97-147): r = rand()/RAND_MAX; position 0 if lut[0] >= r, else
     * the bisection over (left = 1, right = n] that returns `right`. */
    for (size_t j = 0; j < nS; j++) {
        double r = (double)rng_next(&g) / RAND_MAX;
        size_t pos;
        if (lut[0] >= r) {
            pos = 0;
        } else {
            size_t left = 1, right = nR;
            while (right - left > 1) {
                size_t m = (left + right) / 2;
                if (lut[m] < r)
                    left = m;
                else
                    right = m;
            }
            pos = right;
        }
        /* The bisection cannot reach n: lut[n-1] == 1.0 exactly and r <= 1.0. Guard anyway. */
        if (pos >= nR) pos = nR - 1;
        S[j].key = alphabet[pos];
        S[j].row_id = j + 1;
    }
    free(alphabet);
    free(lut);
    return HJ_OK;
}

/* ------------------------------------------------------------------------------------------------ */

typedef struct {
    hj_feistel_t fr, fs;
    uint64_t distinct;
    int payload;
    hj_tuple_t *R, *S;
    size_t nR, nS;
    int tid, nthreads;
} fast_arg_t;

static void *fast_worker(void *p) {
    fast_arg_t *a = (fast_arg_t *)p;
    size_t r0 = a->nR * a->tid / a->nthreads, r1 = a->nR * (a->tid + 1) / a->nthreads;
    for (size_t i = r0; i < r1; i++) hj_fast_r_tuple(&a->fr, a->distinct, a->payload, i, &a->R[i].key, &a->R[i].row_id);
    size_t s0 = a->nS * a->tid / a->nthreads, s1 = a->nS * (a->tid + 1) / a->nthreads;
    for (size_t j = s0; j < s1; j++) hj_fast_s_tuple(&a->fs, a->distinct, a->payload, j, &a->S[j].key, &a->S[j].row_id);
    return NULL;
}

int hj_gen_fast_host(size_t nR, size_t nS, uint64_t seed, int payload, unsigned dup, int threads,
                     hj_tuple_t *R, hj_tuple_t *S) {
    if (nR == 0 || (!R) || (nS && !S)) return HJ_E_INVAL;
    if (dup == 0) dup = 1;
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    fast_arg_t *args = (fast_arg_t *)calloc((size_t)threads, sizeof(fast_arg_t));
    pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    if (!args || !th) {
        free(args);
        free(th);
        return HJ_E_OOM;
    }
    uint64_t distinct = (nR + dup - 1) / dup;
    for (int t = 0; t < threads; t++) {
        hj_feistel_init(&args[t].fr, nR, HJ_GEN_SEED_R(seed));
        hj_feistel_init(&args[t].fs, nS ? nS : 1, HJ_GEN_SEED_S(seed));
        args[t].distinct = distinct;
        args[t].payload = (dup > 1) ? 1 : payload;
        args[t].R = R;
        args[t].S = S;
        args[t].nR = nR;
        args[t].nS = nS;
        args[t].tid = t;
        args[t].nthreads = threads;
    }
    int started = 0;
    for (int t = 1; t < threads; t++)
        if (pthread_create(&th[t], NULL, fast_worker, &args[t]) == 0) started = t;
        else break;
    fast_worker(&args[0]);
    for (int t = 1; t <= started; t++) pthread_join(th[t], NULL);
    /* Any worker that failed to start is run here. */
    for (int t = started + 1; t < threads; t++) fast_worker(&args[t]);
    free(args);
    free(th);
    return HJ_OK;
}

void hj_pkfk_closed_form(size_t nR, size_t nS, uint64_t *matched, uint64_t *checksum) {
    /* Every S tuple matches exactly one R tuple with row_id == key on both sides, so
     * checksum = sum over S of 2*key = m * 2 * n(n+1)/2 (wrapping). */
    uint64_t n = nR, m = nR ? nS / nR : 0;
    uint64_t a = n, b = n + 1;
    if (a % 2 == 0) a /= 2; else b /= 2;
    if (matched) *matched = nS;
    if (checksum) *checksum = 2ULL * m * (a * b);
}
