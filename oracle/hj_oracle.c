/*
 * hj_oracle.c - CPU oracle for the equi-join hot path. TEST INFRASTRUCTURE ONLY: it is linked by the
 * test-suite, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the checker, and never
 * by the product library.
 *
 * Two restatements of the reference's results on 16-byte {key, row_id} tuples:
 *
 * 1. hjo_phj_literal: the reference's radix join step by step, single-threaded.
 *    - pass 1: histogram of IDHASH(key, F1-1, 0) and a stable scatter (src/algo/phj.c:147-215);
 *    - pass 2 (two passes): per pass-1 partition, a stable re-cluster on IDHASH(key, (F2-1) << b1, b1)
 *      (src/algo/phj.c:366-389, 448-491), b1 = bits / passes (src/algo/params.h:34-35);
 *    - a join task per partition with |R_p| > 0 and |S_p| > 0 (src/algo/phj.c:459-491);
 *    - bc_join (src/algo/phj.c:496-571): bucket[next_pow_2(|R_p|)], next[|R_p|], 1-based positions,
 *      insertion by prepending, probe walks the whole chain and adds every equal key;
 *    - lp_join (src/algo/phj.c:574-680): a table of next_pow_2(|R_p|) tuples, key 0 = empty, insert at
 *      the first empty slot from the hash, probe until an empty slot or the first equal key.
 *      The table-full case (an absent key with |R_p| a power of two) loops forever in the reference;
 *      here the walk is bounded by the table size and reports HJO_E_FULL.
 *    next_pow_2 is the reference's floating-point formula (src/inc/utils.c:351-353).
 *
 * 2. hjo_join: the same results computed directly from their definition in O(|R| + |S|):
 *    - HJO_ALL   (bc_join, nphj_sc): every pair with equal keys, checksum += r.row_id + s.row_id
 *      (src/algo/phj.c:555-557, src/algo/nphj.c:348-350);
 *    - HJO_FIRST (phj_radix_lp): per S tuple, the first R tuple in input order with an equal key;
 *      R tuples with key 0 never match because key 0 marks an empty slot (src/algo/phj.c:614, 655);
 *    - HJO_FIRST_NP (nphj_lp): the same without the key-0 rule, since nphj_lp stores hashkey + 1
 *      (src/algo/nphj.c:1064); the reference's winner among equal R keys is a thread race there, so
 *      the single-thread outcome (first in input order) is the contract.
 *    Sums wrap modulo 2^64 as the reference's size_t accumulators do.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    uint64_t key;
    uint64_t row_id;
} hjo_tuple_t;

enum { HJO_ALL = 0, HJO_FIRST = 1, HJO_FIRST_NP = 2 };
enum { HJO_OK = 0, HJO_E_INVAL = 1, HJO_E_OOM = 2, HJO_E_FULL = 4 };

/* src/inc/utils.c:351-353 */
static size_t ref_next_pow_2(size_t x) { return (size_t)pow(2, ceil(log((double)x) / log(2))); }

/* ---------------------------------------------------------------------------------------------- */
/* 1. literal restatement                                                                          */
/* ---------------------------------------------------------------------------------------------- */

/* Stable partition of in[0..n) on (key & mask) >> shift into out[0..n); hist[f+1] = partition starts. */
static void stable_cluster(const hjo_tuple_t *in, size_t n, hjo_tuple_t *out, uint64_t mask, int shift,
                           size_t fanout, size_t *start) {
    memset(start, 0, (fanout + 1) * sizeof(size_t));
    for (size_t i = 0; i < n; i++) start[((in[i].key & mask) >> shift) + 1]++;
    for (size_t f = 0; f < fanout; f++) start[f + 1] += start[f];
    size_t *cur = (size_t *)malloc(fanout * sizeof(size_t));
    memcpy(cur, start, fanout * sizeof(size_t));
    for (size_t i = 0; i < n; i++) out[cur[(in[i].key & mask) >> shift]++] = in[i];
    free(cur);
}

static void bc_join_lit(const hjo_tuple_t *r, size_t nr, const hjo_tuple_t *s, size_t ns, int bits,
                        uint64_t *cnt, uint64_t *sum) {
    const size_t max_hashkey = ref_next_pow_2(nr);
    const uint64_t hashmask = (uint64_t)(max_hashkey - 1) << bits;
    uint64_t *bucket = (uint64_t *)calloc(max_hashkey, sizeof(uint64_t));
    uint64_t *next = (uint64_t *)calloc(nr, sizeof(uint64_t));
    for (size_t idx = 0; idx < nr;) {
        const uint64_t h = (r[idx].key & hashmask) >> bits;
        next[idx] = bucket[h];
        bucket[h] = ++idx;
    }
    for (size_t j = 0; j < ns; j++) {
        const uint64_t h = (s[j].key & hashmask) >> bits;
        for (uint64_t hit = bucket[h]; hit > 0; hit = next[hit - 1]) {
            if (s[j].key == r[hit - 1].key) {
                (*cnt)++;
                *sum += r[hit - 1].row_id + s[j].row_id;
            }
        }
    }
    free(bucket);
    free(next);
}

static int lp_join_lit(const hjo_tuple_t *r, size_t nr, const hjo_tuple_t *s, size_t ns, int bits,
                       uint64_t *cnt, uint64_t *sum) {
    const size_t max_hashkey = ref_next_pow_2(nr);
    const uint64_t hashmask = (uint64_t)(max_hashkey - 1) << bits;
    const uint64_t hashmask0 = max_hashkey - 1;
    hjo_tuple_t *t = (hjo_tuple_t *)calloc(max_hashkey, sizeof(hjo_tuple_t));
    int rc = HJO_OK;
    for (size_t i = 0; i < nr; i++) {
        uint64_t h = (r[i].key & hashmask) >> bits;
        size_t steps = 0;
        while (t[h].key) {
            h = (h + 1) & hashmask0;
            if (++steps > max_hashkey) break;
        }
        if (steps > max_hashkey) {
            rc = HJO_E_FULL;
            continue;
        }
        t[h] = r[i];
    }
    for (size_t j = 0; j < ns; j++) {
        uint64_t h = (s[j].key & hashmask) >> bits;
        size_t steps = 0;
        while (t[h].key && t[h].key != s[j].key) {
            h = (h + 1) & hashmask0;
            if (++steps >= max_hashkey) break;
        }
        if (steps >= max_hashkey) {
            rc = HJO_E_FULL;
            continue;
        }
        if (t[h].key != 0) {
            (*cnt)++;
            *sum += s[j].row_id + t[h].row_id;
        }
    }
    free(t);
    return rc;
}

int hjo_phj_literal(int bits, int passes, int lp, const hjo_tuple_t *R, size_t nR, const hjo_tuple_t *S,
                    size_t nS, uint64_t *cnt, uint64_t *sum) {
    if (bits < 1 || bits > 24 || (passes != 1 && passes != 2)) return HJO_E_INVAL;
    *cnt = 0;
    *sum = 0;
    const int b1 = bits / passes;
    const size_t F1 = (size_t)1 << b1, F2 = (size_t)1 << (bits - b1);
    hjo_tuple_t *r1 = (hjo_tuple_t *)malloc((nR ? nR : 1) * sizeof(hjo_tuple_t));
    hjo_tuple_t *s1 = (hjo_tuple_t *)malloc((nS ? nS : 1) * sizeof(hjo_tuple_t));
    hjo_tuple_t *r2 = (hjo_tuple_t *)malloc((nR ? nR : 1) * sizeof(hjo_tuple_t));
    hjo_tuple_t *s2 = (hjo_tuple_t *)malloc((nS ? nS : 1) * sizeof(hjo_tuple_t));
    size_t *rs1 = (size_t *)malloc((F1 + 1) * sizeof(size_t)), *ss1 = (size_t *)malloc((F1 + 1) * sizeof(size_t));
    size_t *rs2 = (size_t *)malloc((F2 + 1) * sizeof(size_t)), *ss2 = (size_t *)malloc((F2 + 1) * sizeof(size_t));
    if (!r1 || !s1 || !r2 || !s2 || !rs1 || !ss1 || !rs2 || !ss2) return HJO_E_OOM;
    int rc = HJO_OK;
    stable_cluster(R, nR, r1, F1 - 1, 0, F1, rs1);
    stable_cluster(S, nS, s1, F1 - 1, 0, F1, ss1);
    for (size_t p = 0; p < F1; p++) {
        const size_t nr = rs1[p + 1] - rs1[p], ns = ss1[p + 1] - ss1[p];
        if (!(nr > 0 && ns > 0)) continue;
        if (passes == 1) {
            if (lp) rc |= lp_join_lit(r1 + rs1[p], nr, s1 + ss1[p], ns, bits, cnt, sum);
            else bc_join_lit(r1 + rs1[p], nr, s1 + ss1[p], ns, bits, cnt, sum);
            continue;
        }
        stable_cluster(r1 + rs1[p], nr, r2 + rs1[p], (uint64_t)(F2 - 1) << b1, b1, F2, rs2);
        stable_cluster(s1 + ss1[p], ns, s2 + ss1[p], (uint64_t)(F2 - 1) << b1, b1, F2, ss2);
        for (size_t q = 0; q < F2; q++) {
            const size_t mr = rs2[q + 1] - rs2[q], ms = ss2[q + 1] - ss2[q];
            if (!(mr > 0 && ms > 0)) continue;
            const hjo_tuple_t *rp = r2 + rs1[p] + rs2[q], *sp = s2 + ss1[p] + ss2[q];
            if (lp) rc |= lp_join_lit(rp, mr, sp, ms, bits, cnt, sum);
            else bc_join_lit(rp, mr, sp, ms, bits, cnt, sum);
        }
    }
    free(r1); free(s1); free(r2); free(s2); free(rs1); free(ss1); free(rs2); free(ss2);
    return rc;
}

/* ---------------------------------------------------------------------------------------------- */
/* 2. direct definition                                                                            */
/* ---------------------------------------------------------------------------------------------- */

typedef struct {
    uint64_t key;
    uint64_t count;     /* R tuples with this key */
    uint64_t sum;       /* sum of their row ids (wrapping) */
    uint64_t first_rid; /* row id of the first one in input order */
    int used;
} hjo_slot_t;

static uint64_t mixh(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

int hjo_join(int mode, const hjo_tuple_t *R, size_t nR, const hjo_tuple_t *S, size_t nS, uint64_t *cnt,
             uint64_t *sum) {
    if (!cnt || !sum || mode < HJO_ALL || mode > HJO_FIRST_NP) return HJO_E_INVAL;
    *cnt = 0;
    *sum = 0;
    if (nR == 0 || nS == 0) return HJO_OK;
    size_t cap = 16;
    while (cap < 2 * nR) cap <<= 1;
    hjo_slot_t *t = (hjo_slot_t *)calloc(cap, sizeof(hjo_slot_t));
    if (!t) return HJO_E_OOM;
    for (size_t i = 0; i < nR; i++) {
        if (mode == HJO_FIRST && R[i].key == 0) continue;
        size_t h = mixh(R[i].key) & (cap - 1);
        while (t[h].used && t[h].key != R[i].key) h = (h + 1) & (cap - 1);
        if (!t[h].used) {
            t[h].used = 1;
            t[h].key = R[i].key;
            t[h].first_rid = R[i].row_id;
        }
        t[h].count++;
        t[h].sum += R[i].row_id;
    }
    uint64_t c = 0, s = 0;
    for (size_t j = 0; j < nS; j++) {
        size_t h = mixh(S[j].key) & (cap - 1);
        while (t[h].used && t[h].key != S[j].key) h = (h + 1) & (cap - 1);
        if (!t[h].used) continue;
        if (mode == HJO_ALL) {
            c += t[h].count;
            s += t[h].sum + t[h].count * S[j].row_id;
        } else {
            c += 1;
            s += t[h].first_rid + S[j].row_id;
        }
    }
    free(t);
    *cnt = c;
    *sum = s;
    return HJO_OK;
}

/* Dense-key variant of hjo_join for keys in [1, max_key] (the reference's generators): per-key arrays
 * instead of a hash table, O(max_key) memory. Same results as hjo_join. */
int hjo_join_dense(int mode, const hjo_tuple_t *R, size_t nR, const hjo_tuple_t *S, size_t nS,
                   uint64_t max_key, uint64_t *cnt, uint64_t *sum) {
    if (!cnt || !sum) return HJO_E_INVAL;
    *cnt = 0;
    *sum = 0;
    uint64_t *count = (uint64_t *)calloc(max_key + 1, sizeof(uint64_t));
    uint64_t *rsum = (uint64_t *)calloc(max_key + 1, sizeof(uint64_t));
    uint64_t *first = (uint64_t *)calloc(max_key + 1, sizeof(uint64_t));
    if (!count || !rsum || !first) {
        free(count); free(rsum); free(first);
        return HJO_E_OOM;
    }
    int rc = HJO_OK;
    for (size_t i = 0; i < nR; i++) {
        const uint64_t k = R[i].key;
        if (k > max_key) { rc = HJO_E_INVAL; continue; }
        if (mode == HJO_FIRST && k == 0) continue;
        if (count[k] == 0) first[k] = R[i].row_id;
        count[k]++;
        rsum[k] += R[i].row_id;
    }
    uint64_t c = 0, s = 0;
    for (size_t j = 0; j < nS; j++) {
        const uint64_t k = S[j].key;
        if (k > max_key || count[k] == 0) continue;
        if (mode == HJO_ALL) {
            c += count[k];
            s += rsum[k] + count[k] * S[j].row_id;
        } else {
            c += 1;
            s += first[k] + S[j].row_id;
        }
    }
    free(count); free(rsum); free(first);
    *cnt = c;
    *sum = s;
    return rc;
}
