/*
 * hj_feistel.h - seeded bijection on [0, n) shared by the host (C) and device (CUDA) generators.
 *
 * The reference draws a random permutation of 1..n with a sequential Knuth shuffle over glibc rand()
 * (src/gen.c:161-171), which is O(n) dependent random swaps and cannot run in parallel. The parallel
 * generators use a keyed bijection instead: a 6-round unbalanced Feistel network on the smallest
 * power of two >= n, with cycle walking to stay inside [0, n). Every index maps independently, so
 * host threads and GPU threads produce identical output.
 */
#ifndef HJ_FEISTEL_H
#define HJ_FEISTEL_H

#include <stdint.h>

#ifdef __CUDACC__
#define HJ_HD __host__ __device__ __forceinline__
#else
#define HJ_HD static inline
#endif

/* splitmix64 output function (Steele, Lea, Flood 2014). */
HJ_HD uint64_t hj_mix64(uint64_t z) {
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return z;
}

typedef struct {
    uint64_t n;        /* domain size */
    uint32_t lo_bits;  /* width of the right half */
    uint32_t hi_bits;  /* width of the left half */
    uint64_t keys[6];  /* round keys */
} hj_feistel_t;

HJ_HD void hj_feistel_init(hj_feistel_t *f, uint64_t n, uint64_t seed) {
    uint32_t k = 2;
    while (k < 64 && ((uint64_t)1 << k) < n) k++;
    f->n = n;
    f->lo_bits = k / 2;
    f->hi_bits = k - k / 2;
    uint64_t s = seed;
    for (int r = 0; r < 6; r++) {
        s += 0x9e3779b97f4a7c15ULL;
        f->keys[r] = hj_mix64(s);
    }
}

/* One pass of the network over the full power-of-two domain. Even rounds update the left half from
 * the right, odd rounds the right from the left; each round is invertible, so the pass is a bijection
 * of [0, 2^(lo+hi)). */
HJ_HD uint64_t hj_feistel_round_trip(const hj_feistel_t *f, uint64_t x) {
    const uint64_t lo_mask = ((uint64_t)1 << f->lo_bits) - 1;
    const uint64_t hi_mask = ((uint64_t)1 << f->hi_bits) - 1;
    uint64_t lo = x & lo_mask;
    uint64_t hi = (x >> f->lo_bits) & hi_mask;
    for (int r = 0; r < 6; r++) {
        if ((r & 1) == 0)
            hi ^= hj_mix64(lo ^ f->keys[r]) & hi_mask;
        else
            lo ^= hj_mix64(hi ^ f->keys[r]) & lo_mask;
    }
    return (hi << f->lo_bits) | lo;
}

/* Bijection of [0, n): cycle walking terminates because the starting point lies on its own cycle. */
HJ_HD uint64_t hj_feistel_perm(const hj_feistel_t *f, uint64_t i) {
    if (f->n <= 1) return 0;
    uint64_t y = i;
    do {
        y = hj_feistel_round_trip(f, y);
    } while (y >= f->n);
    return y;
}

/* Seeds of the two bijections of one generated relation pair. */
#define HJ_GEN_SEED_R(seed) ((seed) ^ 0x5245u)
#define HJ_GEN_SEED_S(seed) ((seed) ^ 0x53u ^ 0x7f4a7c159e3779b9ULL)

/* Tuple i of R / tuple j of S for the fast generators (see hjscm.h, hj_gen_fast_host). */
HJ_HD void hj_fast_r_tuple(const hj_feistel_t *fr, uint64_t distinct, int payload, uint64_t i,
                           uint64_t *key, uint64_t *row_id) {
    uint64_t p = hj_feistel_perm(fr, i);
    uint64_t k = (distinct == fr->n ? p : p % distinct) + 1;
    *key = k;
    *row_id = payload ? i + 1 : k;
}

HJ_HD void hj_fast_s_tuple(const hj_feistel_t *fs, uint64_t distinct, int payload, uint64_t j,
                           uint64_t *key, uint64_t *row_id) {
    uint64_t p = hj_feistel_perm(fs, j);
    uint64_t k = p % distinct + 1;
    *key = k;
    *row_id = payload ? j + 1 : k;
}

#endif /* HJ_FEISTEL_H */
