/*
 * hjscm_ref.h - the reference-facing plugin interface.
 *
 * The reference's driver (src/main.c) dispatches a join through a static table
 *     typedef struct algo_t { char name[128]; void (*joinalgo)(const datameta_t, timekeeper_t* const); } algo_t;
 * (src/main.c:66-69). This header declares the same structs, byte-compatible with src/inc/store.h,
 * and GPU-backed functions with the exact names and signatures of the reference's join entry points,
 * so that a copy of the reference's main.c links against libhjscm instead of the src/algo sources.
 *
 * Like the reference, each function loads DATA_PATH_PREFIX/<r_path_suffix> and <s_path_suffix>
 * (raw tuple arrays without header, src/algo/phj.c:1884-1890), runs the join and prints
 * "matched_cnt: %zu\tcheck_sum: %zu" (src/algo/phj.c:2206). Loading is not timed. Unlike the
 * reference, a failure prints the error and sets timekeeper->total = -1 instead of exiting.
 * The data prefix and the radix knobs, which the reference compiles in (CMakeLists.txt:32,
 * src/algo/params.h:26-35), are read at run time: hj_ref_configure(), or the environment variables
 * HJ_DATA_PATH_PREFIX, HJ_NUM_RADIX_BITS, HJ_NUM_PASSES, HJ_DEVICE.
 */
#ifndef HJSCM_REF_H
#define HJSCM_REF_H

#include <stddef.h>
#include <stdint.h>

#include "hjscm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* src/inc/store.h:74-78 */
typedef struct {
    double buildpart;
    double probejoin;
    double total;
} timekeeper_t;

/* src/inc/store.h:126-144 (key_t_ is size_t) */
typedef struct {
    char *r_path_suffix;
    char *s_path_suffix;

    double theta;
    double selectivity;
    double density;
    double sparsity;

    size_t r_tuple_num;
    size_t s_tuple_num;
    size_t r_tuple_size;
    size_t s_tuple_size;

    size_t min_key;
    size_t max_key;

    char *workload_name;
} datameta_t;

/* src/main.c:66-69 */
typedef struct algo_t {
    char name[128];
    void (*joinalgo)(const datameta_t, timekeeper_t *const);
} algo_t;

/* Entry points under the reference's names (src/main.c:73-82, 109-116, 126-138). */
void nphj_sc(const datameta_t datameta, timekeeper_t *const timekeeper);
void nphj_lp(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_bc(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_lp(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_bw_reg_bc(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_bw_reg_lp(const datameta_t datameta, timekeeper_t *const timekeeper);
/* Same results as phj_radix_bc (every match counted; src/algo/phj.c:2523-2535). */
void phj_radix_sc(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_hr(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_hro(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_bw_reg_sc(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_bw_reg_hr(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_radix_bw_reg_hro(const datameta_t datameta, timekeeper_t *const timekeeper);
/* Two passes with NUM_RADIX_BITS_PASS1 bits in pass 1 (src/algo/phj_asymm_radix.c,
 * phj_asymm_radix.h:10-19; 11 unless hj_ref_configure_asymm or HJ_NUM_RADIX_BITS_PASS1 says otherwise,
 * clamped so that each pass has at most 8 bits). */
void phj_asymm_radix_bc(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_asymm_radix_sc(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_asymm_radix_hr(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_asymm_radix_hro(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_asymm_radix_bw_reg_bc(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_asymm_radix_bw_reg_sc(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_asymm_radix_bw_reg_hr(const datameta_t datameta, timekeeper_t *const timekeeper);
void phj_asymm_radix_bw_reg_hro(const datameta_t datameta, timekeeper_t *const timekeeper);
/* Materialising joins (src/main.c:87-92, 119-122): pairs, then the retrieve checksum (hj_join_mat);
 * the timekeeper's total includes the retrieve phase. */
void ptr_nphj_sc(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_nphj_lp(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_phj_radix_bc(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_phj_radix_sc(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_phj_radix_lp(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_phj_radix_hr(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_phj_radix_bw_reg_bc(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_phj_radix_bw_reg_sc(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_phj_radix_bw_reg_lp(const datameta_t datameta, timekeeper_t *const timekeeper);
void ptr_phj_radix_bw_reg_hr(const datameta_t datameta, timekeeper_t *const timekeeper);

/* The dispatch table (src/main.c:72-143 restricted to the names above) and its length. */
extern const algo_t hj_ref_algos[];
extern const int hj_ref_algo_count;
/* Exact-name lookup over hj_ref_algos (src/main.c:202-220); NULL if absent. */
const algo_t *hj_ref_find_algo(const char *name);

/* Run-time replacements for the reference's compile-time knobs. prefix may be NULL (keep),
 * num_radix_bits / num_passes / device < 0 keep the current value. */
void hj_ref_configure(const char *data_path_prefix, int num_radix_bits, int num_passes, int device);
/* NUM_RADIX_BITS_PASS1 of the phj_asymm_radix_* entry points (< 0: back to the environment / 11). */
void hj_ref_configure_asymm(int num_radix_bits_pass1);

/* Result of the last call of one of the functions above on this thread (the reference only prints
 * it). */
int hj_ref_last_result(hj_result_t *out);

/* Load a raw tuple file (the reference's .bin format: n * 16 bytes, no header) into buf. */
int hj_load_bin(const char *path, size_t n, hj_tuple_t *buf);
/* Write n tuples to a raw .bin file (the format bin/gen writes, src/gen.c:187-192). */
int hj_store_bin(const char *path, size_t n, const hj_tuple_t *buf);

#ifdef __cplusplus
}
#endif

#endif /* HJSCM_REF_H */
