/*
 * hj_refapi.c - the reference-facing plugin layer (include/hjscm_ref.h).
 *
 * Each function has the name and signature of a reference join entry point and the same observable
 * behaviour: load the two relation files named by datameta (src/algo/phj.c:1884-1890, untimed), run
 * the join, print "matched_cnt: %zu\tcheck_sum: %zu" (src/algo/phj.c:2206) and fill the timekeeper
 * with buildpart / probejoin / total seconds (src/algo/phj.c:2509-2511). The join itself runs on the
 * GPU through hj_join.
 */
#define _GNU_SOURCE
#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/hjscm_ref.h"

static pthread_mutex_t g_cfg_mu = PTHREAD_MUTEX_INITIALIZER;
static char g_prefix[4096] = "";
static int g_bits = -1, g_passes = -1, g_device = -1, g_bits_pass1 = -1;
static __thread hj_result_t t_last;
static __thread int t_have_last;

void hj_ref_configure(const char *prefix, int num_radix_bits, int num_passes, int device) {
    pthread_mutex_lock(&g_cfg_mu);
    if (prefix) snprintf(g_prefix, sizeof(g_prefix), "%s", prefix);
    if (num_radix_bits >= 0) g_bits = num_radix_bits;
    if (num_passes >= 0) g_passes = num_passes;
    if (device >= 0) g_device = device;
    pthread_mutex_unlock(&g_cfg_mu);
}

static int env_int(const char *name, int dflt) {
    const char *v = getenv(name);
    return (v && *v) ? atoi(v) : dflt;
}

static void current_config(char *prefix, size_t plen, hj_params_t *p) {
    hj_params_init(p);
    pthread_mutex_lock(&g_cfg_mu);
    const char *pre = g_prefix[0] ? g_prefix : getenv("HJ_DATA_PATH_PREFIX");
    snprintf(prefix, plen, "%s", pre ? pre : ".");
    p->num_radix_bits = g_bits >= 0 ? g_bits : env_int("HJ_NUM_RADIX_BITS", 14);
    p->num_passes = g_passes >= 0 ? g_passes : env_int("HJ_NUM_PASSES", 2);
    p->device = g_device >= 0 ? g_device : env_int("HJ_DEVICE", 0);
    pthread_mutex_unlock(&g_cfg_mu);
}

void hj_ref_configure_asymm(int num_radix_bits_pass1) {
    pthread_mutex_lock(&g_cfg_mu);
    g_bits_pass1 = num_radix_bits_pass1;
    pthread_mutex_unlock(&g_cfg_mu);
}

/* Pass-1 bits of the phj_asymm_radix_* entry points: NUM_RADIX_BITS_PASS1, 11 unless configured
 * (src/algo/phj_asymm_radix.h:10-17). */
static int asymm_bits_pass1(void) {
    pthread_mutex_lock(&g_cfg_mu);
    const int b = g_bits_pass1 >= 0 ? g_bits_pass1 : env_int("HJ_NUM_RADIX_BITS_PASS1", 11);
    pthread_mutex_unlock(&g_cfg_mu);
    return b;
}

int hj_load_bin(const char *path, size_t n, hj_tuple_t *buf) {
    if (!path || (n && !buf)) return HJ_E_INVAL;
    FILE *f = fopen(path, "rb");
    if (!f) return HJ_E_IO;
    size_t got = n ? fread(buf, sizeof(hj_tuple_t), n, f) : 0;
    fclose(f);
    return got == n ? HJ_OK : HJ_E_IO;
}

int hj_store_bin(const char *path, size_t n, const hj_tuple_t *buf) {
    if (!path || (n && !buf)) return HJ_E_INVAL;
    FILE *f = fopen(path, "wb");
    if (!f) return HJ_E_IO;
    size_t put = n ? fwrite(buf, sizeof(hj_tuple_t), n, f) : 0;
    int rc = fclose(f);
    return (put == n && rc == 0) ? HJ_OK : HJ_E_IO;
}

int hj_ref_last_result(hj_result_t *out) {
    if (!out || !t_have_last) return HJ_E_INVAL;
    *out = t_last;
    return HJ_OK;
}

/* Shared body of the entry points: the part of join_init_run / nphj_sc outside the thread pools. */
static void run_ref_any(hj_algo_t algo, int bits_pass1, int mat, const datameta_t datameta, timekeeper_t *const tk) {
    char prefix[4096], rpath[8192], spath[8192];
    hj_params_t p;
    current_config(prefix, sizeof(prefix), &p);
    p.radix_bits_pass1 = bits_pass1;
    hj_result_t res;
    memset(&res, 0, sizeof(res));
    tk->buildpart = tk->probejoin = 0.0;
    tk->total = -1.0;
    snprintf(rpath, sizeof(rpath), "%s/%s", prefix, datameta.r_path_suffix ? datameta.r_path_suffix : "");
    snprintf(spath, sizeof(spath), "%s/%s", prefix, datameta.s_path_suffix ? datameta.s_path_suffix : "");
    const size_t nR = datameta.r_tuple_num, nS = datameta.s_tuple_num;
    hj_tuple_t *R = (hj_tuple_t *)malloc((nR ? nR : 1) * sizeof(hj_tuple_t));
    hj_tuple_t *S = (hj_tuple_t *)malloc((nS ? nS : 1) * sizeof(hj_tuple_t));
    int rc = (!R || !S) ? HJ_E_OOM : HJ_OK;
    if (!rc) rc = hj_load_bin(rpath, nR, R);
    if (!rc) rc = hj_load_bin(spath, nS, S);
    if (!rc) rc = mat ? hj_join_mat(algo, &p, R, nR, S, nS, NULL, 0, &res) : hj_join(algo, &p, R, nR, S, nS, &res);
    free(R);
    free(S);
    res.status = rc;
    t_last = res;
    t_have_last = 1;
    if (rc) {
        fprintf(stderr, "[ERROR] %s: %s\n", hj_algo_name(algo), hj_status_str(rc));
        return;
    }
    printf("matched_cnt: %zu\tcheck_sum: %zu\n", (size_t)res.matched_cnt, (size_t)res.checksum);
    tk->buildpart = res.buildpart;
    tk->probejoin = res.probejoin;
    tk->total = res.total;
}

static void run_ref(hj_algo_t algo, const datameta_t d, timekeeper_t *const tk) { run_ref_any(algo, 0, 0, d, tk); }
static void run_asymm(hj_algo_t algo, const datameta_t d, timekeeper_t *const tk) {
    run_ref_any(algo, asymm_bits_pass1(), 0, d, tk);
}
/* ptr_* joins: materialise (r_row_id, s_row_id) pairs, then retrieve the checksum (hj_join_mat). */
static void run_ptr(hj_algo_t algo, const datameta_t d, timekeeper_t *const tk) { run_ref_any(algo, 0, 1, d, tk); }

void nphj_sc(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_NPHJ_SC, d, tk); }
void nphj_lp(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_NPHJ_LP, d, tk); }
void phj_radix_bc(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_BC, d, tk); }
void phj_radix_lp(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_LP, d, tk); }
void phj_radix_bw_reg_bc(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_BC, d, tk); }
void phj_radix_bw_reg_lp(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_LP, d, tk); }
void phj_radix_sc(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_SC, d, tk); }
void phj_radix_hr(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_HR, d, tk); }
void phj_radix_hro(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_HRO, d, tk); }
void phj_radix_bw_reg_sc(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_SC, d, tk); }
void phj_radix_bw_reg_hr(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_HR, d, tk); }
void phj_radix_bw_reg_hro(const datameta_t d, timekeeper_t *const tk) { run_ref(HJ_ALGO_PHJ_RADIX_HRO, d, tk); }
void phj_asymm_radix_bc(const datameta_t d, timekeeper_t *const tk) { run_asymm(HJ_ALGO_PHJ_RADIX_BC, d, tk); }
void phj_asymm_radix_sc(const datameta_t d, timekeeper_t *const tk) { run_asymm(HJ_ALGO_PHJ_RADIX_SC, d, tk); }
void phj_asymm_radix_hr(const datameta_t d, timekeeper_t *const tk) { run_asymm(HJ_ALGO_PHJ_RADIX_HR, d, tk); }
void phj_asymm_radix_hro(const datameta_t d, timekeeper_t *const tk) { run_asymm(HJ_ALGO_PHJ_RADIX_HRO, d, tk); }
void phj_asymm_radix_bw_reg_bc(const datameta_t d, timekeeper_t *const tk) { run_asymm(HJ_ALGO_PHJ_RADIX_BC, d, tk); }
void phj_asymm_radix_bw_reg_sc(const datameta_t d, timekeeper_t *const tk) { run_asymm(HJ_ALGO_PHJ_RADIX_SC, d, tk); }
void phj_asymm_radix_bw_reg_hr(const datameta_t d, timekeeper_t *const tk) { run_asymm(HJ_ALGO_PHJ_RADIX_HR, d, tk); }
void phj_asymm_radix_bw_reg_hro(const datameta_t d, timekeeper_t *const tk) { run_asymm(HJ_ALGO_PHJ_RADIX_HRO, d, tk); }
void ptr_nphj_sc(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_NPHJ_SC, d, tk); }
void ptr_nphj_lp(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_NPHJ_LP, d, tk); }
void ptr_phj_radix_bc(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_PHJ_RADIX_BC, d, tk); }
void ptr_phj_radix_sc(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_PHJ_RADIX_SC, d, tk); }
void ptr_phj_radix_lp(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_PHJ_RADIX_LP, d, tk); }
void ptr_phj_radix_hr(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_PHJ_RADIX_HR, d, tk); }
void ptr_phj_radix_bw_reg_bc(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_PHJ_RADIX_BC, d, tk); }
void ptr_phj_radix_bw_reg_sc(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_PHJ_RADIX_SC, d, tk); }
void ptr_phj_radix_bw_reg_lp(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_PHJ_RADIX_LP, d, tk); }
void ptr_phj_radix_bw_reg_hr(const datameta_t d, timekeeper_t *const tk) { run_ptr(HJ_ALGO_PHJ_RADIX_HR, d, tk); }

const algo_t hj_ref_algos[] = {
    {"nphj_sc", nphj_sc},
    {"nphj_lp", nphj_lp},
    {"phj_radix_bc", phj_radix_bc},
    {"phj_radix_lp", phj_radix_lp},
    {"phj_radix_bw_reg_bc", phj_radix_bw_reg_bc},
    {"phj_radix_bw_reg_lp", phj_radix_bw_reg_lp},
    {"phj_radix_sc", phj_radix_sc},
    {"phj_radix_hr", phj_radix_hr},
    {"phj_radix_hro", phj_radix_hro},
    {"phj_radix_bw_reg_sc", phj_radix_bw_reg_sc},
    {"phj_radix_bw_reg_hr", phj_radix_bw_reg_hr},
    {"phj_radix_bw_reg_hro", phj_radix_bw_reg_hro},
    {"phj_asymm_radix_bc", phj_asymm_radix_bc},
    {"phj_asymm_radix_sc", phj_asymm_radix_sc},
    {"phj_asymm_radix_hr", phj_asymm_radix_hr},
    {"phj_asymm_radix_hro", phj_asymm_radix_hro},
    {"phj_asymm_radix_bw_reg_bc", phj_asymm_radix_bw_reg_bc},
    {"phj_asymm_radix_bw_reg_sc", phj_asymm_radix_bw_reg_sc},
    {"phj_asymm_radix_bw_reg_hr", phj_asymm_radix_bw_reg_hr},
    {"phj_asymm_radix_bw_reg_hro", phj_asymm_radix_bw_reg_hro},
    {"ptr_nphj_sc", ptr_nphj_sc},
    {"ptr_nphj_lp", ptr_nphj_lp},
    {"ptr_phj_radix_bc", ptr_phj_radix_bc},
    {"ptr_phj_radix_sc", ptr_phj_radix_sc},
    {"ptr_phj_radix_lp", ptr_phj_radix_lp},
    {"ptr_phj_radix_hr", ptr_phj_radix_hr},
    {"ptr_phj_radix_bw_reg_bc", ptr_phj_radix_bw_reg_bc},
    {"ptr_phj_radix_bw_reg_sc", ptr_phj_radix_bw_reg_sc},
    {"ptr_phj_radix_bw_reg_lp", ptr_phj_radix_bw_reg_lp},
    {"ptr_phj_radix_bw_reg_hr", ptr_phj_radix_bw_reg_hr},
};
const int hj_ref_algo_count = (int)(sizeof(hj_ref_algos) / sizeof(hj_ref_algos[0]));

const algo_t *hj_ref_find_algo(const char *name) {
    if (!name) return NULL;
    for (int i = 0; i < hj_ref_algo_count; i++)
        if (strcmp(name, hj_ref_algos[i].name) == 0) return &hj_ref_algos[i];
    return NULL;
}
