/*
 * ref_driver.c - command-line driver around the reference's own join and generator functions, built
 * from the reference sources by oracle/Makefile into oracle/_ref. TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.
 *
 * It replaces src/main.c's libconfig-driven setup (src/main.c:147-255) with flags and calls the
 * reference functions unmodified:
 *   hjref_pN --algo=NAME --prefix=DIR --r=REL --s=REL --nr=N --ns=M [--bits=14] [--bits1=11]
 *            [--threads=T] [--trials=K]
 *       NAME: nphj_sc, nphj_lp, phj_radix_{bc,lp,sc,hr,hro}, ptr_nphj_{sc,lp}, ptr_phj_radix_{bc,lp,sc,hr}
 *       (materialising joins: pairs, then the retrieve checksum), and with N = 2
 *       phj_asymm_radix_{bc,sc,hr,hro}
 *       (pass-1 bits --bits1, NUM_RADIX_BITS_PASS1, default 11 and at most --bits as
 *       src/algo/phj_asymm_radix.h:10-17 rules).
 *       Each trial prints the reference's "matched_cnt: ..\tcheck_sum: .." line, then
 *       "hjref_trial: <k> buildpart: <s> probejoin: <s> total: <s>".
 *   hjref_pN --gen=<pkfk|payload|dup|zipf> --prefix=DIR --nr=N --ns=M [--factor=F] [--seed=12345]
 *       srand(seed), then gen_pkfk_uniform / payload_gen_pkfk_uniform / gen_dup_uniform /
 *       gen_fk_zipfian_eth exactly as generate_workload does (src/gen.c:29-117); files land under DIR.
 * N (1 or 2) is the reference's compile-time NUM_PASSES.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "inc/store.h"

int hjref_threads = 1;
int hjref_radix_bits = 14;
int hjref_radix_bits_pass1 = 11;
const char *hjref_data_prefix = ".";
const char *hjref_work_prefix = "/tmp";

extern int local_cores[];
extern int remote_cores[];

void nphj_sc(const datameta_t, timekeeper_t *const);
void nphj_lp(const datameta_t, timekeeper_t *const);
void phj_radix_bc(const datameta_t, timekeeper_t *const);
void phj_radix_lp(const datameta_t, timekeeper_t *const);
void phj_radix_sc(const datameta_t, timekeeper_t *const);
void phj_radix_hr(const datameta_t, timekeeper_t *const);
void phj_radix_hro(const datameta_t, timekeeper_t *const);
void ptr_nphj_sc(const datameta_t, timekeeper_t *const);
void ptr_nphj_lp(const datameta_t, timekeeper_t *const);
void ptr_phj_radix_bc(const datameta_t, timekeeper_t *const);
void ptr_phj_radix_lp(const datameta_t, timekeeper_t *const);
void ptr_phj_radix_sc(const datameta_t, timekeeper_t *const);
void ptr_phj_radix_hr(const datameta_t, timekeeper_t *const);
#if NUM_PASSES == 2
void phj_asymm_radix_bc(const datameta_t, timekeeper_t *const);
void phj_asymm_radix_sc(const datameta_t, timekeeper_t *const);
void phj_asymm_radix_hr(const datameta_t, timekeeper_t *const);
void phj_asymm_radix_hro(const datameta_t, timekeeper_t *const);
#endif
void gen_pkfk_uniform(const size_t, const size_t, const char *, const char *, const char *);
void payload_gen_pkfk_uniform(const size_t, const size_t, const char *, const char *, const char *);
void gen_dup_uniform(const size_t, const size_t, const char *, const char *, const char *);
void gen_fk_zipfian_eth(const size_t, const size_t, double);

static const char *arg(int argc, char **argv, const char *name) {
    size_t L = strlen(name);
    for (int i = 1; i < argc; i++)
        if (!strncmp(argv[i], "--", 2) && !strncmp(argv[i] + 2, name, L) && argv[i][2 + L] == '=')
            return argv[i] + 3 + L;
    return NULL;
}

int main(int argc, char **argv) {
    const char *v;
    long nproc = sysconf(_SC_NPROCESSORS_ONLN);
    if (nproc < 1) nproc = 1;
    for (int i = 0; i < 1024; i++) local_cores[i] = remote_cores[i] = (int)(i % nproc);
    hjref_threads = (v = arg(argc, argv, "threads")) ? atoi(v) : (int)nproc;
    if (hjref_threads < 1) hjref_threads = 1;
    hjref_radix_bits = (v = arg(argc, argv, "bits")) ? atoi(v) : 14;
    hjref_radix_bits_pass1 = (v = arg(argc, argv, "bits1")) ? atoi(v) : 11;
    if (hjref_radix_bits_pass1 > hjref_radix_bits) hjref_radix_bits_pass1 = hjref_radix_bits;
    hjref_data_prefix = (v = arg(argc, argv, "prefix")) ? v : ".";
    const size_t nR = (v = arg(argc, argv, "nr")) ? strtoull(v, NULL, 10) : 0;
    const size_t nS = (v = arg(argc, argv, "ns")) ? strtoull(v, NULL, 10) : 0;
    const unsigned seed = (v = arg(argc, argv, "seed")) ? (unsigned)strtoul(v, NULL, 10) : 12345u;

    if ((v = arg(argc, argv, "gen"))) {
        srand(seed);
        if (!strcmp(v, "pkfk")) gen_pkfk_uniform(nR, nS, "gen", "R", "S");
        else if (!strcmp(v, "payload")) payload_gen_pkfk_uniform(nR, nS, "gen", "R", "S");
        else if (!strcmp(v, "dup")) gen_dup_uniform(nR, nS, "gen", "R", "S");
        else if (!strcmp(v, "zipf")) {
            const char *f = arg(argc, argv, "factor");
            /* gen_fk_zipfian_eth adds 1 to its theta argument (src/gen.c:379-380). */
            gen_fk_zipfian_eth(nS, nR, (f ? atof(f) : 1.05) - 1.0);
        } else {
            fprintf(stderr, "unknown --gen=%s\n", v);
            return 2;
        }
        return 0;
    }

    const char *algo = arg(argc, argv, "algo");
    void (*fn)(const datameta_t, timekeeper_t *const) = NULL;
    if (algo && !strcmp(algo, "nphj_sc")) fn = nphj_sc;
    else if (algo && !strcmp(algo, "nphj_lp")) fn = nphj_lp;
    else if (algo && !strcmp(algo, "phj_radix_bc")) fn = phj_radix_bc;
    else if (algo && !strcmp(algo, "phj_radix_lp")) fn = phj_radix_lp;
    else if (algo && !strcmp(algo, "phj_radix_sc")) fn = phj_radix_sc;
    else if (algo && !strcmp(algo, "phj_radix_hr")) fn = phj_radix_hr;
    else if (algo && !strcmp(algo, "phj_radix_hro")) fn = phj_radix_hro;
    else if (algo && !strcmp(algo, "ptr_nphj_sc")) fn = ptr_nphj_sc;
    else if (algo && !strcmp(algo, "ptr_nphj_lp")) fn = ptr_nphj_lp;
    else if (algo && !strcmp(algo, "ptr_phj_radix_bc")) fn = ptr_phj_radix_bc;
    else if (algo && !strcmp(algo, "ptr_phj_radix_lp")) fn = ptr_phj_radix_lp;
    else if (algo && !strcmp(algo, "ptr_phj_radix_sc")) fn = ptr_phj_radix_sc;
    else if (algo && !strcmp(algo, "ptr_phj_radix_hr")) fn = ptr_phj_radix_hr;
#if NUM_PASSES == 2
    else if (algo && !strcmp(algo, "phj_asymm_radix_bc")) fn = phj_asymm_radix_bc;
    else if (algo && !strcmp(algo, "phj_asymm_radix_sc")) fn = phj_asymm_radix_sc;
    else if (algo && !strcmp(algo, "phj_asymm_radix_hr")) fn = phj_asymm_radix_hr;
    else if (algo && !strcmp(algo, "phj_asymm_radix_hro")) fn = phj_asymm_radix_hro;
#endif
    if (!fn) {
        fprintf(stderr, "unknown or missing --algo\n");
        return 2;
    }
    datameta_t d;
    memset(&d, 0, sizeof(d));
    d.r_path_suffix = (char *)arg(argc, argv, "r");
    d.s_path_suffix = (char *)arg(argc, argv, "s");
    d.r_tuple_num = nR;
    d.s_tuple_num = nS;
    d.r_tuple_size = d.s_tuple_size = 16;
    d.min_key = 1;
    d.max_key = nR;
    d.workload_name = (char *)"hjref";
    if (!d.r_path_suffix || !d.s_path_suffix) {
        fprintf(stderr, "missing --r/--s\n");
        return 2;
    }
    const int trials = (v = arg(argc, argv, "trials")) ? atoi(v) : 1;
    for (int t = 0; t < trials; t++) {
        timekeeper_t tk = {0.0, 0.0, 0.0};
        fn(d, &tk);
        printf("hjref_trial: %d buildpart: %.9f probejoin: %.9f total: %.9f\n", t, tk.buildpart, tk.probejoin,
               tk.total);
        fflush(stdout);
    }
    return 0;
}
