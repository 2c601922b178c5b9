/*
 * hj_main.c - command-line driver with the interface of the reference's bin/main (src/main.c) and
 * bin/gen (src/gen.c), running the joins on the GPU.
 *
 *   hj_main --algo=<name> --workload=<w> --subtype=<s> --param=<p> [--trials=N]
 *       Reads <cfg prefix>/data/<w>/<p>_<s>.cfg (src/main.c:244-255; the prefix comes from
 *       HJ_DATA_CFG_PATH_PREFIX), runs N trials (default 4, the reference's TRIAL_NUM) and prints the
 *       reference's per-trial and averaged lines (src/main.c:429-459), the first trial excluded from the
 *       average. Relation files are read from HJ_DATA_PATH_PREFIX.
 *   hj_main --algo=<name> --r=<file> --s=<file> --nr=N --ns=M [--trials=N]
 *       Same, with the relation files given directly.
 *   hj_main --gen=<pkfk|payload|dup|zipf|fast> --nr=N --ns=M --out-r=<file> --out-s=<file>
 *           [--seed=12345] [--factor=F] [--dup=D]
 *       Writes .bin relations (src/gen.c:133-158; seed 12345 as the reference).
 *
 * Knobs the reference compiles in are environment variables here: HJ_NUM_RADIX_BITS (14),
 * HJ_NUM_PASSES (2), HJ_DEVICE (0).
 */
#define _GNU_SOURCE
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/hjscm_ref.h"

static const char *arg_value(int argc, char **argv, const char *name) {
    size_t L = strlen(name);
    for (int i = 1; i < argc; i++) {
        if (strncmp(argv[i], "--", 2) == 0 && strncmp(argv[i] + 2, name, L) == 0 && argv[i][2 + L] == '=')
            return argv[i] + 3 + L;
    }
    return NULL;
}

/* Minimal reader of the reference's libconfig workload files (the files under config/data): lines of
 * `name = value;` with quoted strings; only the keys data_cfg reads (src/inc/utils.c:258-273). */
static int read_cfg(const char *path, datameta_t *d, char *rbuf, size_t rlen, char *sbuf, size_t slen, char *wbuf,
                    size_t wlen) {
    FILE *f = fopen(path, "r");
    if (!f) return HJ_E_IO;
    memset(d, 0, sizeof(*d));
    char line[1024];
    while (fgets(line, sizeof(line), f)) {
        char key[128], val[896];
        char *eq = strchr(line, '=');
        if (!eq) continue;
        *eq = 0;
        if (sscanf(line, " %127s", key) != 1) continue;
        char *v = eq + 1;
        while (*v == ' ' || *v == '\t') v++;
        size_t n = strcspn(v, ";\n");
        v[n] = 0;
        if (*v == '"') {
            v++;
            char *q = strchr(v, '"');
            if (q) *q = 0;
        }
        snprintf(val, sizeof(val), "%s", v);
        if (!strcmp(key, "r_path_suffix")) snprintf(rbuf, rlen, "%s", val);
        else if (!strcmp(key, "s_path_suffix")) snprintf(sbuf, slen, "%s", val);
        else if (!strcmp(key, "workload_name")) snprintf(wbuf, wlen, "%s", val);
        else if (!strcmp(key, "r_tuple_num")) d->r_tuple_num = strtoull(val, NULL, 10);
        else if (!strcmp(key, "s_tuple_num")) d->s_tuple_num = strtoull(val, NULL, 10);
        else if (!strcmp(key, "r_tuple_size")) d->r_tuple_size = strtoull(val, NULL, 10);
        else if (!strcmp(key, "s_tuple_size")) d->s_tuple_size = strtoull(val, NULL, 10);
        else if (!strcmp(key, "min_key")) d->min_key = strtoull(val, NULL, 10);
        else if (!strcmp(key, "max_key")) d->max_key = strtoull(val, NULL, 10);
        else if (!strcmp(key, "theta")) d->theta = atof(val);
        else if (!strcmp(key, "selectivity")) d->selectivity = atof(val);
        else if (!strcmp(key, "density")) d->density = atof(val);
        else if (!strcmp(key, "sparsity")) d->sparsity = atof(val);
    }
    fclose(f);
    d->r_path_suffix = rbuf;
    d->s_path_suffix = sbuf;
    d->workload_name = wbuf;
    return HJ_OK;
}

static int run_gen(int argc, char **argv) {
    const char *kind = arg_value(argc, argv, "gen");
    const char *nr_s = arg_value(argc, argv, "nr"), *ns_s = arg_value(argc, argv, "ns");
    const char *out_r = arg_value(argc, argv, "out-r"), *out_s = arg_value(argc, argv, "out-s");
    const char *seed_s = arg_value(argc, argv, "seed"), *factor_s = arg_value(argc, argv, "factor");
    const char *dup_s = arg_value(argc, argv, "dup");
    if (!nr_s || !ns_s || !out_s) {
        fprintf(stderr, "usage: hj_main --gen=<pkfk|payload|dup|zipf|fast> --nr=N --ns=M --out-r=F --out-s=F\n");
        return 2;
    }
    size_t nR = strtoull(nr_s, NULL, 10), nS = strtoull(ns_s, NULL, 10);
    unsigned seed = seed_s ? (unsigned)strtoul(seed_s, NULL, 10) : 12345u;
    hj_tuple_t *R = (hj_tuple_t *)malloc((nR ? nR : 1) * 16), *S = (hj_tuple_t *)malloc((nS ? nS : 1) * 16);
    if (!R || !S) return 3;
    int rc;
    if (!strcmp(kind, "pkfk")) rc = hj_gen_pkfk_uniform(nR, nS, seed, 0, R, S);
    else if (!strcmp(kind, "payload")) rc = hj_gen_pkfk_uniform(nR, nS, seed, 1, R, S);
    else if (!strcmp(kind, "dup")) rc = hj_gen_dup_uniform(nR, nS, seed, R, S);
    else if (!strcmp(kind, "zipf")) rc = hj_gen_zipf(nS, nR, factor_s ? atof(factor_s) : 1.05, seed, S);
    else if (!strcmp(kind, "fast")) rc = hj_gen_fast_host(nR, nS, seed, 0, dup_s ? (unsigned)atoi(dup_s) : 1u, 0, R, S);
    else rc = HJ_E_INVAL;
    if (!rc && out_r && strcmp(kind, "zipf")) rc = hj_store_bin(out_r, nR, R);
    if (!rc) rc = hj_store_bin(out_s, nS, S);
    free(R);
    free(S);
    if (rc) fprintf(stderr, "[ERROR] gen %s: %s\n", kind, hj_status_str(rc));
    return rc ? 1 : 0;
}

int main(int argc, char **argv) {
    if (arg_value(argc, argv, "gen")) return run_gen(argc, argv);
    const char *algo_name = arg_value(argc, argv, "algo");
    if (!algo_name) {
        fprintf(stderr, "usage: hj_main --algo=<name> --workload=W --subtype=S --param=P | --r=F --s=F --nr=N --ns=M\n");
        return 2;
    }
    const algo_t *algo = hj_ref_find_algo(algo_name);
    if (!algo) {
        printf("[ERROR] Join algorithm named `%s' does not exist!\n", algo_name); /* src/main.c:215 */
        return 1;
    }
    const char *tr = arg_value(argc, argv, "trials");
    int trials = tr ? atoi(tr) : 4;
    if (trials < 1) trials = 1;
    datameta_t d;
    static char rbuf[4096], sbuf[4096], wbuf[256];
    const char *rfile = arg_value(argc, argv, "r");
    if (rfile) {
        const char *sfile = arg_value(argc, argv, "s"), *nr = arg_value(argc, argv, "nr"), *ns = arg_value(argc, argv, "ns");
        if (!sfile || !nr || !ns) {
            fprintf(stderr, "--r needs --s, --nr and --ns\n");
            return 2;
        }
        memset(&d, 0, sizeof(d));
        snprintf(rbuf, sizeof(rbuf), "%s", rfile);
        snprintf(sbuf, sizeof(sbuf), "%s", sfile);
        snprintf(wbuf, sizeof(wbuf), "files");
        d.r_path_suffix = rbuf;
        d.s_path_suffix = sbuf;
        d.workload_name = wbuf;
        d.r_tuple_num = strtoull(nr, NULL, 10);
        d.s_tuple_num = strtoull(ns, NULL, 10);
        d.r_tuple_size = d.s_tuple_size = 16;
        hj_ref_configure("/", -1, -1, -1);
        if (rfile[0] != '/') hj_ref_configure(".", -1, -1, -1);
    } else {
        const char *wl = arg_value(argc, argv, "workload"), *st = arg_value(argc, argv, "subtype"),
                   *pa = arg_value(argc, argv, "param");
        if (!wl || !st || !pa) {
            fprintf(stderr, "missing --workload/--subtype/--param\n");
            return 2;
        }
        const char *cfgp = getenv("HJ_DATA_CFG_PATH_PREFIX");
        char cfg[8192];
        snprintf(cfg, sizeof(cfg), "%s/data/%s/%s_%s.cfg", cfgp ? cfgp : "config", wl, pa, st);
        if (read_cfg(cfg, &d, rbuf, sizeof(rbuf), sbuf, sizeof(sbuf), wbuf, sizeof(wbuf))) {
            fprintf(stderr, "[ERROR] cannot read %s\n", cfg);
            return 1;
        }
    }
    timekeeper_t global = {0.0, 0.0, 0.0};
    int failed = 0;
    for (int t = 0; t < trials; t++) {
        timekeeper_t tk = {0.0, 0.0, 0.0};
        algo->joinalgo(d, &tk);
        if (tk.total < 0) failed = 1;
        if (t != 0) {
            global.total += tk.total;
            global.buildpart += tk.buildpart;
            global.probejoin += tk.probejoin;
        }
        printf("memory_type: %s\talgo: %s\tworkload: %s\tbuildpart_time: %.9f\tprobejoin_time: %.9f\ttotal_time: %.9f\n",
               "HBM", algo->name, d.workload_name, tk.buildpart, tk.probejoin, tk.total);
    }
    if (trials != 1)
        printf("\nnum_trials: %d\tmemory_type: %s\talgo: %s\tworkload: %s\tbuildpart_time: %.9f\tprobejoin_time: %.9f\ttotal_time: %.9f\n\n",
               trials - 1, "HBM", algo->name, d.workload_name, global.buildpart / (trials - 1),
               global.probejoin / (trials - 1), global.total / (trials - 1));
    return failed;
}
