/*
 * Forced-include header for the build of the reference's unchanged driver (src/main.c) against this
 * project's join library (oracle/Makefile, target refmain): the knobs of the CPU-baseline build, with
 * three trials (main.c averages all but the first, src/main.c:429-459) and the workload-file and
 * core-map locations taken at run time ($HJREF_CFG_PREFIX, $HJREF_CPU_CFG).
 */
#ifndef HJREF_MAIN_KNOBS_H
#define HJREF_MAIN_KNOBS_H
#include "hjref_knobs.h"
#undef TRIAL_NUM
#define TRIAL_NUM 3
extern const char *hjref_cfg_prefix;
extern const char *hjref_cpu_cfg;
#undef DATA_CFG_PATH_PREFIX
#define DATA_CFG_PATH_PREFIX hjref_cfg_prefix
#undef CPU_CFG_PATH
#define CPU_CFG_PATH hjref_cpu_cfg
#endif
