/*
 * Forced-include header (gcc -include) for the CPU-baseline build of the reference sources. The
 * reference takes these knobs as -D definitions from CMake (CMakeLists.txt:18-373); thread counts, the
 * radix bits and the data directory become run-time variables of the baseline driver here, so one
 * build serves any core count and configuration. NUM_PASSES stays a -D (it selects code with #if).
 */
#ifndef HJREF_KNOBS_H
#define HJREF_KNOBS_H
extern int hjref_threads;
extern int hjref_radix_bits;
extern int hjref_radix_bits_pass1;
extern const char *hjref_data_prefix;
extern const char *hjref_work_prefix;
#define THREAD_NUM hjref_threads
#define BUILDPART_THREAD_NUM hjref_threads
#define BUILDPART_WRITE_THREAD_NUM (hjref_threads > 1 ? hjref_threads - 1 : 1)
#define PROBEJOIN_THREAD_NUM hjref_threads
#define INTERMEDIATEMEMSET_THREAD_NUM hjref_threads
#define RETRIEVE_THREAD_NUM hjref_threads
#define XSOCKET_THREAD_NUM_DEFAULT 4
#define CORE_NUM 1024
#define SINGLE_SOCKET_CORE_NUM 1024
#define NUM_RADIX_BITS hjref_radix_bits
/* phj_asymm_radix.h compares this with NUM_RADIX_BITS in an #if; as identifiers both read 0 there, so
 * the header keeps this definition, and the driver applies the header's clamp (pass 1 <= all bits). */
#define NUM_RADIX_BITS_PASS1 hjref_radix_bits_pass1
#define DATA_PATH_PREFIX hjref_data_prefix
#define WORK_PATH_PREFIX hjref_work_prefix
#define DUMP_PATH_PREFIX hjref_work_prefix
#define DATA_CFG_PATH_PREFIX "."
#define CPU_CFG_PATH "cpu.cfg"
#define CHAR_BUFFER_LEN 4096
#define TRIAL_NUM 1
#define BUCKET_CAPACITY 2
#define PREFETCH_DISTANCE 32
#define OVERFLOW_BUF_SIZE 1024
#define INTERMEDIATE_SCALING_FACTOR 2
#define PHJ_SC_BUCKET_CAPACITY 2
#define USE_SWWCB_OPTIMIZED_PART
#define USE_SWWCB_OPTIMIZED_RADIX_CLUSTER
#define WARMUP
#endif
