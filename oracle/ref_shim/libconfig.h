/*
 * Stand-in for libconfig's header, used only to compile the reference sources into the CPU baseline
 * under oracle/_ref. The baseline driver fills datameta_t and the core map itself, so the reference's
 * data_cfg/mc_cfg readers (src/inc/utils.c:236-324) are never called; these stubs only let them link.
 */
#ifndef HJREF_LIBCONFIG_SHIM_H
#define HJREF_LIBCONFIG_SHIM_H
typedef struct { int unused; } config_t;
typedef struct { int unused; } config_setting_t;
static inline void config_init(config_t *c) { (void)c; }
static inline void config_destroy(config_t *c) { (void)c; }
static inline int config_read_file(config_t *c, const char *p) { (void)c; (void)p; return 0; }
static inline const char *config_error_file(const config_t *c) { (void)c; return "none"; }
static inline int config_error_line(const config_t *c) { (void)c; return 0; }
static inline const char *config_error_text(const config_t *c) { (void)c; return "libconfig not available"; }
static inline int config_lookup_string(const config_t *c, const char *p, const char **v) { (void)c; (void)p; (void)v; return 0; }
static inline int config_lookup_float(const config_t *c, const char *p, double *v) { (void)c; (void)p; (void)v; return 0; }
static inline int config_lookup_int(const config_t *c, const char *p, int *v) { (void)c; (void)p; (void)v; return 0; }
static inline int config_lookup_int64(const config_t *c, const char *p, long long *v) { (void)c; (void)p; (void)v; return 0; }
static inline config_setting_t *config_lookup(const config_t *c, const char *p) { (void)c; (void)p; return 0; }
static inline int config_setting_length(const config_setting_t *s) { (void)s; return 0; }
static inline int config_setting_get_int_elem(const config_setting_t *s, int i) { (void)s; (void)i; return 0; }
#endif
