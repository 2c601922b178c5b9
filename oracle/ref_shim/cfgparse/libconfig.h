/*
 * A small reader of libconfig's file format, standing in for the absent libconfig library when the
 * reference's unchanged driver (src/main.c) is linked against this project's join library
 * (oracle/Makefile, target refmain). It implements the calls the reference's data_cfg / mc_cfg make
 * (src/inc/utils.c:236-324): scalar settings `name = value;` (quoted strings, integers with an optional
 * L suffix, floats), groups `name = { ... };` or `name : { ... };` whose members are looked up by
 * dotted paths, and integer arrays `[a, b, ...]`. Comments: #, // and block comments.
 * Test infrastructure only.
 */
#ifndef HJREF_CFGPARSE_LIBCONFIG_H
#define HJREF_CFGPARSE_LIBCONFIG_H
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define HJCFG_MAX 128
#define HJCFG_PATH 256
#define HJCFG_STR 1024
#define HJCFG_ARR 4096

typedef struct {
    char path[HJCFG_PATH];
    int type; /* 1 string, 2 integer, 3 float, 4 integer array */
    char str[HJCFG_STR];
    long long i;
    double f;
    int n;
    int *arr;
} config_setting_t;

typedef struct {
    config_setting_t s[HJCFG_MAX];
    int n;
    char file[HJCFG_PATH];
    int err_line;
    char err[128];
} config_t;

static inline void config_init(config_t *c) { memset(c, 0, sizeof(*c)); }
static inline void config_destroy(config_t *c) {
    for (int k = 0; k < c->n; k++) free(c->s[k].arr);
    c->n = 0;
}
static inline const char *config_error_file(const config_t *c) { return c->file; }
static inline int config_error_line(const config_t *c) { return c->err_line; }
static inline const char *config_error_text(const config_t *c) { return c->err; }

typedef struct {
    const char *p;
    int line;
} hjcfg_lex;

static inline void hjcfg_skip(hjcfg_lex *L) {
    for (;;) {
        while (*L->p && isspace((unsigned char)*L->p)) {
            if (*L->p == '\n') L->line++;
            L->p++;
        }
        if (*L->p == '#' || (L->p[0] == '/' && L->p[1] == '/')) {
            while (*L->p && *L->p != '\n') L->p++;
        } else if (L->p[0] == '/' && L->p[1] == '*') {
            L->p += 2;
            while (*L->p && !(L->p[0] == '*' && L->p[1] == '/')) {
                if (*L->p == '\n') L->line++;
                L->p++;
            }
            if (*L->p) L->p += 2;
        } else {
            return;
        }
    }
}

static inline int hjcfg_fail(config_t *c, hjcfg_lex *L, const char *what) {
    c->err_line = L->line;
    snprintf(c->err, sizeof(c->err), "%s", what);
    return 0;
}

static inline int hjcfg_number(const char **pp, long long *iv, double *fv, int *is_float) {
    char *end = NULL;
    const char *p = *pp;
    const char *q = p;
    if (*q == '-' || *q == '+') q++;
    int fl = 0;
    while (isdigit((unsigned char)*q) || *q == '.' || *q == 'e' || *q == 'E' ||
           ((*q == '-' || *q == '+') && (q[-1] == 'e' || q[-1] == 'E'))) {
        if (*q == '.' || *q == 'e' || *q == 'E') fl = 1;
        q++;
    }
    if (q == p) return 0;
    if (fl) {
        *fv = strtod(p, &end);
        *iv = (long long)*fv;
    } else {
        *iv = strtoll(p, &end, 0);
        *fv = (double)*iv;
    }
    if (end && (*end == 'L' || *end == 'l')) end++;
    if (end && (*end == 'L' || *end == 'l')) end++;
    *is_float = fl;
    *pp = end ? end : q;
    return 1;
}

static inline int hjcfg_group(config_t *c, hjcfg_lex *L, const char *prefix, int depth);

static inline int hjcfg_setting(config_t *c, hjcfg_lex *L, const char *prefix, int depth) {
    char name[HJCFG_PATH];
    int k = 0;
    while (*L->p && (isalnum((unsigned char)*L->p) || *L->p == '_' || *L->p == '-' || *L->p == '*')) {
        if (k < HJCFG_PATH - 1) name[k++] = *L->p;
        L->p++;
    }
    name[k] = 0;
    if (!k) return hjcfg_fail(c, L, "setting name expected");
    char path[HJCFG_PATH];
    if (prefix[0])
        snprintf(path, sizeof(path), "%s.%s", prefix, name);
    else
        snprintf(path, sizeof(path), "%s", name);
    hjcfg_skip(L);
    if (*L->p != '=' && *L->p != ':') return hjcfg_fail(c, L, "'=' or ':' expected");
    L->p++;
    hjcfg_skip(L);
    if (*L->p == '{') {
        L->p++;
        if (!hjcfg_group(c, L, path, depth + 1)) return 0;
        if (*L->p != '}') return hjcfg_fail(c, L, "'}' expected");
        L->p++;
    } else {
        if (c->n >= HJCFG_MAX) return hjcfg_fail(c, L, "too many settings");
        config_setting_t *s = &c->s[c->n];
        memset(s, 0, sizeof(*s));
        snprintf(s->path, sizeof(s->path), "%s", path);
        if (*L->p == '"') {
            L->p++;
            int m = 0;
            while (*L->p && *L->p != '"') {
                if (m < HJCFG_STR - 1) s->str[m++] = *L->p;
                L->p++;
            }
            if (*L->p != '"') return hjcfg_fail(c, L, "unterminated string");
            L->p++;
            s->type = 1;
        } else if (*L->p == '[') {
            L->p++;
            s->arr = (int *)calloc(HJCFG_ARR, sizeof(int));
            if (!s->arr) return hjcfg_fail(c, L, "out of memory");
            s->type = 4;
            for (;;) {
                hjcfg_skip(L);
                if (*L->p == ']') {
                    L->p++;
                    break;
                }
                long long iv;
                double fv;
                int isf;
                if (!hjcfg_number(&L->p, &iv, &fv, &isf)) return hjcfg_fail(c, L, "array element expected");
                if (s->n < HJCFG_ARR) s->arr[s->n++] = (int)iv;
                hjcfg_skip(L);
                if (*L->p == ',') L->p++;
            }
        } else {
            int isf;
            if (!hjcfg_number(&L->p, &s->i, &s->f, &isf)) return hjcfg_fail(c, L, "value expected");
            s->type = isf ? 3 : 2;
        }
        c->n++;
    }
    hjcfg_skip(L);
    if (*L->p == ';' || *L->p == ',') L->p++;
    return 1;
}

static inline int hjcfg_group(config_t *c, hjcfg_lex *L, const char *prefix, int depth) {
    if (depth > 8) return hjcfg_fail(c, L, "groups nested too deep");
    for (;;) {
        hjcfg_skip(L);
        if (!*L->p || *L->p == '}') return 1;
        if (!hjcfg_setting(c, L, prefix, depth)) return 0;
    }
}

static inline int config_read_file(config_t *c, const char *path) {
    config_destroy(c);
    snprintf(c->file, sizeof(c->file), "%s", path ? path : "");
    FILE *f = path ? fopen(path, "rb") : NULL;
    if (!f) {
        snprintf(c->err, sizeof(c->err), "file I/O error");
        return 0;
    }
    fseek(f, 0, SEEK_END);
    long len = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)(len > 0 ? len : 0) + 1);
    if (!buf) {
        fclose(f);
        return 0;
    }
    size_t got = fread(buf, 1, (size_t)(len > 0 ? len : 0), f);
    fclose(f);
    buf[got] = 0;
    hjcfg_lex L = {buf, 1};
    int ok = hjcfg_group(c, &L, "", 0);
    if (ok && *L.p) ok = hjcfg_fail(c, &L, "unexpected '}'");
    free(buf);
    return ok;
}

static inline config_setting_t *config_lookup(const config_t *c, const char *path) {
    for (int k = 0; k < c->n; k++)
        if (strcmp(c->s[k].path, path) == 0) return (config_setting_t *)&c->s[k];
    return NULL;
}
static inline int config_lookup_string(const config_t *c, const char *path, const char **v) {
    config_setting_t *s = config_lookup(c, path);
    if (!s || s->type != 1) return 0;
    *v = s->str;
    return 1;
}
static inline int config_lookup_int64(const config_t *c, const char *path, long long *v) {
    config_setting_t *s = config_lookup(c, path);
    if (!s || s->type != 2) return 0;
    *v = s->i;
    return 1;
}
static inline int config_lookup_int(const config_t *c, const char *path, int *v) {
    config_setting_t *s = config_lookup(c, path);
    if (!s || s->type != 2) return 0;
    *v = (int)s->i;
    return 1;
}
static inline int config_lookup_float(const config_t *c, const char *path, double *v) {
    config_setting_t *s = config_lookup(c, path);
    if (!s || s->type != 3) return 0;
    *v = s->f;
    return 1;
}
static inline int config_setting_length(const config_setting_t *s) { return s && s->type == 4 ? s->n : 0; }
static inline int config_setting_get_int_elem(const config_setting_t *s, int idx) {
    return s && s->type == 4 && idx >= 0 && idx < s->n ? s->arr[idx] : 0;
}
#endif
