/* Runtime of the translated reference -- TEST INFRASTRUCTURE ONLY.
 *
 * Arrays: allocated zero-filled with GUARD elements before and after the
 * Fortran extent, so index 0 and writes just past the last column land in
 * zeroed storage of their own (unchecked Fortran indexing into zeroed memory).
 * Files: the caller registers the text of "3d_input_data" and
 * "stored-solution.dat"; READ statements parse it list-directed (each READ
 * starts a new record and drops what is left of its last record). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "ref_runtime.h"

#define GUARD 256
#define MAXALLOC 4096
#define MAXFILES 8
#define MAXPARAMS 32

static void *g_allocs[MAXALLOC];
static int g_nalloc = 0;

static struct { char name[64]; char *text; } g_files[MAXFILES];
static int g_nfiles = 0;
static const char *g_unit_text[256];
static const char *g_cursor[256];
static int g_cur_unit = -1;

static struct { char name[32]; double v; } g_params[MAXPARAMS];
static int g_nparams = 0;

static void *track(void *p) {
    if (g_nalloc < MAXALLOC) g_allocs[g_nalloc++] = p;
    return p;
}

int *ref_alloc_int(long n) {
    int *p = (int *)calloc((size_t)n + 2 * GUARD, sizeof(int));
    if (!p) { fprintf(stderr, "ref: out of memory\n"); exit(3); }
    return (int *)track(p) + GUARD;
}

double *ref_alloc_dbl(long n) {
    double *p = (double *)calloc((size_t)n + 2 * GUARD, sizeof(double));
    if (!p) { fprintf(stderr, "ref: out of memory\n"); exit(3); }
    return (double *)track(p) + GUARD;
}

void ref_open(int unit, const char *name) {
    for (int i = 0; i < g_nfiles; ++i)
        if (!strcmp(g_files[i].name, name)) {
            g_unit_text[unit & 255] = g_files[i].text;
            g_cursor[unit & 255] = g_files[i].text;
            return;
        }
    fprintf(stderr, "ref: file %s was not registered\n", name);
    exit(4);
}

void ref_read_begin(int unit) { g_cur_unit = unit & 255; }

static const char *next_token(size_t *len) {
    const char *c = g_cursor[g_cur_unit];
    while (*c && (*c == ' ' || *c == '\t' || *c == ',' || *c == '\n' || *c == '\r')) ++c;
    const char *s = c;
    while (*c && !(*c == ' ' || *c == '\t' || *c == ',' || *c == '\n' || *c == '\r')) ++c;
    *len = (size_t)(c - s);
    g_cursor[g_cur_unit] = c;
    return s;
}

void ref_read_int(int *v) {
    size_t n;
    const char *s = next_token(&n);
    char buf[64];
    if (n == 0 || n >= sizeof buf) { fprintf(stderr, "ref: read past end of input\n"); exit(5); }
    memcpy(buf, s, n); buf[n] = 0;
    *v = (int)strtol(buf, NULL, 10);
}

void ref_read_dbl(double *v) {
    size_t n;
    const char *s = next_token(&n);
    char buf[64];
    if (n == 0 || n >= sizeof buf) { fprintf(stderr, "ref: read past end of input\n"); exit(5); }
    memcpy(buf, s, n); buf[n] = 0;
    for (size_t i = 0; i < n; ++i) if (buf[i] == 'd' || buf[i] == 'D') buf[i] = 'e';
    *v = strtod(buf, NULL);
}

void ref_read_end(int unit) {
    const char *c = g_cursor[unit & 255];
    while (*c && *c != '\n') ++c;
    if (*c == '\n') ++c;
    g_cursor[unit & 255] = c;
}

int ref_param_overridden(const char *name) {
    for (int i = 0; i < g_nparams; ++i) if (!strcmp(g_params[i].name, name)) return 1;
    return 0;
}

double ref_param_value(const char *name) {
    for (int i = 0; i < g_nparams; ++i) if (!strcmp(g_params[i].name, name)) return g_params[i].v;
    return 0.0;
}

int ref_strcmp(const char *a, const char *b) { return strcmp(a, b); }

void ref_unknown_call(const char *name) {
    fprintf(stderr, "ref: no argument-less subroutine %s\n", name);
    exit(6);
}

/* ---- API used from Python (ctypes) ---- */

void ref_register_file(const char *name, const char *text) {
    for (int i = 0; i < g_nfiles; ++i)
        if (!strcmp(g_files[i].name, name)) {
            free(g_files[i].text);
            g_files[i].text = strdup(text);
            return;
        }
    if (g_nfiles == MAXFILES) { fprintf(stderr, "ref: too many files\n"); exit(7); }
    snprintf(g_files[g_nfiles].name, sizeof g_files[0].name, "%s", name);
    g_files[g_nfiles].text = strdup(text);
    ++g_nfiles;
}

void ref_set_param(const char *name, double v) {
    for (int i = 0; i < g_nparams; ++i)
        if (!strcmp(g_params[i].name, name)) { g_params[i].v = v; return; }
    if (g_nparams == MAXPARAMS) return;
    snprintf(g_params[g_nparams].name, sizeof g_params[0].name, "%s", name);
    g_params[g_nparams].v = v;
    ++g_nparams;
}

void ref_free_all(void) {
    for (int i = 0; i < g_nalloc; ++i) free(g_allocs[i]);
    g_nalloc = 0;
}
