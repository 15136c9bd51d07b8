/* Runtime for the mechanically translated reference (oracle/f2c_ref.py).
 * TEST INFRASTRUCTURE ONLY: guarded zero-filled arrays, named input files for
 * the reference's list-directed READs, parameter overrides. */
#pragma once
#include <stddef.h>

int *ref_alloc_int(long n);
double *ref_alloc_dbl(long n);
void ref_open(int unit, const char *name);
void ref_read_begin(int unit);
void ref_read_int(int *v);
void ref_read_dbl(double *v);
void ref_read_end(int unit);
int ref_param_overridden(const char *name);
double ref_param_value(const char *name);
int ref_strcmp(const char *a, const char *b);
void ref_unknown_call(const char *name);
