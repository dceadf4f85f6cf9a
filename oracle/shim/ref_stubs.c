/*
 * Abort-stubs for the FFTW and netCDF entry points that the reference
 * sources reference but that the e_iso / a_iso_3d trace paths never call.
 * Linked only into the oracle builds under oracle/_ref/.  Test infrastructure.
 */
#include <stdio.h>
#include <stdlib.h>
#include "fftw3.h"
#include "netcdf.h"

static void sm_shim_abort(const char *what)
{
    fprintf(stderr, "oracle shim: %s is not available in this build\n", what);
    abort();
}

void fftw_execute(const fftw_plan p) { (void)p; sm_shim_abort("fftw_execute"); }
void fftw_destroy_plan(fftw_plan p) { (void)p; sm_shim_abort("fftw_destroy_plan"); }
void *fftw_malloc(size_t n) { (void)n; sm_shim_abort("fftw_malloc"); return NULL; }
void fftw_free(void *p) { (void)p; sm_shim_abort("fftw_free"); }
int fftw_init_threads(void) { sm_shim_abort("fftw_init_threads"); return 0; }
void fftw_plan_with_nthreads(int n) { (void)n; sm_shim_abort("fftw_plan_with_nthreads"); }
int fftw_export_wisdom_to_file(FILE *f) { (void)f; sm_shim_abort("fftw_export_wisdom_to_file"); return 0; }
int fftw_import_wisdom_from_file(FILE *f) { (void)f; sm_shim_abort("fftw_import_wisdom_from_file"); return 0; }
fftw_plan fftw_plan_many_dft_r2c(int a, const int *b, int c, double *d, const int *e, int f, int g,
                                 fftw_complex *h, const int *i, int j, int k, unsigned l)
{ (void)a;(void)b;(void)c;(void)d;(void)e;(void)f;(void)g;(void)h;(void)i;(void)j;(void)k;(void)l;
  sm_shim_abort("fftw_plan_many_dft_r2c"); return NULL; }
fftw_plan fftw_plan_many_dft_c2r(int a, const int *b, int c, fftw_complex *d, const int *e, int f, int g,
                                 double *h, const int *i, int j, int k, unsigned l)
{ (void)a;(void)b;(void)c;(void)d;(void)e;(void)f;(void)g;(void)h;(void)i;(void)j;(void)k;(void)l;
  sm_shim_abort("fftw_plan_many_dft_c2r"); return NULL; }

int nc_create(const char *p, int m, int *id) { (void)p;(void)m;(void)id; sm_shim_abort("nc_create"); return 1; }
int nc_def_dim(int a, const char *b, size_t c, int *d) { (void)a;(void)b;(void)c;(void)d; sm_shim_abort("nc_def_dim"); return 1; }
int nc_def_var(int a, const char *b, nc_type c, int d, const int *e, int *f) { (void)a;(void)b;(void)c;(void)d;(void)e;(void)f; sm_shim_abort("nc_def_var"); return 1; }
int nc_put_att_text(int a, int b, const char *c, size_t d, const char *e) { (void)a;(void)b;(void)c;(void)d;(void)e; sm_shim_abort("nc_put_att_text"); return 1; }
int nc_put_att_int(int a, int b, const char *c, nc_type d, size_t e, const int *f) { (void)a;(void)b;(void)c;(void)d;(void)e;(void)f; sm_shim_abort("nc_put_att_int"); return 1; }
int nc_put_att_double(int a, int b, const char *c, nc_type d, size_t e, const double *f) { (void)a;(void)b;(void)c;(void)d;(void)e;(void)f; sm_shim_abort("nc_put_att_double"); return 1; }
int nc_put_var_double(int a, int b, const double *c) { (void)a;(void)b;(void)c; sm_shim_abort("nc_put_var_double"); return 1; }
int nc_put_vara_float(int a, int b, const size_t *c, const size_t *d, const float *e) { (void)a;(void)b;(void)c;(void)d;(void)e; sm_shim_abort("nc_put_vara_float"); return 1; }
int nc_enddef(int a) { (void)a; sm_shim_abort("nc_enddef"); return 1; }
int nc_close(int a) { (void)a; sm_shim_abort("nc_close"); return 1; }
const char *nc_strerror(int e) { (void)e; return "netCDF unavailable in the oracle build"; }
