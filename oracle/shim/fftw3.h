/*
 * Stand-in declarations for the FFTW 3 interface, used ONLY to compile the
 * reference sources (propagate.c, io_utils.c via structs.h) into the oracle
 * under oracle/_ref/.  FFTW is absent from this image and is never called on
 * the e_iso / a_iso_3d paths; every function here is defined in ref_stubs.c
 * as an abort.  Test infrastructure, not product code.
 */
#ifndef SM_SHIM_FFTW3_H
#define SM_SHIM_FFTW3_H
#include <stdio.h>
#include <stddef.h>
#include <complex.h>

typedef double _Complex fftw_complex;
typedef struct sm_shim_fftw_plan_s *fftw_plan;

#define FFTW_PATIENT (1U << 5)

void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
int fftw_export_wisdom_to_file(FILE *output_file);
int fftw_import_wisdom_from_file(FILE *input_file);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
#endif
