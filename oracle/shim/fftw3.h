/*
 * FFTW-API shim: test infrastructure for building the reference solver
 * (MHD2DCFDFFTW) from its own, unmodified sources in a container without
 * FFTW.  It offers exactly the subset the reference calls
 * (calcDerivs.c:89,101,130,142; filtering.c:55,86; initialize.c:323-326):
 * 1-D real-to-complex and complex-to-real plans with FFTW's conventions
 * (both directions unnormalised; r2c writes n/2+1 bins with zero imaginary
 * parts at DC and, for even n, at Nyquist; c2r ignores those imaginary parts).
 * The transforms are this project's own code (fftshim.c).
 */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct oracle_fftw_plan *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif
#endif
