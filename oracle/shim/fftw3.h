/*
 * FFTW 3 API subset -- TEST INFRASTRUCTURE ONLY (oracle build).
 *
 * The reference pins FFTW 3.3.4 only through its include path
 * (Makefile:7-8); the library is not vendored and is absent here.  This header
 * declares the few entry points fft.c uses (fft.c:38-63 r2c/c2r "many" plans,
 * fft.c:97-118 rank-1 guru c2c plans, fft.c:161-208 execute) plus the
 * allocator used by d3tensor.c/c3tensor.c.  The implementation
 * (fftw_shim.c) follows FFTW's published conventions: unnormalised
 * transforms, forward sign e^{-i}, backward sign e^{+i}, c2r reading only the
 * non-redundant half spectrum and ignoring the imaginary parts of the DC and
 * Nyquist bins.  FFTW's exact output bits are not reproduced (its algorithm
 * choice under FFTW_MEASURE is timing dependent even in the real library).
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct shim_fftw_plan *fftw_plan;
typedef struct { int n, is, os; } fftw_iodim;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)

void *fftw_malloc(size_t n);
void fftw_free(void *p);

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed, int istride, int idist,
                                 double *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_guru_dft(int rank, const fftw_iodim *dims,
                             int howmany_rank, const fftw_iodim *howmany_dims,
                             fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* Shim extra (not an FFTW symbol): unnormalised 1-D complex DFT of length n,
 * unit stride, used by the oracle's own tests of this shim. */
void shim_fft_c2c(int n, int sign, const fftw_complex *in, fftw_complex *out);

#ifdef __cplusplus
}
#endif

#endif
