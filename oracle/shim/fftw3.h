/*
 * Minimal FFTW3 API declarations for compiling the reference's CPU path against the
 * oracle's own DFT (oracle/fftw_shim.c).  Test infrastructure only.
 *
 * FFTW3 itself is absent from this image; only the subset of its documented interface
 * that the reference calls is declared here:
 *   2D_Program/solver_functions/solver.c:42-45,61-62,99-105 and DST.c:18-19,38-39
 *   3D_Program/solver_functions/solver.c:428-454,517-522 and DST.c:171,189
 * fftw_complex follows FFTW's documented rule: the C99 complex type when <complex.h>
 * was included first, otherwise double[2].
 */
#ifndef HH_SHIM_FFTW3_H
#define HH_SHIM_FFTW3_H

#include <stddef.h>

#if defined(_Complex_I) && defined(complex) && defined(I)
typedef double _Complex fftw_complex;
#else
typedef double fftw_complex[2];
#endif

typedef struct hh_shim_plan *fftw_plan;

#define FFTW_ESTIMATE (1U << 6)

#ifdef __cplusplus
extern "C" {
#endif

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags);
void  fftw_execute(const fftw_plan plan);
void  fftw_destroy_plan(fftw_plan plan);
void *fftw_malloc(size_t n);
void  fftw_free(void *p);

#ifdef __cplusplus
}
#endif

#endif
