/*
 * CPU discrete Fourier transform used by the oracle (test infrastructure only).
 *
 * This is NOT part of the product: only tests/, the smoke check and the bench's
 * CPU-baseline leg load code from oracle/.  It exists because FFTW3 (the library the
 * reference links, `-lfftw3_omp -lfftw3` in 2D_Program/Makefile:16-19 and
 * 3D_Program/Makefile:33-36; version unpinned, not vendored) is absent from this image.
 *
 * What it computes is the textbook unnormalised forward DFT that FFTW documents for
 * its r2c/c2c transforms:  X[k] = sum_n x[n] exp(-2 pi i k n / L).
 *   - L a power of two: iterative radix-2 decimation-in-time with a twiddle table
 *     computed directly by sin/cos (no recurrences, so error ~ log2(L) ulp).
 *   - any other L: direct O(L^2) summation with exact index reduction (k*n mod L).
 */
#ifndef HH_ORACLE_FFT_REF_H
#define HH_ORACLE_FFT_REF_H

#include <stddef.h>

typedef struct ora_fft {
    int     len;      /* transform length L                                  */
    int     pow2;     /* 1 if L is a power of two                            */
    double *cs;       /* cos(2 pi t / L), t = 0..L-1                         */
    double *sn;       /* sin(2 pi t / L), t = 0..L-1                         */
    int    *rev;      /* bit-reversal permutation (power-of-two only)        */
    double *work;     /* 4*L doubles of scratch (interleaved re,im)          */
} ora_fft;

/* Returns 0 on success. */
int  ora_fft_init(ora_fft *p, int len);
void ora_fft_free(ora_fft *p);

/* In-place forward complex DFT on interleaved (re,im) data of length L. */
void ora_fft_c2c(const ora_fft *p, double *data);

/* Forward DFT of L real samples; writes the first L/2+1 complex bins (interleaved). */
void ora_fft_r2c(const ora_fft *p, const double *in, double *out);

#endif
