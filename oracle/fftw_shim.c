/*
 * FFTW3-API shim over the oracle's own DFT (fft_ref.c).  Test infrastructure only:
 * it lets the reference's unchanged CPU sources (2D_Program/solver_functions/*.c,
 * 3D_Program/solver_functions/*.c) build into oracle/_ref/ as the parity reference and
 * the timed CPU baseline.  FFTW3 is a third-party dependency of the reference that is
 * absent here (version unpinned); the shim implements only the real-to-complex
 * forward transforms the reference plans (r2c 1D and "many" rank-1 r2c), following the
 * documented FFTW semantics: unnormalised X[k] = sum_n x[n] e^{-2 pi i k n / L},
 * k = 0..L/2, with FFTW's stride/dist addressing.
 *
 * Plans are independent objects, so concurrent execution of different plans from
 * several OpenMP threads (as 2D solver.c does under USE_OMP) is safe.
 */
#include "shim/fftw3.h"
#include "fft_ref.h"

#include <stdlib.h>
#include <string.h>

struct hh_shim_plan {
    int     n, howmany, istride, idist, ostride, odist;
    double *in;
    double *out; /* interleaved (re,im) */
    double *stage_in;
    double *stage_out;
    ora_fft fft;
};

static fftw_plan make_plan(int n, int howmany, double *in, int istride, int idist,
                           void *out, int ostride, int odist) {
    struct hh_shim_plan *p = (struct hh_shim_plan *)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->n = n;
    p->howmany = howmany;
    p->in = in;
    p->out = (double *)out;
    p->istride = istride;
    p->idist = idist;
    p->ostride = ostride;
    p->odist = odist;
    p->stage_in = (double *)malloc(sizeof(double) * (size_t)n);
    p->stage_out = (double *)malloc(sizeof(double) * 2 * (size_t)(n / 2 + 1));
    if (!p->stage_in || !p->stage_out || ora_fft_init(&p->fft, n) != 0) {
        free(p->stage_in);
        free(p->stage_out);
        free(p);
        return NULL;
    }
    return p;
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags) {
    (void)flags;
    return make_plan(n, 1, in, 1, n, out, 1, n / 2 + 1);
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride, int idist,
                                 fftw_complex *out, const int *onembed, int ostride, int odist,
                                 unsigned flags) {
    (void)inembed;
    (void)onembed;
    (void)flags;
    if (rank != 1) return NULL; /* the reference only plans rank-1 batches */
    return make_plan(n[0], howmany, in, istride, idist, out, ostride, odist);
}

void fftw_execute(const fftw_plan p) {
    if (!p) return;
    const int nc = p->n / 2 + 1;
    for (int h = 0; h < p->howmany; h++) {
        const double *src = p->in + (size_t)h * (size_t)p->idist;
        for (int t = 0; t < p->n; t++) p->stage_in[t] = src[(size_t)t * (size_t)p->istride];
        ora_fft_r2c(&p->fft, p->stage_in, p->stage_out);
        double *dst = p->out + 2 * (size_t)h * (size_t)p->odist;
        for (int k = 0; k < nc; k++) {
            dst[2 * (size_t)k * (size_t)p->ostride]     = p->stage_out[2 * k];
            dst[2 * (size_t)k * (size_t)p->ostride + 1] = p->stage_out[2 * k + 1];
        }
    }
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    ora_fft_free(&p->fft);
    free(p->stage_in);
    free(p->stage_out);
    free(p);
}

/* plain malloc: the reference releases some fftw_malloc buffers with free()
 * (2D_Program/solver_functions/solver.c:99,101). */
void *fftw_malloc(size_t n) { return malloc(n); }
void  fftw_free(void *p) { free(p); }
