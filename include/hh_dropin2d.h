/*
 * hh_dropin2d.h -- drop-in replacement for the 2D program's solver entry points.
 *
 * libhh2d.so exports, with the reference's names and by-value struct ABI:
 *   void solver(System sys)        -- 2D_Program/solver_functions/solver.c:14
 *   void forwardDST(...)           -- 2D_Program/solver_functions/DST.c:6
 *   void reverseDST(...)           -- 2D_Program/solver_functions/DST.c:26
 * A reference build links them instead of solver.o and DST.o; its own main(), setup,
 * coefficients(), rhs(), LU() and residual() stay unchanged.
 *
 * The struct types below reproduce 2D_Program/headers/structs.h:12-30 field for field (same
 * sizes and offsets, 192-byte System) under hh2d_ names so this header can be included next
 * to the reference's own.  The FFTW plan/buffer arguments of forwardDST/reverseDST are
 * accepted and ignored (declared as void *, ABI-identical to the reference's pointer types);
 * dst.Nx (transform length, 1..sys.lat.Nx) and dst.coef (output scale) are honoured as in
 * DST.c:15-21,35-40.  Device and host staging are kept between calls, so a loop of calls does not
 * allocate per call.
 *
 * Semantics: solver() reads sys.rhs and the stencil rows sys.bp..sys.am, rebuilds the shifted
 * Thomas factors on the GPU (the values LU() leaves in sys.L/U/Up are not read), and writes
 * sys.sol on the host.  Errors are printed to stderr like the reference's CUDA_RT_CALL and
 * leave sys.sol untouched; hh2d_status() returns the last status (include/hh.h codes).
 * The GPU device is 0 unless HH_DEVICE is set.
 */
#ifndef HH_DROPIN2D_H
#define HH_DROPIN2D_H

#ifdef __cplusplus
extern "C" {
#endif

enum hh2d_order { hh2d_second, hh2d_fourth, hh2d_sixth };

typedef struct {
    int    Nx, N;
    double coef;
} hh2d_DSTN;

typedef struct {
    int    Nx, Ny, Nxy;
    double hx, hy, x0, x1, y0, y1;
} hh2d_Lattice;

typedef struct {
    hh2d_Lattice    lat;
    int             threadCount;
    enum hh2d_order order;
    double _Complex *k, *rhs, *L, *U, *Up, *sol, *sol_analytic, *res, *error;
    double _Complex *bp, *ap, *b, *a, *bm, *am;
} hh2d_System;

void solver(hh2d_System sys);
void forwardDST(hh2d_System sys, hh2d_DSTN dst, double _Complex *rhs, double _Complex *rhat, void *plan, double *in,
                void *out, void *plan2, double *in2, void *out2);
void reverseDST(hh2d_System sys, hh2d_DSTN dst, double _Complex *xhat, double _Complex *sol, void *plan, double *in,
                void *out, void *plan2, double *in2, void *out2);
int  hh2d_status(void);

#ifdef __cplusplus
}
#endif

#endif
