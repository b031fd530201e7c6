/*
 * hh_dropin3d.h -- drop-in replacement for the 3D program's solver entry points.
 *
 * libhh3d.so exports, with the reference's names and by-value struct ABI:
 *   void solver(System sys)   -- 3D_Program/solver_functions/solver.c:263 (CPU) / :55 (GPU)
 *   void DST(int Nx, int Ny, double *b_2D, double *bhat, p1, in1, out1, p2, in2, out2)
 *                             -- 3D_Program/solver_functions/DST.c:148 (FFTW) / :88 (cuFFT)
 *
 * The struct types reproduce 3D_Program/headers/structs.h:39-58 field for field (312-byte
 * System) under hh3d_ names.  Plan/buffer arguments of DST are accepted and ignored.
 *
 * Semantics: solver() reads sys.rhs and the per-layer stencil sys.a..sys.dm, rebuilds the
 * z-line factors on the GPU (sys.L/U/Up from LU() are not read) and writes sys.sol on the
 * host.  DST() writes bhat and, unlike the reference (which leaves its x-pass intermediate in
 * b_2D, DST.c:175-179), does not modify b_2D.  Errors go to stderr and hh3d_status().
 */
#ifndef HH_DROPIN3D_H
#define HH_DROPIN3D_H

#ifdef __cplusplus
extern "C" {
#endif

enum hh3d_order { hh3d_second, hh3d_fourth, hh3d_sixth };

typedef struct {
    int    Nx, Ny, Nz, Nxyz;
    double hx, hy, hz, x0, x1, y0, y1, z0, z1;
} hh3d_Lattice;

typedef struct {
    hh3d_Lattice    lat;
    enum hh3d_order order;
    double _Complex *a;
    double _Complex *b, *c, *d, *ap, *bp, *cp, *dp, *am, *bm, *cm, *dm;
    double _Complex *k_bg_ext, *k2_bg_ext;
    double A, B, C, beta, gamma;
    double _Complex *sol_analytic, *rhs;
    double _Complex *L, *U, *Up;
    double _Complex *sol, *res, *error;
} hh3d_System;

void solver(hh3d_System sys);
void DST(int Nx, int Ny, double *b_2D, double *bhat, void *p1, double *in1, void *out1, void *p2, double *in2,
         void *out2);
int  hh3d_status(void);

#ifdef __cplusplus
}
#endif

#endif
