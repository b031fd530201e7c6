/*
 * ORACLE -- CPU restatement of gonzrona/hackathon's compact Helmholtz direct-solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (hackathon_b200/, include/) links,
 * loads or calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only to check results or to time the CPU baseline.
 *
 * Pinning: every function here is checked against the reference's own C sources built
 * unchanged into oracle/_ref/ (tests/golden/make_golden.py writes those outputs as
 * fixtures; tests/test_oracle.py compares).  The reference has no tests or golden
 * vectors of its own.
 *
 * Conventions (as the reference): complex double, x fastest.  2D interior index
 * i + j*Nx (2D_Program/headers/structs.h:9); extended (Nx+2)x(Ny+2) grid index
 * ie + je*(Nx+2).  3D interior i + j*Nx + l*Nx*Ny; extended likewise with (Nx+2),(Ny+2).
 * Problem data that the reference evaluates through user callbacks (f, k, boundary
 * derivatives, Dirichlet data) is passed here as sampled arrays; a NULL array means
 * "identically zero".
 */
#ifndef HH_ORACLE_H
#define HH_ORACLE_H

#include <complex.h>

typedef double _Complex ora_cplx;

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ DST-I ---- */
/* Orthonormal DST-I along contiguous rows of length n (the reference's forwardDST /
 * reverseDST kernel, 2D_Program/solver_functions/DST.c:6-24,26-44): each of the real and
 * imaginary planes is zero-padded to L = 2n+2, forward real DFT, keep -Im(bin i+1),
 * scale sqrt(2/(n+1)).  Returns 0 on success. */
int ora_dst1_rows(int n, long rows, const ora_cplx *in, long in_ld, ora_cplx *out, long out_ld);

/* 2D DST-I of one REAL Nx x Ny plane exactly as 3D_Program/solver_functions/DST.c:148-204:
 * x-pass, transpose, y-pass, then one scale by 2/sqrt(Nx+1)/sqrt(Ny+1). */
int ora_dst2_plane_real(int nx, int ny, const double *in, double *out);

/* ---------------------------------------------------------------------- 2D ---- */
typedef struct {
    int    nx, ny, order;          /* order 2, 4 or 6                                  */
    double x0, x1, y0, y1, hx, hy;
    const ora_cplx *k_ext;         /* k(y0 + j*hy), j = 0..ny+1                        */
    const ora_cplx *k2y_ext;       /* analytic d(k^2)/dy at y0 + j*hy, j = 0..ny+1     */
    const ora_cplx *k2yy;          /* analytic d2(k^2)/dy2 at interior rows, ny        */
    const ora_cplx *f_ext;         /* f on the extended grid, (nx+2)*(ny+2)            */
    const ora_cplx *fxx_xb;        /* f_xx on x=x0 (je=0..ny+1) then x=x1: 2*(ny+2)    */
    const ora_cplx *fxx_yb;        /* f_xx on y=y0 (ie=0..nx+1) then y=y1: 2*(nx+2)    */
    const ora_cplx *fyy_xb;        /* f_yy on x=x0, x=x1: 2*(ny+2)                     */
    const ora_cplx *fyy_yb;        /* f_yy on y=y0, y=y1: 2*(nx+2)                     */
    const ora_cplx *fy_yb;         /* f_y on y=y0 at interior x (nx) then y=y1: 2*nx   */
    const double   *u_xb;          /* Dirichlet data on x=x0, x=x1: 2*(ny+2) (real)    */
    const double   *u_yb;          /* Dirichlet data on y=y0, y=y1: 2*(nx+2) (real)    */
} ora_problem2d;

typedef struct {                   /* per-row 9-point stencil [bm am bm; b a b; bp ap bp] */
    ora_cplx *bp, *ap, *b, *a, *bm, *am;   /* each ny                                   */
} ora_coef2d;

/* 2D_Program/main_functions/coefficients.c:9-67 */
void ora_coefficients_2d(const ora_problem2d *pb, ora_coef2d *c);
/* 2D_Program/main_functions/rhs.c:4-150 with partial_derivatives/*.c: writes nx*ny. */
void ora_rhs_2d(const ora_problem2d *pb, const ora_coef2d *c, ora_cplx *rhs);
/* 2D_Program/main_functions/LU.c:3-46: factors stored line-major [j + i*ny]; U = pivot. */
void ora_lu_2d(int nx, int ny, const ora_coef2d *c, ora_cplx *L, ora_cplx *U, ora_cplx *Up);
/* 2D_Program/solver_functions/solver.c:14-117 (forward DST, per-mode Thomas, inverse). */
int  ora_solver_2d(int nx, int ny, const ora_cplx *rhs, const ora_cplx *L, const ora_cplx *U,
                   const ora_cplx *Up, ora_cplx *sol);
/* solver.c:14-117 with the per-mode Thomas solves in long double: the exact solution of the
 * discrete system to ~1e-18 relative per line, for measuring rounding error on ill-conditioned
 * (near-resonant) lines.  Factors are formed from the stencil rows as LU.c:12-40 does. */
int  ora_solver_2d_ld(int nx, int ny, const ora_coef2d *c, const ora_cplx *rhs, ora_cplx *sol);
/* 2D_Program/main_functions/residual.c:3-34: res = A*sol - rhs (zero Dirichlet ring). */
void ora_residual_2d(int nx, int ny, const ora_coef2d *c, const ora_cplx *sol, const ora_cplx *rhs,
                     ora_cplx *res);

/* ---------------------------------------------------------------------- 3D ---- */
typedef struct {                   /* per-layer 27-point stencil, each nz               */
    ora_cplx *a, *b, *c, *d, *ap, *bp, *cp, *dp, *am, *bm, *cm, *dm;
} ora_coef3d;

typedef struct {
    int    nx, ny, nz, order;
    double hx, hy, hz;
    const ora_cplx *k2_ext;        /* k^2 at z0 + l*hz, l = 0..nz+1                    */
    /* 6th order only: boundary values that 4th_order_partials.c:314-315,359-360 add to the
     * Pade right-hand sides of d(k^2)/dz and d2(k^2)/dz2 (the reference hard-codes them for
     * k = A - B sin(Cz)); NULL = zero. Each holds {value at z0, value at z1}. */
    const ora_cplx *kz_bc, *kzz_bc;
    const ora_cplx *rhs_ext;       /* h_z^2-scaled source on the extended grid          */
    const ora_cplx *ue_ext;        /* Dirichlet data; only layers l=0 and l=nz+1 are read */
    const ora_cplx *fxx_b, *fyy_b, *fzz_b; /* boundary second derivatives (6th order),
                                      layouts of 3D rhs.c:83-109; NULL = zero           */
} ora_problem3d;

/* d(k^2)/dz by the [1 4 1] Pade scheme, 3D_Program/partial_derivatives/4th_order_partials.c:296-340 */
void ora_kz_3d(int nz, double hz, const ora_cplx *k2_ext, const ora_cplx *bc, ora_cplx *kz);
/* d2(k^2)/dz2 by the [1 10 1] Pade scheme, 4th_order_partials.c:342-385 */
void ora_kzz_3d(int nz, double hz, const ora_cplx *k2_ext, const ora_cplx *bc, ora_cplx *kzz);
/* 3D_Program/main_functions/coefficients.c:293-397 */
void ora_coefficients_3d(const ora_problem3d *pb, ora_coef3d *c);
/* 3D_Program/main_functions/rhs.c:13-194 (interior assembly + z-face Dirichlet terms). */
void ora_rhs_3d(const ora_problem3d *pb, const ora_coef3d *c, ora_cplx *rhs);
/* 3D_Program/main_functions/LU.c:4-81: factors [l + i*nz + j*nx*nz]; U = reciprocal. */
void ora_lu_3d(int nx, int ny, int nz, const ora_coef3d *c, ora_cplx *L, ora_cplx *U, ora_cplx *Up);
/* 3D_Program/solver_functions/solver.c:390-540 (CPU path). */
int  ora_solver_3d(int nx, int ny, int nz, const ora_cplx *rhs, const ora_cplx *L, const ora_cplx *U,
                   const ora_cplx *Up, ora_cplx *sol);
/* 3D_Program/main_functions/residual.c:42-96 */
void ora_residual_3d(int nx, int ny, int nz, const ora_coef3d *c, const ora_cplx *sol,
                     const ora_cplx *rhs, ora_cplx *res);

#ifdef __cplusplus
}
#endif

#endif
