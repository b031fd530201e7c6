/*
 * ORACLE -- CPU restatement of gonzrona/hackathon's compact Helmholtz direct-solver path.
 * TEST INFRASTRUCTURE ONLY (see hh_oracle.h).  Not linked into the product.
 *
 * Floating-point operations are performed in the same order as the cited reference lines
 * so that, compiled by the same gcc with the same flags, results agree with the reference
 * built in oracle/_ref/ to the last bit wherever the reference is deterministic.
 * Deliberate, documented deviations (all invisible for zero boundary data):
 *   - 3D_Program/main_functions/rhs.c:149 holds the five 6th-order partial sums in `double`,
 *     dropping the imaginary part of a complex source; ora_problem3d keeps the complex sums
 *     unless `ref_real_sums` is requested through ora_set_3d_real_sums().
 *   - 3D_Program/partial_derivatives/4th_order_partials.c:144 writes the x = x1 ghost column
 *     of f_xx at a wrong index; here it is written where it belongs.
 */
#include "hh_oracle.h"
#include "fft_ref.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef ora_cplx cplx;

static int g_real_sums_3d = 0;
void ora_set_3d_real_sums(int on) { g_real_sums_3d = on; }

/* ============================================================= transforms ====== */

int ora_dst1_rows(int n, long rows, const cplx *in, long in_ld, cplx *out, long out_ld) {
    const int L = 2 * n + 2;
    ora_fft   fft;
    if (ora_fft_init(&fft, L) != 0) return -1;
    double *re = (double *)calloc((size_t)L, sizeof(double));
    double *im = (double *)calloc((size_t)L, sizeof(double));
    double *bre = (double *)malloc(sizeof(double) * 2 * (size_t)(L / 2 + 1));
    double *bim = (double *)malloc(sizeof(double) * 2 * (size_t)(L / 2 + 1));
    const double coef = sqrt(2.0 / (n + 1));
    for (long r = 0; r < rows; r++) {
        const cplx *src = in + r * in_ld;
        cplx       *dst = out + r * out_ld;
        for (int i = 0; i < n; i++) re[i + 1] = creal(src[i]);
        for (int i = 0; i < n; i++) im[i + 1] = cimag(src[i]);
        ora_fft_r2c(&fft, re, bre);
        ora_fft_r2c(&fft, im, bim);
        for (int i = 0; i < n; i++) {
            /* coef * (-Im(bin) - I*Im(bin2)), component-wise */
            double a = -bre[2 * (i + 1) + 1];
            double b = -bim[2 * (i + 1) + 1];
            dst[i] = CMPLX(coef * a, coef * b);
        }
    }
    free(re); free(im); free(bre); free(bim);
    ora_fft_free(&fft);
    return 0;
}

int ora_dst2_plane_real(int nx, int ny, const double *in, double *out) {
    const int Lx = 2 * nx + 2, Ly = 2 * ny + 2;
    ora_fft   fx, fy;
    if (ora_fft_init(&fx, Lx) != 0) return -1;
    if (ora_fft_init(&fy, Ly) != 0) { ora_fft_free(&fx); return -1; }
    double *stage = (double *)calloc((size_t)((Lx > Ly) ? Lx : Ly), sizeof(double));
    double *bins  = (double *)malloc(sizeof(double) * 2 * (size_t)(((Lx > Ly) ? Lx : Ly) / 2 + 1));
    double *mid   = (double *)malloc(sizeof(double) * (size_t)nx * (size_t)ny);
    const double coef = 2.0 / sqrt(nx + 1) / sqrt(ny + 1);
    /* x-pass: keep Im(bin i+1) of each row (no sign flip; the two flips cancel) */
    for (int j = 0; j < ny; j++) {
        memset(stage, 0, sizeof(double) * (size_t)Lx);
        for (int i = 0; i < nx; i++) stage[i + 1] = in[i + (long)j * nx];
        ora_fft_r2c(&fx, stage, bins);
        for (int i = 0; i < nx; i++) mid[i + (long)j * nx] = bins[2 * (i + 1) + 1];
    }
    /* y-pass over columns */
    for (int i = 0; i < nx; i++) {
        memset(stage, 0, sizeof(double) * (size_t)Ly);
        for (int j = 0; j < ny; j++) stage[j + 1] = mid[i + (long)j * nx];
        ora_fft_r2c(&fy, stage, bins);
        for (int j = 0; j < ny; j++) out[i + (long)j * nx] = bins[2 * (j + 1) + 1];
    }
    for (long t = 0; t < (long)nx * ny; t++) out[t] = coef * out[t];
    free(stage); free(bins); free(mid);
    ora_fft_free(&fx); ora_fft_free(&fy);
    return 0;
}

/* ========================================================== line solvers ====== */

/* Constant-diagonal Pade system tridiag(1, diag, 1) solved in place along a strided line
 * of n points, factor recurrence U_0 = diag, L_j = 1/U_{j-1}, U_j = diag - L_j
 * (2D_Program/partial_derivatives/4th_order_first_derivative.c:41-54,
 *  3D_Program/partial_derivatives/4th_order_partials.c:118-139). */
static void pade_line(cplx *v, long stride, int n, const double *Lf, const double *Uf) {
    for (int j = 1; j < n; j++) v[j * stride] = v[j * stride] - Lf[j] * v[(j - 1) * stride];
    v[(n - 1) * stride] = v[(n - 1) * stride] / Uf[n - 1];
    for (int j = n - 2; j >= 0; j--) v[j * stride] = (v[j * stride] - v[(j + 1) * stride]) / Uf[j];
}

static void pade_factors(int n, double diag, double *Lf, double *Uf) {
    Lf[0] = 0.0;
    Uf[0] = diag;
    for (int j = 1; j < n; j++) {
        Lf[j] = 1.0 / Uf[j - 1];
        Uf[j] = diag - Lf[j];
    }
}

/* ==================================================================== 2D ====== */

#define E2(ie, je) ((long)(ie) + (long)(je) * (long)(pb->nx + 2))

static cplx opt_c(const cplx *a, long i) { return a ? a[i] : 0.0; }
static double opt_d(const double *a, long i) { return a ? a[i] : 0.0; }

void ora_coefficients_2d(const ora_problem2d *pb, ora_coef2d *c) {
    const int ny = pb->ny;
    const double hx = pb->hx, hy = pb->hy;
    if (pb->order == 6) {
        /* coefficients.c:44-61 */
        const double hy2 = hy * hy, hy3 = hy2 * hy, hy4 = hy2 * hy2;
        for (int j = 0; j < ny; j++) {
            cplx k0 = pb->k_ext[j + 1], kp = pb->k_ext[j + 2], km = pb->k_ext[j];
            cplx k2 = k0 * k0, k2p = kp * kp, k2m = km * km;
            cplx ky2 = opt_c(pb->k2y_ext, j + 1);
            cplx kyy = opt_c(pb->k2yy, j);
            c->ap[j] = 2.0 / 3.0 + hy2 * k2p / 90.0 + hy3 * ky2 * (hy2 * k2p / 6.0 + 2.0 / 3.0) / 20.0;
            c->bp[j] = 1.0 / 6.0 + hy2 * k2p / 90.0 + hy3 * ky2 / 120.0;
            c->a[j]  = -10.0 / 3.0 + 41.0 * hy2 * k2 / 45.0 - hy4 * k2 * k2 / 20.0 + hy4 * kyy / 20.0;
            c->b[j]  = 2.0 / 3.0 + hy2 * k2 / 90.0;
            c->am[j] = 2.0 / 3.0 + hy2 * k2m / 90.0 - hy3 * ky2 * (hy2 * k2m / 6.0 + 2.0 / 3.0) / 20.0;
            c->bm[j] = 1.0 / 6.0 + hy2 * k2m / 90.0 - hy3 * ky2 / 120.0;
        }
    } else if (pb->order == 4) {
        /* coefficients.c:25-42 */
        const double hy2 = hy * hy, Ryx = hy * hy / hx / hx;
        for (int j = 0; j < ny; j++) {
            cplx k0 = pb->k_ext[j + 1], kp = pb->k_ext[j + 2], km = pb->k_ext[j];
            cplx k2 = k0 * k0, k2p = kp * kp, k2m = km * km;
            c->bp[j] = Ryx / 12.0 + 1.0 / 12.0;
            c->ap[j] = 5.0 / 6.0 - Ryx / 6.0 + hy2 * k2p / 12.0;
            c->b[j]  = Ryx * (5.0 / 6.0) - 1.0 / 6.0 + hy2 * k2 / 12.0;
            c->a[j]  = -Ryx * (5.0 / 3.0) - 5.0 / 3.0 + 2.0 * hy2 * k2 / 3.0;
            c->bm[j] = Ryx / 12.0 + 1.0 / 12.0;
            c->am[j] = 5.0 / 6.0 - Ryx / 6.0 + hy2 * k2m / 12.0;
        }
    } else {
        /* coefficients.c:9-23 */
        const double hy2 = hy * hy, Ryx = hy * hy / hx / hx;
        for (int j = 0; j < ny; j++) {
            cplx k0 = pb->k_ext[j + 1];
            c->bp[j] = 0.0;
            c->ap[j] = 1.0;
            c->b[j]  = Ryx;
            c->a[j]  = -2.0 * Ryx - 2.0 + k0 * k0 * hy2;
            c->bm[j] = 0.0;
            c->am[j] = 1.0;
        }
    }
}

/* 6th-order assembly, rhs.c:40-97 with the partial-derivative helpers. */
static void rhs6_2d(const ora_problem2d *pb, cplx *rhs) {
    const int nx = pb->nx, ny = pb->ny;
    const long nxy = (long)nx * ny, next = (long)(nx + 2) * (ny + 2);
    const double hx = pb->hx, hy = pb->hy, hy2 = hy * hy, hy4 = hy2 * hy2;
    const cplx *fe = pb->f_ext;
    cplx *fxx_e = (cplx *)calloc((size_t)next, sizeof(cplx));
    cplx *fyy_e = (cplx *)calloc((size_t)next, sizeof(cplx));
    cplx *fxx   = (cplx *)malloc(sizeof(cplx) * (size_t)nxy);
    cplx *fyy   = (cplx *)malloc(sizeof(cplx) * (size_t)nxy);
    cplx *fy    = (cplx *)malloc(sizeof(cplx) * (size_t)nxy);
    cplx *k2y   = (cplx *)malloc(sizeof(cplx) * (size_t)ny);
    int   nmax  = nx > ny ? nx : ny;
    double *Lf = (double *)malloc(sizeof(double) * (size_t)nmax);
    double *Uf = (double *)malloc(sizeof(double) * (size_t)nmax);

    /* f_y: [1 4 1] Pade along y, 4th_order_first_derivative.c:60-98 */
    pade_factors(ny, 4.0, Lf, Uf);
    for (int i = 0; i < nx; i++) {
        for (int j = 0; j < ny; j++)
            fy[i + (long)j * nx] = 3.0 * (fe[E2(i + 1, j + 2)] - fe[E2(i + 1, j)]) / hy;
        fy[i] = fy[i] - opt_c(pb->fy_yb, i);
        fy[i + (long)(ny - 1) * nx] = fy[i + (long)(ny - 1) * nx] - opt_c(pb->fy_yb, nx + i);
        pade_line(fy + i, nx, ny, Lf, Uf);
    }
    /* d(k^2)/dy: same scheme on the k^2 profile, 4th_order_first_derivative.c:28-58 */
    for (int j = 0; j < ny; j++) {
        cplx kp = pb->k_ext[j + 2], km = pb->k_ext[j];
        k2y[j] = 3.0 * (kp * kp - km * km) / hy;
    }
    k2y[0] = k2y[0] - opt_c(pb->k2y_ext, 0);
    k2y[ny - 1] = k2y[ny - 1] - opt_c(pb->k2y_ext, ny + 1);
    pade_line(k2y, 1, ny, Lf, Uf);

    /* f_yy: [1 10 1] Pade along y, 4th_order_second_derivative.c:61-120 */
    pade_factors(ny, 10.0, Lf, Uf);
    for (int i = 0; i < nx; i++) {
        for (int j = 0; j < ny; j++)
            fyy[i + (long)j * nx] =
                12.0 * (fe[E2(i + 1, j + 2)] - 2.0 * fe[E2(i + 1, j + 1)] + fe[E2(i + 1, j)]) / hy / hy;
        fyy[i] = fyy[i] - opt_c(pb->fyy_yb, i + 1);
        fyy[i + (long)(ny - 1) * nx] = fyy[i + (long)(ny - 1) * nx] - opt_c(pb->fyy_yb, (nx + 2) + i + 1);
        pade_line(fyy + i, nx, ny, Lf, Uf);
    }
    for (int ie = 0; ie < nx + 2; ie++) {
        fyy_e[E2(ie, 0)] = opt_c(pb->fyy_yb, ie);
        fyy_e[E2(ie, ny + 1)] = opt_c(pb->fyy_yb, (nx + 2) + ie);
    }
    for (int je = 0; je < ny + 2; je++) {
        fyy_e[E2(0, je)] = opt_c(pb->fyy_xb, je);
        fyy_e[E2(nx + 1, je)] = opt_c(pb->fyy_xb, (ny + 2) + je);
    }
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) fyy_e[E2(i + 1, j + 1)] = fyy[i + (long)j * nx];

    /* f_xx: [1 10 1] Pade along x, 4th_order_second_derivative.c:4-59 */
    pade_factors(nx, 10.0, Lf, Uf);
    for (int j = 0; j < ny; j++) {
        cplx *row = fxx + (long)j * nx;
        for (int i = 0; i < nx; i++)
            row[i] = 12.0 * (fe[E2(i + 2, j + 1)] - 2.0 * fe[E2(i + 1, j + 1)] + fe[E2(i, j + 1)]) / hx / hx;
        row[0] = row[0] - opt_c(pb->fxx_xb, j + 1);
        row[nx - 1] = row[nx - 1] - opt_c(pb->fxx_xb, (ny + 2) + j + 1);
        pade_line(row, 1, nx, Lf, Uf);
    }
    for (int ie = 0; ie < nx + 2; ie++) {
        fxx_e[E2(ie, 0)] = opt_c(pb->fxx_yb, ie);
        fxx_e[E2(ie, ny + 1)] = opt_c(pb->fxx_yb, (nx + 2) + ie);
    }
    for (int je = 0; je < ny + 2; je++) {
        fxx_e[E2(0, je)] = opt_c(pb->fxx_xb, je);
        fxx_e[E2(nx + 1, je)] = opt_c(pb->fxx_xb, (ny + 2) + je);
    }
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) fxx_e[E2(i + 1, j + 1)] = fxx[i + (long)j * nx];

    /* combination, rhs.c:78-86, with the 2nd-order differences of 2nd_order.c:4-24 inline */
    const double hx2 = hx * hx, hyy = hy * hy;
    for (int j = 0; j < ny; j++) {
        cplx k0 = pb->k_ext[j + 1];
        cplx k2c = k0 * k0;
        for (int i = 0; i < nx; i++) {
            long c = E2(i + 1, j + 1);
            cplx fxxxx = (fxx_e[E2(i, j + 1)] - 2.0 * fxx_e[c] + fxx_e[E2(i + 2, j + 1)]) / hx2;
            cplx fxxyy = (fxx_e[E2(i + 1, j)] - 2.0 * fxx_e[c] + fxx_e[E2(i + 1, j + 2)]) / hyy;
            cplx fyyyy = (fyy_e[E2(i + 1, j)] - 2.0 * fyy_e[c] + fyy_e[E2(i + 1, j + 2)]) / hyy;
            rhs[i + (long)j * nx] =
                hy2 * ((1.0 - k2c * hy2 / 20.0) * fe[c] + hy2 * (fxx_e[c] + fyy_e[c]) / 12.0 +
                       hy4 * (fxxxx + fyyyy) / 360.0 + hy4 * fxxyy / 90.0 +
                       hy4 * k2y[j] * fy[i + (long)j * nx] / 60.0);
        }
    }
    free(fxx_e); free(fyy_e); free(fxx); free(fyy); free(fy); free(k2y); free(Lf); free(Uf);
}

void ora_rhs_2d(const ora_problem2d *pb, const ora_coef2d *c, cplx *rhs) {
    const int nx = pb->nx, ny = pb->ny;
    const double hy = pb->hy;
    const cplx *fe = pb->f_ext;
    if (pb->order == 6) {
        rhs6_2d(pb, rhs);
    } else if (pb->order == 4) {
        /* rhs.c:21-38 */
        const double hy2 = hy * hy, a = 2.0 / 3.0, b = 1.0 / 12.0;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
                rhs[i + (long)j * nx] =
                    hy2 * (a * fe[E2(i + 1, j + 1)] +
                           b * (fe[E2(i + 1, j)] + fe[E2(i + 1, j + 2)] + fe[E2(i, j + 1)] + fe[E2(i + 2, j + 1)]));
    } else {
        /* rhs.c:4-19 */
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) rhs[i + (long)j * nx] = hy * hy * fe[E2(i + 1, j + 1)];
    }
    /* Dirichlet corrections of the four edges and corners, rhs.c:126-148 */
    const double *ux = pb->u_xb, *uy = pb->u_yb;
    const long xb1 = ny + 2, yb1 = nx + 2; /* offsets of the x=x1 / y=y1 halves */
    const long top = (long)(ny - 1) * nx;
    rhs[0] = rhs[0] - c->bm[0] * opt_d(uy, 0) - c->am[0] * opt_d(uy, 1) - c->bm[0] * opt_d(uy, 2) -
             c->b[0] * opt_d(ux, 1) - c->bp[0] * opt_d(ux, 2);
    rhs[nx - 1] = rhs[nx - 1] - c->bm[0] * opt_d(uy, nx - 1) - c->am[0] * opt_d(uy, nx) -
                  c->bm[0] * opt_d(uy, nx + 1) - c->b[0] * opt_d(ux, xb1 + 1) - c->bp[0] * opt_d(ux, xb1 + 2);
    rhs[top] = rhs[top] - c->bm[ny - 1] * opt_d(ux, ny - 1) - c->b[ny - 1] * opt_d(ux, ny) -
               c->bp[ny - 1] * opt_d(uy, yb1 + 0) - c->ap[ny - 1] * opt_d(uy, yb1 + 1) -
               c->bp[ny - 1] * opt_d(uy, yb1 + 2);
    rhs[nx - 1 + top] = rhs[nx - 1 + top] - c->bm[ny - 1] * opt_d(ux, xb1 + ny - 1) -
                        c->b[ny - 1] * opt_d(ux, xb1 + ny) - c->bp[ny - 1] * opt_d(uy, yb1 + nx + 1) -
                        c->ap[ny - 1] * opt_d(uy, yb1 + nx) - c->bp[ny - 1] * opt_d(uy, yb1 + nx - 1);
    for (int j = 1; j < ny - 1; j++) {
        long my = (long)j * nx;
        rhs[my] = rhs[my] - c->b[j] * opt_d(ux, j + 1) - c->bm[j] * opt_d(ux, j) - c->bp[j] * opt_d(ux, j + 2);
        rhs[my + nx - 1] = rhs[my + nx - 1] - c->b[j] * opt_d(ux, xb1 + j + 1) -
                           c->bm[j] * opt_d(ux, xb1 + j) - c->bp[j] * opt_d(ux, xb1 + j + 2);
    }
    for (int i = 1; i < nx - 1; i++) {
        rhs[i] = rhs[i] - c->am[0] * opt_d(uy, i + 1) - c->bm[0] * opt_d(uy, i) - c->bm[0] * opt_d(uy, i + 2);
        rhs[i + top] = rhs[i + top] - c->ap[ny - 1] * opt_d(uy, yb1 + i + 1) -
                       c->bp[ny - 1] * opt_d(uy, yb1 + i) - c->bp[ny - 1] * opt_d(uy, yb1 + i + 2);
    }
}
#undef E2

void ora_lu_2d(int nx, int ny, const ora_coef2d *c, cplx *L, cplx *U, cplx *Up) {
    /* LU.c:3-46; eigenvalue shift then Thomas factors per x-mode i, line-major [j + i*ny] */
    for (int i = 0; i < nx; i++) {
        const double ex = 2.0 * cos((i + 1) * M_PI / (nx + 1));
        const long   m  = (long)i * ny;
        L[m]  = 0.0;
        U[m]  = c->b[0] * ex + c->a[0];
        Up[m] = c->bp[0] * ex + c->ap[0];
        for (int j = 1; j < ny; j++) {
            cplx sub = c->bm[j] * ex + c->am[j];
            cplx dia = c->b[j] * ex + c->a[j];
            L[j + m]  = sub / U[j + m - 1];
            U[j + m]  = dia - L[j + m] * Up[j + m - 1];
            Up[j + m] = c->bp[j] * ex + c->ap[j];
        }
    }
}

int ora_solver_2d(int nx, int ny, const cplx *rhs, const cplx *L, const cplx *U, const cplx *Up,
                  cplx *sol) {
    const long nxy = (long)nx * ny;
    cplx *rhat = (cplx *)malloc(sizeof(cplx) * (size_t)nxy);
    cplx *xhat = (cplx *)malloc(sizeof(cplx) * (size_t)nxy);
    cplx *y    = (cplx *)malloc(sizeof(cplx) * (size_t)ny);
    cplx *rowt = (cplx *)malloc(sizeof(cplx) * (size_t)nx);
    if (!rhat || !xhat || !y || !rowt) return -1;
    /* forward DST along x of every row (DST.c:6-24) */
    if (ora_dst1_rows(nx, ny, rhs, nx, rhat, nx) != 0) return -1;
    /* per-mode Thomas along y (solver.c:71-86); xhat stored transposed [j + i*ny] */
    for (int i = 0; i < nx; i++) {
        const long m = (long)i * ny;
        y[0] = rhat[i];
        for (int j = 1; j < ny; j++) y[j] = rhat[i + (long)j * nx] - L[j + m] * y[j - 1];
        xhat[ny - 1 + m] = y[ny - 1] / U[ny - 1 + m];
        for (int j = ny - 2; j >= 0; j--) xhat[j + m] = (y[j] - Up[j + m] * xhat[j + 1 + m]) / U[j + m];
    }
    /* inverse DST: row j gathers xhat[j + i*ny] (DST.c:26-44) */
    for (int j = 0; j < ny; j++) {
        for (int i = 0; i < nx; i++) rowt[i] = xhat[j + (long)i * ny];
        if (ora_dst1_rows(nx, 1, rowt, nx, sol + (long)j * nx, nx) != 0) return -1;
    }
    free(rhat); free(xhat); free(y); free(rowt);
    return 0;
}

void ora_residual_2d(int nx, int ny, const ora_coef2d *c, const cplx *sol, const cplx *rhs, cplx *res) {
    /* residual.c:3-34 with a zero Dirichlet ring */
    const long w = nx + 2;
    cplx *se = (cplx *)calloc((size_t)(w * (ny + 2)), sizeof(cplx));
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) se[(i + 1) + (j + 1) * w] = sol[i + (long)j * nx];
    for (int j = 0; j < ny; j++) {
        cplx ap = c->ap[j], bp = c->bp[j], a = c->a[j], b = c->b[j], am = c->am[j], bm = c->bm[j];
        for (int i = 0; i < nx; i++) {
            long q = (i + 1) + (j + 1) * w;
            cplx top    = bp * se[q + w - 1] + ap * se[q + w] + bp * se[q + w + 1];
            cplx middle = b * se[q - 1] + a * se[q] + b * se[q + 1];
            cplx bottom = bm * se[q - w - 1] + am * se[q - w] + bm * se[q - w + 1];
            res[i + (long)j * nx] = top + middle + bottom - rhs[i + (long)j * nx];
        }
    }
    free(se);
}

/* ==================================================================== 3D ====== */

void ora_kz_3d(int nz, double hz, const cplx *k, const cplx *bc, cplx *kz) {
    double *Lf = (double *)malloc(sizeof(double) * (size_t)nz);
    double *Uf = (double *)malloc(sizeof(double) * (size_t)nz);
    for (int l = 0; l < nz; l++) kz[l] = 3.0 * (k[l + 2] - k[l]) / hz;
    kz[0] = kz[0] + opt_c(bc, 0);
    kz[nz - 1] = kz[nz - 1] + opt_c(bc, 1);
    pade_factors(nz, 4.0, Lf, Uf);
    pade_line(kz, 1, nz, Lf, Uf);
    free(Lf); free(Uf);
}

void ora_kzz_3d(int nz, double hz, const cplx *k, const cplx *bc, cplx *kzz) {
    double *Lf = (double *)malloc(sizeof(double) * (size_t)nz);
    double *Uf = (double *)malloc(sizeof(double) * (size_t)nz);
    for (int l = 0; l < nz; l++) kzz[l] = 12.0 * (k[l] - 2.0 * k[l + 1] + k[l + 2]) / hz / hz;
    kzz[0] = kzz[0] + opt_c(bc, 0);
    kzz[nz - 1] = kzz[nz - 1] + opt_c(bc, 1);
    pade_factors(nz, 10.0, Lf, Uf);
    pade_line(kzz, 1, nz, Lf, Uf);
    free(Lf); free(Uf);
}

void ora_coefficients_3d(const ora_problem3d *pb, ora_coef3d *c) {
    const int nz = pb->nz;
    const double hx = pb->hx, hy = pb->hy, hz = pb->hz;
    const cplx *k2 = pb->k2_ext;
    if (pb->order == 6) {
        /* coefficients.c:353-389 */
        cplx *kp  = (cplx *)malloc(sizeof(cplx) * (size_t)nz);
        cplx *kdp = (cplx *)malloc(sizeof(cplx) * (size_t)nz);
        ora_kz_3d(nz, hz, k2, pb->kz_bc, kp);
        ora_kzz_3d(nz, hz, k2, pb->kzz_bc, kdp);
        for (int i = 0; i < nz; i++) {
            c->a[i] = 1.0 / 10.0 + hz * hz * k2[i + 1] / 90.0;
            c->b[i] = 7.0 / 15.0 - hz * hz * k2[i + 1] / 90.0;
            c->c[i] = 7.0 / 15.0 - hz * hz * k2[i + 1] / 90.0;
            c->d[i] = -64.0 / 15.0 + 14.0 * hz * hz * k2[i + 1] / 15.0 -
                      hz * hz * hz * hz * k2[i + 1] * k2[i + 1] / 20.0 + hz * hz * hz * hz * kdp[i] / 20.0;
            c->ap[i] = 1.0 / 30.0;
            c->bp[i] = 1.0 / 10.0 + hz * hz * k2[i + 2] / 90.0 + (kp[i] * hz * hz * hz / 120.0);
            c->cp[i] = 1.0 / 10.0 + hz * hz * k2[i + 2] / 90.0 + (kp[i] * hz * hz * hz / 120.0);
            c->dp[i] = 7.0 / 15.0 - hz * hz * k2[i + 2] / 90.0 +
                       (kp[i] * hz * hz * hz / 20.0) * (1.0 / 3.0 + k2[i + 2] * hz * hz / 6.0);
            c->am[i] = 1.0 / 30.0;
            c->bm[i] = 1.0 / 10.0 + hz * hz * k2[i] / 90.0 - (kp[i] * hz * hz * hz / 120.0);
            c->cm[i] = 1.0 / 10.0 + hz * hz * k2[i] / 90.0 - (kp[i] * hz * hz * hz / 120.0);
            c->dm[i] = 7.0 / 15.0 - hz * hz * k2[i] / 90.0 -
                       (kp[i] * hz * hz * hz / 20.0) * (1.0 / 3.0 + k2[i] * hz * hz / 6.0);
        }
        free(kp); free(kdp);
    } else if (pb->order == 4) {
        /* coefficients.c:321-351 */
        const double Rzx = hz * hz / hx / hx, Rzy = hz * hz / hy / hy;
        const double one_sixth = 1.0 / 6.0, one_twelfth = 1.0 / 12.0;
        for (int i = 0; i < nz; i++) {
            c->a[i] = one_twelfth * (Rzx + Rzy);
            c->b[i] = one_sixth * (4.0 * Rzx - Rzy - 1.0 + 0.5 * hz * hz * k2[i + 1]);
            c->c[i] = one_sixth * (4.0 * Rzy - Rzx - 1.0 + 0.5 * hz * hz * k2[i + 1]);
            c->d[i] = -4.0 * (1.0 + Rzx + Rzy) / 3.0 + 0.5 * hz * hz * k2[i + 1];
            c->ap[i] = 0.0;
            c->bp[i] = one_twelfth * (1.0 + Rzx);
            c->cp[i] = one_twelfth * (1.0 + Rzy);
            c->dp[i] = 1.0 - one_sixth * (2.0 + Rzx + Rzy) + one_twelfth * hz * hz * k2[i + 2];
            c->am[i] = 0.0;
            c->bm[i] = one_twelfth * (1.0 + Rzx);
            c->cm[i] = one_twelfth * (1.0 + Rzy);
            c->dm[i] = 1.0 - one_sixth * (2.0 + Rzx + Rzy) + one_twelfth * hz * hz * k2[i];
        }
    } else {
        /* coefficients.c:293-319 */
        const double Rzx = hz * hz / hx / hx, Rzy = hz * hz / hy / hy;
        for (int i = 0; i < nz; i++) {
            c->a[i] = 0;
            c->b[i] = Rzx;
            c->c[i] = Rzy;
            c->d[i] = -2.0 * (Rzx + Rzy + 1.0) + hz * hz * k2[i + 1];
            c->ap[i] = 0; c->bp[i] = 0; c->cp[i] = 0; c->dp[i] = 1;
            c->am[i] = 0; c->bm[i] = 0; c->cm[i] = 0; c->dm[i] = 1;
        }
    }
}

/* index helpers on the extended 3D grid */
#define X3(ie, je, le) ((long)(ie) + (long)(je) * (long)(nx + 2) + (long)(le) * (long)(nx + 2) * (long)(ny + 2))

/* z-face Dirichlet terms shared by all orders (rhs.c:24-29, 55-62, 167-174) */
static void rhs3d_zfaces(int nx, int ny, int nz, int order, const ora_coef3d *c, const cplx *ue, cplx *rhsl) {
    if (!ue) return;
    const long nxy = (long)nx * ny;
    for (int i = 0; i < nx; i++) {
        for (int j = 0; j < ny; j++) {
            const long b = i + (long)j * nx, t = b + (long)(nz - 1) * nxy;
            if (order == 2) {
                rhsl[b] = rhsl[b] - ue[X3(i + 1, j + 1, 0)];
                rhsl[t] = rhsl[t] - ue[X3(i + 1, j + 1, nz + 1)];
            } else {
                rhsl[b] = rhsl[b] -
                          c->am[0] * (ue[X3(i, j, 0)] + ue[X3(i + 2, j, 0)] + ue[X3(i, j + 2, 0)] + ue[X3(i + 2, j + 2, 0)]) -
                          c->bm[0] * (ue[X3(i, j + 1, 0)] + ue[X3(i + 2, j + 1, 0)]) -
                          c->cm[0] * (ue[X3(i + 1, j, 0)] + ue[X3(i + 1, j + 2, 0)]) - c->dm[0] * ue[X3(i + 1, j + 1, 0)];
                const int L = nz + 1;
                rhsl[t] = rhsl[t] -
                          c->ap[nz - 1] * (ue[X3(i, j, L)] + ue[X3(i + 2, j, L)] + ue[X3(i, j + 2, L)] + ue[X3(i + 2, j + 2, L)]) -
                          c->bp[nz - 1] * (ue[X3(i, j + 1, L)] + ue[X3(i + 2, j + 1, L)]) -
                          c->cp[nz - 1] * (ue[X3(i + 1, j, L)] + ue[X3(i + 1, j + 2, L)]) -
                          c->dp[nz - 1] * ue[X3(i + 1, j + 1, L)];
            }
        }
    }
}

void ora_rhs_3d(const ora_problem3d *pb, const ora_coef3d *c, cplx *rhsl) {
    const int nx = pb->nx, ny = pb->ny, nz = pb->nz;
    const long nxy = (long)nx * ny, nxyz = nxy * nz;
    const long next = (long)(nx + 2) * (ny + 2) * (nz + 2);
    const double hx = pb->hx, hy = pb->hy, hz = pb->hz;
    const cplx *f = pb->rhs_ext;
    if (pb->order == 2) {
        for (int l = 0; l < nz; l++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) rhsl[i + j * (long)nx + l * nxy] = f[X3(i + 1, j + 1, l + 1)];
        rhs3d_zfaces(nx, ny, nz, 2, c, pb->ue_ext, rhsl);
        return;
    }
    if (pb->order == 4) {
        for (int l = 0; l < nz; l++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    long q = i + j * (long)nx + l * nxy;
                    rhsl[q] = f[X3(i + 1, j + 1, l + 1)];
                    rhsl[q] = rhsl[q] + (1.0 / 12.0) * (f[X3(i, j + 1, l + 1)] + f[X3(i + 2, j + 1, l + 1)] +
                                                        f[X3(i + 1, j, l + 1)] + f[X3(i + 1, j + 2, l + 1)] +
                                                        f[X3(i + 1, j + 1, l)] + f[X3(i + 1, j + 1, l + 2)] -
                                                        6 * f[X3(i + 1, j + 1, l + 1)]);
                }
        rhs3d_zfaces(nx, ny, nz, 4, c, pb->ue_ext, rhsl);
        return;
    }
    /* 6th order, rhs.c:67-194 */
    cplx *fxx = (cplx *)calloc((size_t)next, sizeof(cplx));
    cplx *fyy = (cplx *)calloc((size_t)next, sizeof(cplx));
    cplx *fzz = (cplx *)calloc((size_t)next, sizeof(cplx));
    cplx *tmp = (cplx *)malloc(sizeof(cplx) * (size_t)nxyz);
    int nmax = nx > ny ? nx : ny; if (nz > nmax) nmax = nz;
    double *Lf = (double *)malloc(sizeof(double) * (size_t)nmax);
    double *Uf = (double *)malloc(sizeof(double) * (size_t)nmax);
    const long fxb1 = (long)(ny + 2) * (nz + 2), fyb1 = (long)(nx + 2) * (nz + 2), fzb1 = (long)(nx + 2) * (ny + 2);

    /* f_xx along x (4th_order_partials.c:94-160); temp rows i-fastest */
    pade_factors(nx, 10.0, Lf, Uf);
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++) {
            cplx *row = tmp + (long)j * nx + l * nxy;
            for (int i = 0; i < nx; i++)
                row[i] = 12.0 * (f[X3(i, j + 1, l + 1)] - 2.0 * f[X3(i + 1, j + 1, l + 1)] + f[X3(i + 2, j + 1, l + 1)]) / hx / hx;
            row[0] = row[0] - opt_c(pb->fxx_b, (j + 1) + (long)(l + 1) * (ny + 2));
            row[nx - 1] = row[nx - 1] - opt_c(pb->fxx_b, (j + 1) + (long)(l + 1) * (ny + 2) + fxb1);
            pade_line(row, 1, nx, Lf, Uf);
        }
    for (int l = 0; l < nz + 2; l++)
        for (int j = 0; j < ny + 2; j++) {
            fxx[X3(0, j, l)] = opt_c(pb->fxx_b, j + (long)l * (ny + 2));
            fxx[X3(nx + 1, j, l)] = opt_c(pb->fxx_b, j + (long)l * (ny + 2) + fxb1);
        }
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) fxx[X3(i + 1, j + 1, l + 1)] = tmp[i + (long)j * nx + l * nxy];

    /* f_yy along y (4th_order_partials.c:162-227); temp [j + i*ny + l*nxy] */
    pade_factors(ny, 10.0, Lf, Uf);
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
                tmp[j + (long)i * ny + l * nxy] =
                    12.0 * (f[X3(i + 1, j, l + 1)] - 2.0 * f[X3(i + 1, j + 1, l + 1)] + f[X3(i + 1, j + 2, l + 1)]) / hy / hy;
    for (int l = 0; l < nz; l++)
        for (int i = 0; i < nx; i++) {
            cplx *line = tmp + (long)i * ny + l * nxy;
            line[0] = line[0] - opt_c(pb->fyy_b, (i + 1) + (long)(l + 1) * (nx + 2));
            line[ny - 1] = line[ny - 1] - opt_c(pb->fyy_b, (i + 1) + (long)(l + 1) * (nx + 2) + fyb1);
            pade_line(line, 1, ny, Lf, Uf);
        }
    for (int l = 0; l < nz + 2; l++)
        for (int i = 0; i < nx + 2; i++) {
            fyy[X3(i, 0, l)] = opt_c(pb->fyy_b, i + (long)l * (nx + 2));
            fyy[X3(i, ny + 1, l)] = opt_c(pb->fyy_b, i + (long)l * (nx + 2) + fyb1);
        }
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) fyy[X3(i + 1, j + 1, l + 1)] = tmp[(long)i * ny + j + l * nxy];

    /* f_zz along z (4th_order_partials.c:229-294); temp [l + i*nz + j*nx*nz] */
    const long nxz = (long)nx * nz;
    pade_factors(nz, 10.0, Lf, Uf);
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
                tmp[l + (long)i * nz + j * nxz] =
                    12.0 * (f[X3(i + 1, j + 1, l)] - 2.0 * f[X3(i + 1, j + 1, l + 1)] + f[X3(i + 1, j + 1, l + 2)]) / hz / hz;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            cplx *line = tmp + (long)i * nz + j * nxz;
            line[0] = line[0] - opt_c(pb->fzz_b, (i + 1) + (long)(j + 1) * (nx + 2));
            line[nz - 1] = line[nz - 1] - opt_c(pb->fzz_b, (i + 1) + (long)(j + 1) * (nx + 2) + fzb1);
            pade_line(line, 1, nz, Lf, Uf);
        }
    for (int j = 0; j < ny + 2; j++)
        for (int i = 0; i < nx + 2; i++) {
            fzz[X3(i, j, 0)] = opt_c(pb->fzz_b, i + (long)j * (nx + 2));
            fzz[X3(i, j, nz + 1)] = opt_c(pb->fzz_b, i + (long)j * (nx + 2) + fzb1);
        }
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) fzz[X3(i + 1, j + 1, l + 1)] = tmp[l + (long)i * nz + j * nxz];

    cplx *kp = (cplx *)malloc(sizeof(cplx) * (size_t)nz);
    ora_kz_3d(nz, hz, pb->k2_ext, pb->kz_bc, kp);

    /* combination, rhs.c:149-166 (2nd-order differences of 2nd_order_partials.c inline) */
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                long C = X3(i + 1, j + 1, l + 1);
                long W = X3(i, j + 1, l + 1), E = X3(i + 2, j + 1, l + 1);
                long S = X3(i + 1, j, l + 1), N = X3(i + 1, j + 2, l + 1);
                long D = X3(i + 1, j + 1, l), U = X3(i + 1, j + 1, l + 2);
                cplx fxxxx = (fxx[W] - 2.0 * fxx[C] + fxx[E]) / hx / hx;
                cplx fyyyy = (fyy[S] - 2.0 * fyy[C] + fyy[N]) / hy / hy;
                cplx fzzzz = (fzz[D] - 2.0 * fzz[C] + fzz[U]) / hz / hz;
                cplx fxxyy = (fxx[S] - 2.0 * fxx[C] + fxx[N]) / hy / hy;
                cplx fxxzz = (fxx[D] - 2.0 * fxx[C] + fxx[U]) / hz / hz;
                cplx fyyzz = (fyy[D] - 2.0 * fyy[C] + fyy[U]) / hz / hz;
                cplx first  = (1.0 - pb->k2_ext[l + 1] * hz * hz / 20.0) * f[C];
                cplx second = (hz * hz / 12.0) * (fxx[C] + fyy[C] + fzz[C]);
                cplx third  = (hz * hz * hz * hz / 360.0) * (fxxxx + fyyyy + fzzzz);
                cplx fourth = (hz * hz * hz * hz / 90.0) * (fxxyy + fxxzz + fyyzz);
                cplx fifth  = (hz * hz * hz / 120.0) * kp[l] * (f[U] - f[D]);
                if (g_real_sums_3d) {
                    first = creal(first); second = creal(second); third = creal(third);
                    fourth = creal(fourth); fifth = creal(fifth);
                }
                rhsl[i + j * (long)nx + l * nxy] = first + second + third + fourth + fifth;
            }
    rhs3d_zfaces(nx, ny, nz, 6, c, pb->ue_ext, rhsl);
    free(fxx); free(fyy); free(fzz); free(tmp); free(Lf); free(Uf); free(kp);
}
#undef X3

void ora_lu_3d(int nx, int ny, int nz, const ora_coef3d *c, cplx *L, cplx *U, cplx *Up) {
    /* LU.c:4-81; factors [l + i*nz + j*nx*nz], U stored as its reciprocal */
    const long nxz = (long)nx * nz;
    for (int j = 0; j < ny; j++) {
        const double ey = 2.0 * cos((j + 1) * M_PI / (ny + 1));
        for (int i = 0; i < nx; i++) {
            const double ex  = 2.0 * cos((i + 1) * M_PI / (nx + 1));
            const double exy = ex * ey;
            const long   m   = (long)i * nz + j * nxz;
            L[m]  = 0.0;
            U[m]  = 1.0 / (c->a[0] * exy + c->b[0] * ex + c->c[0] * ey + c->d[0]);
            Up[m] = c->ap[0] * exy + c->bp[0] * ex + c->cp[0] * ey + c->dp[0];
            for (int l = 1; l < nz; l++) {
                cplx e3  = c->a[l] * exy + c->b[l] * ex + c->c[l] * ey + c->d[l];
                cplx e3m = c->am[l] * exy + c->bm[l] * ex + c->cm[l] * ey + c->dm[l];
                L[l + m]  = e3m * U[l - 1 + m];
                U[l + m]  = 1.0 / (e3 - Up[l - 1 + m] * L[l + m]);
                Up[l + m] = c->ap[l] * exy + c->bp[l] * ex + c->cp[l] * ey + c->dp[l];
            }
        }
    }
}

int ora_solver_3d(int nx, int ny, int nz, const cplx *rhs, const cplx *L, const cplx *U, const cplx *Up,
                  cplx *sol) {
    const long nxy = (long)nx * ny, nxz = (long)nx * nz, nxyz = nxy * nz;
    cplx   *rhat = (cplx *)malloc(sizeof(cplx) * (size_t)nxyz);
    cplx   *xhat = (cplx *)malloc(sizeof(cplx) * (size_t)nxyz);
    cplx   *ya   = (cplx *)malloc(sizeof(cplx) * (size_t)nz);
    double *br = (double *)malloc(sizeof(double) * (size_t)nxy), *bi = (double *)malloc(sizeof(double) * (size_t)nxy);
    double *hr = (double *)malloc(sizeof(double) * (size_t)nxy), *hi = (double *)malloc(sizeof(double) * (size_t)nxy);
    if (!rhat || !xhat || !ya || !br || !bi || !hr || !hi) return -1;
    /* layer-wise 2D DST of the real and imaginary planes (solver.c:465-477) */
    for (int l = 0; l < nz; l++) {
        for (long t = 0; t < nxy; t++) { br[t] = creal(rhs[t + l * nxy]); bi[t] = cimag(rhs[t + l * nxy]); }
        ora_dst2_plane_real(nx, ny, br, hr);
        ora_dst2_plane_real(nx, ny, bi, hi);
        for (long t = 0; t < nxy; t++) rhat[t + l * nxy] = CMPLX(hr[t], hi[t]);
    }
    /* Thomas along z per (i,j) with reciprocal pivots (solver.c:483-496) */
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const long m = (long)i * nz + j * nxz, p = i + (long)j * nx;
            ya[0] = rhat[p];
            for (int l = 1; l < nz; l++) ya[l] = rhat[p + l * nxy] - L[l + m] * ya[l - 1];
            xhat[nz - 1 + m] = ya[nz - 1] * U[nz - 1 + m];
            for (int l = nz - 2; l >= 0; l--) xhat[l + m] = (ya[l] - Up[l + m] * xhat[l + 1 + m]) * U[l + m];
        }
    /* inverse, gathering layer l from the z-fastest xhat (solver.c:503-515) */
    for (int l = 0; l < nz; l++) {
        for (long t = 0; t < nxy; t++) { br[t] = creal(xhat[l + t * nz]); bi[t] = cimag(xhat[l + t * nz]); }
        ora_dst2_plane_real(nx, ny, br, hr);
        ora_dst2_plane_real(nx, ny, bi, hi);
        for (long t = 0; t < nxy; t++) sol[t + l * nxy] = CMPLX(hr[t], hi[t]);
    }
    free(rhat); free(xhat); free(ya); free(br); free(bi); free(hr); free(hi);
    return 0;
}

void ora_residual_3d(int nx, int ny, int nz, const ora_coef3d *c, const cplx *sol, const cplx *rhs, cplx *res) {
    /* residual.c:42-96 with a zero Dirichlet shell */
    const long sx = 1, sy = nx + 2, sz = (long)(nx + 2) * (ny + 2), nxy = (long)nx * ny;
    cplx *e = (cplx *)calloc((size_t)(sz * (nz + 2)), sizeof(cplx));
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) e[(i + 1) + (j + 1) * sy + (l + 1) * sz] = sol[i + j * (long)nx + l * nxy];
    for (int l = 0; l < nz; l++)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const long q = (i + 1) + (j + 1) * sy + (l + 1) * sz;
                const long t = q + sz, b = q - sz;
                cplx top = c->dp[l] * e[t] + c->ap[l] * (e[t + sx + sy] + e[t - sx + sy] + e[t + sx - sy] + e[t - sx - sy]) +
                           c->bp[l] * (e[t + sx] + e[t - sx]) + c->cp[l] * (e[t + sy] + e[t - sy]);
                cplx mid = c->d[l] * e[q] + c->a[l] * (e[q + sx + sy] + e[q - sx + sy] + e[q + sx - sy] + e[q - sx - sy]) +
                           c->b[l] * (e[q + sx] + e[q - sx]) + c->c[l] * (e[q + sy] + e[q - sy]);
                cplx bot = c->dm[l] * e[b] + c->am[l] * (e[b + sx + sy] + e[b - sx + sy] + e[b + sx - sy] + e[b - sx - sy]) +
                           c->bm[l] * (e[b + sx] + e[b - sx]) + c->cm[l] * (e[b + sy] + e[b - sy]);
                res[i + j * (long)nx + l * nxy] = (top + mid + bot);
            }
    for (long t = 0; t < nxy * nz; t++) res[t] = res[t] - rhs[t];
    free(e);
}

/* ============================================================ extended precision ====== */
/* The 2D solve with the per-mode Thomas factorisation and substitutions carried out in long
 * double (x87 80-bit) instead of double; the two DSTs stay in double (their rounding is at the
 * 1e-16 level and is not amplified).  It restates solver.c:71-86 and LU.c:12-40 in higher
 * precision so tests can measure how far the reference's own double result is from the exact
 * solution of its discrete system on ill-conditioned (near-resonant) lines. */
int ora_solver_2d_ld(int nx, int ny, const ora_coef2d *c, const cplx *rhs, cplx *sol) {
    typedef long double _Complex lcplx;
    const long nxy = (long)nx * ny;
    cplx  *rhat = (cplx *)malloc(sizeof(cplx) * (size_t)nxy);
    cplx  *xhat = (cplx *)malloc(sizeof(cplx) * (size_t)nxy);
    cplx  *rowt = (cplx *)malloc(sizeof(cplx) * (size_t)nx);
    lcplx *U = (lcplx *)malloc(sizeof(lcplx) * (size_t)ny);
    lcplx *y = (lcplx *)malloc(sizeof(lcplx) * (size_t)ny);
    if (!rhat || !xhat || !rowt || !U || !y) return -1;
    if (ora_dst1_rows(nx, ny, rhs, nx, rhat, nx) != 0) return -1;
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < nx; i++) {
        const long double ex = 2.0L * cosl((i + 1) * pi / (nx + 1));
        lcplx sup_prev = 0;
        for (int j = 0; j < ny; j++) {
            const lcplx sub = (lcplx)c->bm[j] * ex + (lcplx)c->am[j];
            const lcplx dia = (lcplx)c->b[j] * ex + (lcplx)c->a[j];
            if (j == 0) {
                U[0] = dia;
                y[0] = rhat[i];
            } else {
                const lcplx L = sub / U[j - 1];
                U[j] = dia - L * sup_prev;
                y[j] = (lcplx)rhat[i + (long)j * nx] - L * y[j - 1];
            }
            sup_prev = (lcplx)c->bp[j] * ex + (lcplx)c->ap[j];
        }
        lcplx x = y[ny - 1] / U[ny - 1];
        xhat[ny - 1 + (long)i * ny] = (cplx)x;
        for (int j = ny - 2; j >= 0; j--) {
            const lcplx sup = (lcplx)c->bp[j] * ex + (lcplx)c->ap[j];
            x = (y[j] - sup * x) / U[j];
            xhat[j + (long)i * ny] = (cplx)x;
        }
    }
    for (int j = 0; j < ny; j++) {
        for (int i = 0; i < nx; i++) rowt[i] = xhat[j + (long)i * ny];
        if (ora_dst1_rows(nx, 1, rowt, nx, sol + (long)j * nx, nx) != 0) return -1;
    }
    free(rhat); free(xhat); free(rowt); free(U); free(y);
    return 0;
}
