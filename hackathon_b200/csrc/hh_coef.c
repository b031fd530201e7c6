/*
 * Stencil coefficients of the compact schemes for the constant-k problem class (host, O(n)).
 *
 * Restates the reference's coefficients() for a constant wavenumber on a uniform grid
 * (hx = hy [= hz] = h = 1/(n+1)):
 *   2D: 2D_Program/main_functions/coefficients.c:9-61 (k2_y = k2_yy = 0 for constant k)
 *   3D: 3D_Program/main_functions/coefficients.c:293-389 (k' = k'' = 0 for constant k)
 * The expressions keep the reference's operation order and C99 complex arithmetic so the
 * values are identical to what the reference computes for the same k.
 */
#include <complex.h>
#include <string.h>

#include "../../include/hh.h"

typedef double _Complex cplx;

static void put(double *dst, int j, cplx v) {
    dst[2 * j] = creal(v);
    dst[2 * j + 1] = cimag(v);
}

int hh_coefficients2d(int n, int order, double k_re, double k_im, double *const out[6]) {
    if (n < 1 || !out) return HH_ERR_INVALID;
    for (int t = 0; t < 6; t++)
        if (!out[t]) return HH_ERR_INVALID;
    const cplx   kk = CMPLX(k_re, k_im);
    const double h = 1.0 / (n + 1), hx = h, hy = h;
    double *bp = out[0], *ap = out[1], *b = out[2], *a = out[3], *bm = out[4], *am = out[5];
    for (int j = 0; j < n; j++) {
        if (order == 6) {
            const double hy2 = hy * hy, hy3 = hy2 * hy, hy4 = hy2 * hy2;
            const cplx   k2 = kk * kk, k2p = kk * kk, k2m = kk * kk, ky2 = 0.0, kyy = 0.0;
            put(ap, j, 2.0 / 3.0 + hy2 * k2p / 90.0 + hy3 * ky2 * (hy2 * k2p / 6.0 + 2.0 / 3.0) / 20.0);
            put(bp, j, 1.0 / 6.0 + hy2 * k2p / 90.0 + hy3 * ky2 / 120.0);
            put(a, j, -10.0 / 3.0 + 41.0 * hy2 * k2 / 45.0 - hy4 * k2 * k2 / 20.0 + hy4 * kyy / 20.0);
            put(b, j, 2.0 / 3.0 + hy2 * k2 / 90.0);
            put(am, j, 2.0 / 3.0 + hy2 * k2m / 90.0 - hy3 * ky2 * (hy2 * k2m / 6.0 + 2.0 / 3.0) / 20.0);
            put(bm, j, 1.0 / 6.0 + hy2 * k2m / 90.0 - hy3 * ky2 / 120.0);
        } else if (order == 4) {
            const double hy2 = hy * hy, Ryx = hy * hy / hx / hx;
            const cplx   k2 = kk * kk, k2p = kk * kk, k2m = kk * kk;
            put(bp, j, Ryx / 12.0 + 1.0 / 12.0);
            put(ap, j, 5.0 / 6.0 - Ryx / 6.0 + hy2 * k2p / 12.0);
            put(b, j, Ryx * (5.0 / 6.0) - 1.0 / 6.0 + hy2 * k2 / 12.0);
            put(a, j, -Ryx * (5.0 / 3.0) - 5.0 / 3.0 + 2.0 * hy2 * k2 / 3.0);
            put(bm, j, Ryx / 12.0 + 1.0 / 12.0);
            put(am, j, 5.0 / 6.0 - Ryx / 6.0 + hy2 * k2m / 12.0);
        } else if (order == 2) {
            const double hy2 = hy * hy, Ryx = hy * hy / hx / hx;
            put(bp, j, 0.0);
            put(ap, j, 1.0);
            put(b, j, Ryx);
            put(a, j, -2.0 * Ryx - 2.0 + kk * kk * hy2);
            put(bm, j, 0.0);
            put(am, j, 1.0);
        } else {
            return HH_ERR_INVALID;
        }
    }
    return HH_OK;
}

int hh_coefficients3d(int n, int order, double k_re, double k_im, double *const out[12]) {
    if (n < 1 || !out) return HH_ERR_INVALID;
    for (int t = 0; t < 12; t++)
        if (!out[t]) return HH_ERR_INVALID;
    const cplx   kk = CMPLX(k_re, k_im);
    const cplx   k2 = kk * kk; /* k2_bg_ext[l] for every layer */
    const double h = 1.0 / (n + 1), hx = h, hy = h, hz = h;
    double *a = out[0], *b = out[1], *c = out[2], *d = out[3], *ap = out[4], *bp = out[5], *cp = out[6],
           *dp = out[7], *am = out[8], *bm = out[9], *cm = out[10], *dm = out[11];
    for (int i = 0; i < n; i++) {
        if (order == 6) {
            const cplx kp = 0.0, kdp = 0.0; /* Pade d(k^2)/dz and d2(k^2)/dz2 of a constant */
            put(a, i, 1.0 / 10.0 + hz * hz * k2 / 90.0);
            put(b, i, 7.0 / 15.0 - hz * hz * k2 / 90.0);
            put(c, i, 7.0 / 15.0 - hz * hz * k2 / 90.0);
            put(d, i, -64.0 / 15.0 + 14.0 * hz * hz * k2 / 15.0 - hz * hz * hz * hz * k2 * k2 / 20.0 +
                          hz * hz * hz * hz * kdp / 20.0);
            put(ap, i, 1.0 / 30.0);
            put(bp, i, 1.0 / 10.0 + hz * hz * k2 / 90.0 + (kp * hz * hz * hz / 120.0));
            put(cp, i, 1.0 / 10.0 + hz * hz * k2 / 90.0 + (kp * hz * hz * hz / 120.0));
            put(dp, i, 7.0 / 15.0 - hz * hz * k2 / 90.0 + (kp * hz * hz * hz / 20.0) * (1.0 / 3.0 + k2 * hz * hz / 6.0));
            put(am, i, 1.0 / 30.0);
            put(bm, i, 1.0 / 10.0 + hz * hz * k2 / 90.0 - (kp * hz * hz * hz / 120.0));
            put(cm, i, 1.0 / 10.0 + hz * hz * k2 / 90.0 - (kp * hz * hz * hz / 120.0));
            put(dm, i, 7.0 / 15.0 - hz * hz * k2 / 90.0 - (kp * hz * hz * hz / 20.0) * (1.0 / 3.0 + k2 * hz * hz / 6.0));
        } else if (order == 4) {
            const double Rzx = hz * hz / hx / hx, Rzy = hz * hz / hy / hy;
            const double one_sixth = 1.0 / 6.0, one_twelfth = 1.0 / 12.0;
            put(a, i, one_twelfth * (Rzx + Rzy));
            put(b, i, one_sixth * (4.0 * Rzx - Rzy - 1.0 + 0.5 * hz * hz * k2));
            put(c, i, one_sixth * (4.0 * Rzy - Rzx - 1.0 + 0.5 * hz * hz * k2));
            put(d, i, -4.0 * (1.0 + Rzx + Rzy) / 3.0 + 0.5 * hz * hz * k2);
            put(ap, i, 0.0);
            put(bp, i, one_twelfth * (1.0 + Rzx));
            put(cp, i, one_twelfth * (1.0 + Rzy));
            put(dp, i, 1.0 - one_sixth * (2.0 + Rzx + Rzy) + one_twelfth * hz * hz * k2);
            put(am, i, 0.0);
            put(bm, i, one_twelfth * (1.0 + Rzx));
            put(cm, i, one_twelfth * (1.0 + Rzy));
            put(dm, i, 1.0 - one_sixth * (2.0 + Rzx + Rzy) + one_twelfth * hz * hz * k2);
        } else if (order == 2) {
            const double Rzx = hz * hz / hx / hx, Rzy = hz * hz / hy / hy;
            put(a, i, 0.0);
            put(b, i, Rzx);
            put(c, i, Rzy);
            put(d, i, -2.0 * (Rzx + Rzy + 1.0) + hz * hz * k2);
            put(ap, i, 0.0); put(bp, i, 0.0); put(cp, i, 0.0); put(dp, i, 1.0);
            put(am, i, 0.0); put(bm, i, 0.0); put(cm, i, 0.0); put(dm, i, 1.0);
        } else {
            return HH_ERR_INVALID;
        }
    }
    return HH_OK;
}
