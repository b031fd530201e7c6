/*
 * Problem hook for building the reference's 2D sources into oracle/_ref/libref2d.so.
 * TEST INFRASTRUCTURE ONLY.
 *
 * The reference defines its test problem through callbacks in 2D_Program/user_input.c
 * (k, k2, k2_y, k2_yy, f, f_y, f_xx, f_yy, analytic_solution).  The configs need a
 * different problem class: constant k, homogeneous Dirichlet data, and a source f given
 * by its samples on the extended (N+2)^2 grid (sine modes plus optional noise).  These
 * callbacks therefore look the grid samples up by index; every boundary datum is zero.
 * Signatures follow 2D_Program/headers/prototypes.h:4-14.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static int     g_n;            /* interior points per direction              */
static double  g_x0, g_y0, g_h;
static double _Complex g_k;    /* constant wavenumber                        */
static double _Complex *g_f;   /* (n+2)^2 samples, x fastest                 */

void hhref2d_set_problem(int n, double x0, double y0, double h, double kre, double kim,
                         const double *f_ext_interleaved) {
    g_n = n; g_x0 = x0; g_y0 = y0; g_h = h;
    g_k = CMPLX(kre, kim);
    free(g_f);
    g_f = (double _Complex *)malloc(sizeof(double _Complex) * (size_t)(n + 2) * (size_t)(n + 2));
    memcpy(g_f, f_ext_interleaved, sizeof(double _Complex) * (size_t)(n + 2) * (size_t)(n + 2));
}

static long grid_index(double x, double y) {
    long i = lround((x - g_x0) / g_h), j = lround((y - g_y0) / g_h);
    if (i < 0 || j < 0 || i > g_n + 1 || j > g_n + 1) return -1;
    return i + j * (long)(g_n + 2);
}

double _Complex k(double y) { (void)y; return g_k; }
double _Complex k2(double y) { return k(y) * k(y); }
double _Complex k2_y(double y) { (void)y; return 0.0; }
double _Complex k2_yy(double y) { (void)y; return 0.0; }
double analytic_solution(double x, double y) { (void)x; (void)y; return 0.0; }
double _Complex f(double x, double y) {
    long q = grid_index(x, y);
    return (q < 0 || !g_f) ? 0.0 : g_f[q];
}
double _Complex f_y(double x, double y) { (void)x; (void)y; return 0.0; }
double _Complex f_xx(double x, double y) { (void)x; (void)y; return 0.0; }
double _Complex f_yy(double x, double y) { (void)x; (void)y; return 0.0; }
