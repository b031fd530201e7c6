/*
 * libhh2d.so -- the reference 2D program's solver entry points on the GPU
 * (2D_Program/solver_functions/solver.c:14, DST.c:6,26).  See include/hh_dropin2d.h.
 */
#include <complex.h>
#include <math.h>

#include "hh_dropin2d.h"
#include "hh_dropin_common.h"

int hh2d_status(void) { return g_status; }

static hh_plan *plan_for(const hh2d_System *s) {
    const int nx = s->lat.Nx, ny = s->lat.Ny;
    const size_t row = sizeof(double _Complex) * (size_t)ny;
    const void  *parts[8] = {&nx, &ny, s->bp, s->ap, s->b, s->a, s->bm, s->am};
    const size_t lens[8] = {sizeof nx, sizeof ny, row, row, row, row, row, row};
    if (key_matches(parts, lens, 8)) return g_plan;
    hh_ctx *c = context();
    if (!c) { key_forget(); return NULL; }
    if (g_plan) { hh_plan_destroy(g_plan); g_plan = NULL; }
    if (report(hh_plan2d_create(c, nx, ny, (const double *)s->bp, (const double *)s->ap, (const double *)s->b,
                                (const double *)s->a, (const double *)s->bm, (const double *)s->am, &g_plan),
               "hh_plan2d_create") != HH_OK) {
        key_forget();
        return NULL;
    }
    return g_plan;
}

void solver(hh2d_System sys) {
    hh_plan *p = plan_for(&sys);
    if (!p) return;
    report(hh_solve_host(p, (const double *)sys.rhs, (double *)sys.sol, 1), "solver");
}

/* The transform length is dst.Nx and the scale dst.coef, as in the reference (DST.c:15-21: the
 * first dst.Nx values of each of the sys.lat.Ny rows of stride sys.lat.Nx, times dst.coef).  The
 * device transform is orthonormal (sqrt(2/(dst.Nx+1))); any other dst.coef rescales on the host.
 * Values past dst.Nx in a row are left as they were. */
static int dst_length_ok(const hh2d_System *sys, const hh2d_DSTN *dst, const char *what) {
    if (dst->Nx < 1 || dst->Nx > sys->lat.Nx || sys->lat.Ny < 1) {
        fprintf(stderr, "ERROR: %s: dst.Nx = %d must be in 1..sys.lat.Nx = %d\n", what, dst->Nx, sys->lat.Nx);
        g_status = HH_ERR_INVALID;
        return 0;
    }
    return 1;
}

static double rescale_of(const hh2d_DSTN *dst) {
    const double ortho = sqrt(2.0 / (dst->Nx + 1));
    return dst->coef == ortho ? 1.0 : dst->coef / ortho;
}

void forwardDST(hh2d_System sys, hh2d_DSTN dst, double _Complex *rhs, double _Complex *rhat, void *plan, double *in,
                void *out, void *plan2, double *in2, void *out2) {
    (void)plan; (void)in; (void)out; (void)plan2; (void)in2; (void)out2;
    if (!dst_length_ok(&sys, &dst, "forwardDST")) return;
    const int    nx = sys.lat.Nx, ny = sys.lat.Ny, n = dst.Nx;
    const size_t bytes = sizeof(double _Complex) * (size_t)nx * (size_t)ny;
    void        *a, *b;
    if (report(device_staging(bytes, &a, &b), "forwardDST staging") != HH_OK) return;
    hh_ctx *c = g_ctx;
    int     rc = hh_memcpy_h2d(c, a, rhs, bytes);
    if (rc == HH_OK && n < nx) rc = hh_memcpy_h2d(c, b, rhat, bytes); /* the tails stay as they are */
    if (rc == HH_OK) rc = hh_dst1_rows(c, n, ny, (const double *)a, nx, (double *)b, nx);
    if (rc == HH_OK) rc = hh_ctx_synchronize(c);
    if (rc == HH_OK) rc = hh_memcpy_d2h(c, rhat, b, bytes);
    const double r = rescale_of(&dst);
    if (rc == HH_OK && r != 1.0)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < n; i++) rhat[i + (size_t)j * nx] *= r;
    report(rc, "forwardDST");
}

/* xhat arrives in the reference's transposed layout xhat[j + i*Ny] (solver.c:81-84) and sol
 * leaves x fastest (DST.c:35-40). */
void reverseDST(hh2d_System sys, hh2d_DSTN dst, double _Complex *xhat, double _Complex *sol, void *plan, double *in,
                void *out, void *plan2, double *in2, void *out2) {
    (void)plan; (void)in; (void)out; (void)plan2; (void)in2; (void)out2;
    if (!dst_length_ok(&sys, &dst, "reverseDST")) return;
    const int    nx = sys.lat.Nx, ny = sys.lat.Ny, n = dst.Nx;
    const size_t cnt = (size_t)nx * (size_t)ny, bytes = sizeof(double _Complex) * cnt;
    void        *a, *b;
    if (report(device_staging(bytes, &a, &b), "reverseDST staging") != HH_OK) return;
    hh_ctx          *c = g_ctx;
    double _Complex *tmp = (double _Complex *)host_staging(bytes);
    int              rc = tmp ? HH_OK : HH_ERR_NOMEM;
    if (rc == HH_OK) rc = hh_memcpy_h2d(c, a, xhat, bytes);
    /* column j of the [i][j] array: element i at j + i*ny, i < dst.Nx */
    if (rc == HH_OK) rc = hh_dst1_cols(c, n, ny, 1, (const double *)a, ny, (long)cnt, (double *)b);
    if (rc == HH_OK) rc = hh_ctx_synchronize(c);
    if (rc == HH_OK) rc = hh_memcpy_d2h(c, tmp, b, bytes);
    const double r = rescale_of(&dst);
    if (rc == HH_OK)
        for (int i = 0; i < n; i++)
            for (int j = 0; j < ny; j++) sol[i + (size_t)j * nx] = r == 1.0 ? tmp[j + (size_t)i * ny] : r * tmp[j + (size_t)i * ny];
    report(rc, "reverseDST");
}
