/*
 * libhh2d.so -- the reference 2D program's solver entry points on the GPU
 * (2D_Program/solver_functions/solver.c:14, DST.c:6,26).  See include/hh_dropin2d.h.
 */
#include <complex.h>

#include "hh_dropin2d.h"
#include "hh_dropin_common.h"

int hh2d_status(void) { return g_status; }

static hh_plan *plan_for(const hh2d_System *s) {
    const int nx = s->lat.Nx, ny = s->lat.Ny;
    uint64_t  key = 1469598103934665603ULL;
    key = fnv1a(key, &nx, sizeof nx);
    key = fnv1a(key, &ny, sizeof ny);
    const double _Complex *rows[6] = {s->bp, s->ap, s->b, s->a, s->bm, s->am};
    for (int t = 0; t < 6; t++) key = fnv1a(key, rows[t], sizeof(double _Complex) * (size_t)ny);
    if (g_plan && key == g_key) return g_plan;
    hh_ctx *c = context();
    if (!c) return NULL;
    if (g_plan) { hh_plan_destroy(g_plan); g_plan = NULL; }
    if (report(hh_plan2d_create(c, nx, ny, (const double *)s->bp, (const double *)s->ap, (const double *)s->b,
                                (const double *)s->a, (const double *)s->bm, (const double *)s->am, &g_plan),
               "hh_plan2d_create") != HH_OK)
        return NULL;
    g_key = key;
    return g_plan;
}

void solver(hh2d_System sys) {
    hh_plan *p = plan_for(&sys);
    if (!p) return;
    report(hh_solve_host(p, (const double *)sys.rhs, (double *)sys.sol, 1), "solver");
}

void forwardDST(hh2d_System sys, hh2d_DSTN dst, double _Complex *rhs, double _Complex *rhat, void *plan, double *in,
                void *out, void *plan2, double *in2, void *out2) {
    (void)dst; (void)plan; (void)in; (void)out; (void)plan2; (void)in2; (void)out2;
    const int    nx = sys.lat.Nx, ny = sys.lat.Ny;
    const size_t bytes = sizeof(double _Complex) * (size_t)nx * (size_t)ny;
    void        *a, *b;
    if (report(device_staging(bytes, &a, &b), "forwardDST staging") != HH_OK) return;
    hh_ctx *c = g_ctx;
    int     rc = hh_memcpy_h2d(c, a, rhs, bytes);
    if (rc == HH_OK) rc = hh_dst1_rows(c, nx, ny, (const double *)a, nx, (double *)b, nx);
    if (rc == HH_OK) rc = hh_ctx_synchronize(c);
    if (rc == HH_OK) rc = hh_memcpy_d2h(c, rhat, b, bytes);
    report(rc, "forwardDST");
    hh_free(c, a);
    hh_free(c, b);
}

/* xhat arrives in the reference's transposed layout xhat[j + i*Ny] (solver.c:81-84) and sol
 * leaves x fastest (DST.c:35-40). */
void reverseDST(hh2d_System sys, hh2d_DSTN dst, double _Complex *xhat, double _Complex *sol, void *plan, double *in,
                void *out, void *plan2, double *in2, void *out2) {
    (void)dst; (void)plan; (void)in; (void)out; (void)plan2; (void)in2; (void)out2;
    const int    nx = sys.lat.Nx, ny = sys.lat.Ny;
    const size_t n = (size_t)nx * (size_t)ny, bytes = sizeof(double _Complex) * n;
    void        *a, *b;
    if (report(device_staging(bytes, &a, &b), "reverseDST staging") != HH_OK) return;
    hh_ctx          *c = g_ctx;
    double _Complex *tmp = (double _Complex *)malloc(bytes);
    int              rc = tmp ? HH_OK : HH_ERR_NOMEM;
    if (rc == HH_OK) rc = hh_memcpy_h2d(c, a, xhat, bytes);
    /* column j of the [i][j] array: element i at j + i*ny */
    if (rc == HH_OK) rc = hh_dst1_cols(c, nx, ny, 1, (const double *)a, ny, (long)n, (double *)b);
    if (rc == HH_OK) rc = hh_ctx_synchronize(c);
    if (rc == HH_OK) rc = hh_memcpy_d2h(c, tmp, b, bytes);
    if (rc == HH_OK)
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) sol[i + (size_t)j * nx] = tmp[j + (size_t)i * ny];
    report(rc, "reverseDST");
    free(tmp);
    hh_free(c, a);
    hh_free(c, b);
}
