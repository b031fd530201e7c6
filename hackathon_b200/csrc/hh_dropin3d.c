/*
 * libhh3d.so -- the reference 3D program's solver entry points on the GPU
 * (3D_Program/solver_functions/solver.c:263, DST.c:148).  See include/hh_dropin3d.h.
 */
#include <complex.h>

#include "hh_dropin3d.h"
#include "hh_dropin_common.h"

int hh3d_status(void) { return g_status; }

static hh_plan *plan_for(const hh3d_System *s) {
    const int nx = s->lat.Nx, ny = s->lat.Ny, nz = s->lat.Nz;
    const double _Complex *layers[12] = {s->a, s->b, s->c, s->d, s->ap, s->bp, s->cp, s->dp,
                                         s->am, s->bm, s->cm, s->dm};
    const void  *parts[15] = {&nx, &ny, &nz};
    size_t       lens[15] = {sizeof nx, sizeof ny, sizeof nz};
    for (int t = 0; t < 12; t++) {
        parts[3 + t] = layers[t];
        lens[3 + t] = sizeof(double _Complex) * (size_t)nz;
    }
    if (key_matches(parts, lens, 15)) return g_plan;
    hh_ctx *c = context();
    if (!c) { key_forget(); return NULL; }
    if (g_plan) { hh_plan_destroy(g_plan); g_plan = NULL; }
    const double *coef[12];
    for (int t = 0; t < 12; t++) coef[t] = (const double *)layers[t];
    if (report(hh_plan3d_create(c, nx, ny, nz, coef, &g_plan), "hh_plan3d_create") != HH_OK) {
        key_forget();
        return NULL;
    }
    return g_plan;
}

void solver(hh3d_System sys) {
    hh_plan *p = plan_for(&sys);
    if (!p) return;
    report(hh_solve_host(p, (const double *)sys.rhs, (double *)sys.sol, 1), "solver");
}

void DST(int Nx, int Ny, double *b_2D, double *bhat, void *p1, double *in1, void *out1, void *p2, double *in2,
         void *out2) {
    (void)p1; (void)in1; (void)out1; (void)p2; (void)in2; (void)out2;
    if (Nx < 1 || Ny < 1) {
        fprintf(stderr, "ERROR: DST: plane %d x %d\n", Nx, Ny);
        g_status = HH_ERR_INVALID;
        return;
    }
    const size_t n = (size_t)Nx * (size_t)Ny, bytes = sizeof(double _Complex) * n;
    void        *a, *b;
    if (report(device_staging(bytes, &a, &b), "DST staging") != HH_OK) return;
    hh_ctx          *c = g_ctx;
    double _Complex *tmp = (double _Complex *)host_staging(bytes);
    int              rc = tmp ? HH_OK : HH_ERR_NOMEM;
    if (rc == HH_OK) {
        for (size_t t = 0; t < n; t++) tmp[t] = b_2D[t]; /* real plane as complex */
        rc = hh_memcpy_h2d(c, a, tmp, bytes);
    }
    if (rc == HH_OK) rc = hh_dst2_planes(c, Nx, Ny, 1, (const double *)a, (double *)b);
    if (rc == HH_OK) rc = hh_ctx_synchronize(c);
    if (rc == HH_OK) rc = hh_memcpy_d2h(c, tmp, b, bytes);
    if (rc == HH_OK)
        for (size_t t = 0; t < n; t++) bhat[t] = creal(tmp[t]);
    report(rc, "DST");
}
