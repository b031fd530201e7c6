/*
 * Timing harness (TEST INFRASTRUCTURE ONLY): the reference 3D program's call sequence
 * (3D_Program/main_functions/main.c:4-31: defineSystem, background3D, coefficients, rhs, LU,
 * solver, residual) with solver() timed by wall clock HH_REPS times (default 5) instead of
 * once.  Linked against the reference's own GPU solver (target _ref/time3d_gpu) or the drop-in
 * libhh3d.so (target _ref/time3d_hh), so both solver() implementations are timed the same way
 * on the same problem: the reference's own 3D problem (3D_Program/user_input.c).
 * Usage: time3d_<x> order Nx Ny Nz
 */
#include "structs.h"
#include "prototypes.h"

int main(int argc, char **argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: %s order Nx Ny Nz  (HH_REPS solver calls, default 5)\n", argv[0]);
        return 2;
    }
    const char *e = getenv("HH_REPS");
    const int   reps = e ? atoi(e) : 5;
    System      sys = defineSystem(argc, argv);
    printf("grid %d x %d x %d, order %s\n", sys.lat.Nx, sys.lat.Ny, sys.lat.Nz, argv[1]);
    background3D(sys);
    coefficients(sys);
    rhs(sys);
    LU(sys);
    for (int r = 0; r < reps; r++) {
        Time t = tic();
        solver(sys);
        t = toc(t);
        printf("solver call %d: wall %.6f s\n", r, t.computed_t_n);
    }
    residual(sys);
    printf("||error||_inf = %.7e  ||res||_inf = %.7e\n", normInf(sys.lat.Nxyz, sys.error),
           normInf(sys.lat.Nxyz, sys.res));
    clearMemory(sys);
    return 0;
}
