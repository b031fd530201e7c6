/* The reference's 2D sources include <cufftw.h> unconditionally
 * (2D_Program/solver_functions/DST.c:3, solver.c:6); on the CPU oracle build it resolves
 * to the FFTW-API shim. Test infrastructure only. */
#include "fftw3.h"
