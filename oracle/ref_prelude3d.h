/*
 * Forced include for the reference's 3D sources in oracle/_ref/ (TEST INFRASTRUCTURE).
 * 3D_Program/partial_derivatives/4th_order_partials.c:144 writes the x = x1 ghost column of
 * f_xx at a wrong index, and rhs.c never sets the y/z ghost faces of f_xx or the z faces of
 * f_yy, yet 2nd_order_partials.c reads them.  The reference therefore relies on freshly
 * mapped (zeroed) heap memory.  Routing its malloc to calloc makes that assumption hold
 * for every problem size instead of only for allocations above the mmap threshold.
 */
#include <stdlib.h>
static inline void *hh_ref_zeroed_malloc(size_t n) { return calloc(1, n); }
#define malloc(n) hh_ref_zeroed_malloc(n)
