/*
 * hh.h -- C ABI of the B200 (sm_100a) compact Helmholtz direct solver.
 *
 * The solver follows gonzrona/hackathon: orthonormal DST-I in the constant-coefficient
 * direction(s), shifted tridiagonal line solves in the remaining direction, inverse DST-I
 * (2D_Program/solver_functions/solver.c:14-117, 3D_Program/solver_functions/solver.c:263-413).
 *
 * Conventions
 *  - Complex values are C99 `double _Complex` / interleaved (re, im) doubles; a `const double *`
 *    argument that carries complex data points at 2*count doubles.
 *  - Fields are x fastest: 2D index i + j*nx, 3D index i + j*nx + l*nx*ny (as the reference,
 *    2D_Program/headers/structs.h:9).  A batch of fields is contiguous, field after field.
 *  - Every function returns an int status (HH_OK = 0); hh_last_error() returns a message for the
 *    calling thread's most recent failure.  The reference's own entry points return void and
 *    print CUDA errors (solver_functions/cuda_helper.h:33-48); the drop-in libraries keep that
 *    signature (hh_dropin2d.h, hh_dropin3d.h) and report through hh_last_error().
 *  - "_dev" pointers are device memory on the context's device; "_host" pointers are host memory.
 *  - One context = one device + one CUDA stream; a context is used by one host thread at a
 *    time.  Separate contexts are independent.
 *  - Failures never fall back to a CPU path: if the CUDA module cannot run, calls fail.
 */
#ifndef HH_H
#define HH_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HH_OK              0
#define HH_ERR_INVALID     1  /* bad argument                                   */
#define HH_ERR_CUDA        2  /* CUDA runtime error                             */
#define HH_ERR_NOMEM       3  /* device allocation failed                       */
#define HH_ERR_UNSUPPORTED 4  /* size or option not implemented                 */
#define HH_ERR_DEVICE      5  /* a kernel reported a failure (bounded wait hit) */

typedef struct hh_ctx  hh_ctx;
typedef struct hh_plan hh_plan;

/* ---------------------------------------------------------------- library ---- */
const char *hh_last_error(void);
int         hh_version(void);                 /* major*10000 + minor*100 + patch */

/* --------------------------------------------------------------- contexts ---- */
/* stream: a cudaStream_t to launch on, or NULL for a context-owned stream. */
int hh_ctx_create(int device, void *stream, hh_ctx **out);
/* Destroys the context together with every plan still alive on it (those plan handles become
 * invalid).  To launch on the legacy default stream pass cudaStreamLegacy ((void *)1). */
int hh_ctx_destroy(hh_ctx *ctx);
int hh_ctx_set_stream(hh_ctx *ctx, void *stream);
int hh_ctx_synchronize(hh_ctx *ctx);          /* also surfaces kernel-reported failures   */
long long hh_ctx_launch_count(const hh_ctx *ctx); /* kernels launched through this context */
/* Failure injection on the device (no counterpart in the reference): the next rows transform
 * launched on the context with n + 1 in 64 .. 512 (the per-warp kernel of the 2D solves at those
 * sizes and of the 3D x-transforms) makes one of its copies' barriers wait for 16 bytes that never
 * arrive.  That bounded wait expires after a short budget, the kernel reports it, drains its own
 * copies and ends; its output is incomplete and the next hh_ctx_synchronize returns
 * HH_ERR_DEVICE (and clears it).  Nothing faults or hangs; the context stays usable. */
int hh_ctx_inject_wait_expiry(hh_ctx *ctx);

/* Stage timing: when enabled, every solve records CUDA events on the context's stream around
 * its three stages (forward transform, line solves, inverse transform) and accumulates the
 * elapsed device time.  hh_ctx_stage_times() synchronizes, then returns per-stage totals in
 * milliseconds and the number of solves timed, and resets them. */
#define HH_STAGE_FORWARD 0
#define HH_STAGE_LINES   1
#define HH_STAGE_INVERSE 2
#define HH_NUM_STAGES    3
int hh_ctx_set_stage_timing(hh_ctx *ctx, int on);
int hh_ctx_stage_times(hh_ctx *ctx, double ms[HH_NUM_STAGES], long long *solves);

/* device memory helpers for callers without their own CUDA bindings */
int hh_malloc(hh_ctx *ctx, size_t bytes, void **ptr_dev);
int hh_free(hh_ctx *ctx, void *ptr_dev);
int hh_memcpy_h2d(hh_ctx *ctx, void *dst_dev, const void *src_host, size_t bytes);
int hh_memcpy_d2h(hh_ctx *ctx, void *dst_host, const void *src_dev, size_t bytes);

/* ------------------------------------------------------------- transforms ---- */
/* Orthonormal DST-I of `rows` contiguous complex rows of length n (row r at offset r*ld).
 * Replaces forwardDST/reverseDST, 2D_Program/solver_functions/DST.c:6,26, which take the
 * same transform of every row through two zero-padded length-(2n+2) real FFTs. */
int hh_dst1_rows(hh_ctx *ctx, int n, long rows, const double *in_dev, long in_ld, double *out_dev, long out_ld);

/* DST-I along the strided direction: for each of `planes` planes (plane stride
 * plane_stride), transform each of `ncols` columns whose element j sits at col + j*ld. */
int hh_dst1_cols(hh_ctx *ctx, int n, long ncols, long planes, const double *in_dev, long ld, long plane_stride,
                 double *out_dev);

/* 2D DST-I (x then y) of nz planes of nx*ny complex values, in place or out of place.
 * Replaces DST(), 3D_Program/solver_functions/DST.c:148 (one real plane through two FFTW
 * batches and a transpose) and DST1/DST2 (DST.c:13,50). */
int hh_dst2_planes(hh_ctx *ctx, int nx, int ny, long nplanes, const double *in_dev, double *out_dev);
/* The exchange layout of a slab/pencil 3D solve (no counterpart in the reference): unpack = 0 cuts
 * a slab [batch][planes][nlines] into the parts of the world ranks' lines, out being
 * [planes][batch][cnt_0], [planes][batch][cnt_1], ... for the balanced contiguous split of the
 * lines (cnt_s = nlines / world + (s < nlines % world)); unpack = 1 is the inverse.  in and out
 * must not overlap; batch * planes <= 65535. */
int hh_lines_pack(hh_ctx *ctx, const double *in_dev, double *out_dev, long batch, long planes, long nlines, int world,
                  int unpack);

/* ------------------------------------------------------------------ plans ---- */
/* 2D plan from the reference's per-row 9-point stencil [bm am bm; b a b; bp ap bp]
 * (2D_Program/main_functions/coefficients.c:5-7), each array ny complex values on the host.
 * Builds the shifted Thomas factors on the device (replaces LU(), 2D_Program/main_functions/LU.c:3). */
int hh_plan2d_create(hh_ctx *ctx, int nx, int ny, const double *bp, const double *ap, const double *b,
                     const double *a, const double *bm, const double *am, hh_plan **out);

/* 3D plan from the reference's per-layer 27-point stencil a..dm (3D_Program/main_functions/
 * coefficients.c, order a,b,c,d,ap,bp,cp,dp,am,bm,cm,dm), each nz complex values on the host.
 * Replaces LU(), 3D_Program/main_functions/LU.c:4. */
int hh_plan3d_create(hh_ctx *ctx, int nx, int ny, int nz, const double *const coef[12], hh_plan **out);

/* Plans for the constant-k, unit-domain, homogeneous-Dirichlet problem class with the compact
 * right-hand-side operator fused into the line solve (order 2, 4 or 6).  The stencil follows
 * coefficients.c (2D :9-61, 3D :293-389) with k constant. */
int hh_plan2d_create_helmholtz(hh_ctx *ctx, int n, int order, double k_re, double k_im, hh_plan **out);
int hh_plan3d_create_helmholtz(hh_ctx *ctx, int n, int order, double k_re, double k_im, hh_plan **out);
/* One rank's part of a 3D solve split over ranks (no counterpart in the reference, whose solve
 * runs in one process; the slab/pencil decomposition is that of the paper the reference
 * accompanies): the z line solves of lines [q0, q1) of the n^2 lines, q = i + j n, laid out
 * [z][q - q0] per right-hand side (field size (q1 - q0) n).  Such a plan only solves lines
 * (hh_solve_lines); the other solve entry points, hh_residual, hh_rhs3d and hh_plan_tune refuse
 * it with HH_ERR_INVALID.  hackathon_b200/slab_pencil.py drives the whole decomposition. */
int hh_plan3d_create_helmholtz_lines(hh_ctx *ctx, int n, int order, double k_re, double k_im, long q0, long q1,
                                     hh_plan **out);

int hh_plan_destroy(hh_plan *plan);
long hh_plan_field_size(const hh_plan *plan);  /* complex values per right-hand side */

/* The line solve has several kernels: 0 and 1 for any stencil (512 threads x 1 block or 256 x 2
 * per SM); for constant-coefficient symmetric lines (the Helmholtz plans) also 2 (two blocks
 * per SM), 3 (one block, no register cap), 4 (two right-hand sides per pass), 5 (16-row
 * segments) and 6 (16-row segments, right-hand sides brought in as TMA tiles where a CTA holds
 * at least two lines, i.e. lines of up to 2048 rows).  hh_plan_tune
 * times each on `batch` right-hand sides and keeps the fastest (blocking; not during stream
 * capture); set/get select one directly.  A new symmetric plan starts at 2, or at 5 for lines
 * longer than 2048 rows. */
int hh_plan_tune(hh_plan *plan, int batch);
int hh_plan_set_variant(hh_plan *plan, int variant);
int hh_plan_variant(const hh_plan *plan);

/* Tuning cache (the reference launches fixed shapes: grid = (numSMs, numSMs), block = (16, 16),
 * 3D_Program/solver_functions/cuda_kernels.cu:336-346).  hh_plan_tune remembers what it measured
 * per device model and problem shape (dim, nx, ny, nz, fused source order, and which line-solve
 * kernels the stencil admits; not k, which does not change which kernel is fastest) and applies
 * a remembered entry instead of timing: a cache hit launches nothing (entries: line-solve variant,
 * column and rows transform kernels, 3D slab).  The cache is process-wide
 * and thread-safe.  hh_plan_apply_tuning applies an entry if one exists (*found = 1) and never
 * measures.  save/load keep the cache in a text file; load adds to what is cached. */
int hh_plan_apply_tuning(hh_plan *plan, int *found);
int hh_tune_cache_stats(long long *hits, long long *misses, long long *entries);
int hh_tune_cache_clear(void);
int hh_tune_cache_save(const char *path);
int hh_tune_cache_load(const char *path, long long *loaded);

/* 3D plans: the transform passes can run slab by slab (rows pass over a slab of planes, then the
 * columns pass over the same slab while the rows pass's output is still in L2).  `planes` per
 * slab; 0 (the default) makes the whole batch one slab.  hh_plan_tune also times a few slab
 * sizes for 3D plans and keeps the fastest.  The result does not depend on the slab. */
int  hh_plan_set_slab(hh_plan *plan, long planes);
long hh_plan_slab(const hh_plan *plan);
/* 3D plans: the kernel of the transform along y (columns): 0 (the default) brings 8 neighbouring
 * columns of all rows into a CTA as 128-byte-wide swizzled tensor boxes, 1 gives each warp its own
 * tiles of as many columns as it transforms at once (2 at n = 255).  Lengths n + 1 = 64 .. 512 have
 * both; other lengths use the second.  hh_plan_tune times both for 3D plans.  The result does
 * not depend on the variant. */
int  hh_plan_set_dst_variant(hh_plan *plan, int variant);
int  hh_plan_dst_variant(const hh_plan *plan);
/* The kernel of the transform along x (contiguous rows) for lengths n + 1 = 64 .. 1024: 1 a CTA
 * ring (the warps of a CTA share line buffers, the warp that frees one loads the CTA's line six
 * tickets ahead into it), 2 per-warp double buffers, 0 (the default) the length's own choice (the
 * ring at n + 1 = 1024).  The result does not depend on it.  At n + 1 = 2048: 0 and 1 two warps
 * per line (in a CTA ring), 2 the Stockham kernel of the longer lengths; the two agree to
 * rounding.  hh_plan_tune times both choices for every plan of these lengths. */
int  hh_plan_set_rows_variant(hh_plan *plan, int variant);
int  hh_plan_rows_variant(const hh_plan *plan);

/* Solve A u = rhs for `batch` assembled right-hand sides (the reference's solver(System),
 * 2D_Program/solver_functions/solver.c:14, 3D_Program/solver_functions/solver.c:263). */
int hh_solve(hh_plan *plan, const double *rhs_dev, double *sol_dev, int batch);
/* Same with host buffers: host-to-device copy, solve, device-to-host copy on the plan's stream. */
int hh_solve_host(hh_plan *plan, const double *rhs_host, double *sol_host, int batch);

/* Helmholtz plans only: u from the source samples f at the interior grid points (the
 * compact right-hand side is assembled on the device; replaces rhs(),
 * 2D_Program/main_functions/rhs.c:100, 3D_Program/main_functions/rhs.c:198, for this class). */
int hh_solve_source(hh_plan *plan, const double *f_dev, double *u_dev, int batch);
int hh_solve_source_host(hh_plan *plan, const double *f_host, double *u_host, int batch);
/* The line solve alone, on right-hand sides already transformed along the other axes (the
 * middle step of the reference's solver(): 2D_Program/solver_functions/solver.c:71-86,
 * 3D_Program/solver_functions/solver.c:483-496): fused = 0 for assembled right-hand sides (as in
 * hh_solve), 1 for transformed sources with the plan's compact operator (as in hh_solve_source,
 * Helmholtz plans).  Asynchronous on the plan's stream; in may equal out. */
int hh_solve_lines(hh_plan *plan, const double *in_dev, double *out_dev, int batch, int fused);
/* The same over another layout: element (row r, line q) of right-hand side b at
 * b field + r row_stride + q, the fields either one after another (field >= rows row_stride) or
 * interleaved row by row (row_stride >= batch field, e.g. a pencil [row][b][line]); lines are
 * contiguous.  Other layouts fail with HH_ERR_INVALID. */
int hh_solve_lines_strided(hh_plan *plan, const double *in_dev, double *out_dev, int batch, int fused,
                           long row_stride, long field);
/* Several wavenumbers in one solve (no counterpart in the reference, which solves one k per
 * run): nplans Helmholtz plans of one shape (dim, n, order) on one context, plan i taking the
 * nrhs[i] consecutive fields of f_dev and u_dev that follow those of plans 0..i-1.  The transforms
 * do not depend on k, so each direction is one launch over the whole batch; where every plan takes
 * the same symmetric line-solve variant (set by hh_plan_set_variant, or hh_plan_tune / the tuning
 * cache, which give plans of one shape the same one) the line solves are one launch as well, with
 * a table of which right-hand sides use which plan's factors; otherwise one line-solve launch per
 * plan.  Each field gets exactly the arithmetic of hh_solve_source on its own plan.  The table
 * lives in a context buffer grown on demand (allocation outside stream capture). */
int hh_solve_source_multi(hh_plan *const *plans, const int *nrhs, int nplans, const double *f_dev, double *u_dev);

/* The same host-buffer solve without any allocation (no counterpart in the reference).  For
 * callers that must not allocate device memory while they run, e.g. with a fixed memory budget
 * or where allocator latency is unwelcome: the device staging is a 32 MiB array of the library
 * (2^21 complex values, so field size * batch <= 2097152, e.g. two 1023^2 or one 127^3
 * right-hand sides; larger requests fail with HH_ERR_UNSUPPORTED).  hh_ctx_create looks up the
 * array's address on its device (this also loads the library's device code), so no call of this
 * function allocates, its first call on a new context included; a context must not outlive a
 * reset of its device.  The array is shared by all contexts on a device: calls that overlap in
 * time race and must be serialized by the caller. */
int hh_solve_source_host_noalloc(hh_plan *plan, const double *f_host, double *u_host, int batch);

/* FP64 residual res = A_h sol - rhs of the plan's compact operator for `batch` fields on the
 * device, with a zero Dirichlet ring (the reference's residual(), 2D_Program/main_functions/
 * residual.c:3-34, 3D_Program/main_functions/residual.c:42-96; its error-vs-analytic part is the
 * caller's).  res must not be the sol buffer.  If max_res or max_rhs is not NULL the call waits
 * and returns max |res| and max |rhs| over the batch (complex modulus). */
int hh_residual(hh_plan *plan, const double *sol_dev, const double *rhs_dev, double *res_dev, int batch,
                double *max_res, double *max_rhs);

/* The reference's right-hand-side assembly rhs() on the device, for plans of any stencil (the
 * reference's own variable-k problems and Dirichlet data): 2D_Program/main_functions/rhs.c:4-150
 * and 3D_Program/main_functions/rhs.c:13-194, with the compact [1 10 1] / [1 4 1] Pade derivatives
 * of the partial_derivatives/ files solved along each axis on the device.  The data the reference
 * evaluates through its user callbacks comes as sampled arrays, x fastest, complex unless noted;
 * a NULL boundary array means identically zero.  rhs_dev receives nx*ny (nx*ny*nz) values, the
 * input of hh_solve on the same plan.  The plan's stencil rows give the Dirichlet corrections.
 * Arithmetic follows the reference's expression order (complex throughout; the reference's 3D
 * rhs.c:149 keeps its partial sums in real doubles, which agrees for real data). */
typedef struct {
    int           order;        /* 2, 4 or 6                                                    */
    double        hx, hy;       /* grid spacings                                                */
    const double *f_ext;        /* device: f on the extended grid, (nx+2)(ny+2)                 */
    const double *k_ext;        /* host: k at y0 + j hy, j = 0..ny+1 (order 6)                  */
    const double *k2y_bc;       /* host: d(k^2)/dy at y0 and at y1, 2 values                    */
    const double *fxx_xb;       /* device: f_xx on x = x0 (j = 0..ny+1), then on x = x1          */
    const double *fxx_yb;       /* device: f_xx on y = y0 (i = 0..nx+1), then on y = y1          */
    const double *fyy_xb;       /* device: f_yy on x = x0, then x = x1: 2 (ny+2)                */
    const double *fyy_yb;       /* device: f_yy on y = y0, then y = y1: 2 (nx+2)                */
    const double *fy_yb;        /* device: f_y on y = y0 at interior x (nx), then on y = y1     */
    const double *u_xb, *u_yb;  /* device, real: Dirichlet data on x = x0, x1: 2 (ny+2); on
                                   y = y0, y1: 2 (nx+2)                                          */
} hh_rhs2d_data;
int hh_rhs2d(hh_plan *plan, const hh_rhs2d_data *data, double *rhs_dev);

typedef struct {
    int           order;        /* 2, 4 or 6                                                    */
    double        hx, hy, hz;   /* grid spacings                                                */
    const double *f_ext;        /* device: the source on the extended grid scaled by hz^2 (the
                                   reference's rhs_ext), (nx+2)(ny+2)(nz+2)                      */
    const double *k2_ext;       /* host: k^2 at z0 + l hz, l = 0..nz+1 (order 6)                */
    const double *kz_bc;        /* host: the boundary terms of d(k^2)/dz at z0 and z1, 2 values */
    const double *fxx_b;        /* device: f_xx on x = x0 (j + l (ny+2)), then on x = x1        */
    const double *fyy_b;        /* device: f_yy on y = y0 (i + l (nx+2)), then on y = y1        */
    const double *fzz_b;        /* device: f_zz on z = z0 (i + j (nx+2)), then on z = z1        */
    const double *ue_ext;       /* device: Dirichlet data on the extended grid (its z faces)    */
} hh_rhs3d_data;
int hh_rhs3d(hh_plan *plan, const hh_rhs3d_data *data, double *rhs_dev);

/* Mixed-precision refined solve of `batch` assembled right-hand sides on the device (an
 * addition: the reference solves in plain FP64 only): every solve in
 * the loop runs its DSTs in single-precision arithmetic (where n + 1 is a power of two up to
 * 1024; FP64 otherwise) and its line solves in FP64, and hh_residual's FP64 residual drives
 * the corrections:  u_0 = S(rhs),  u_{k+1} = u_k - S(A_h u_k - rhs)  until
 * max|A_h u - rhs| / max|rhs| <= tol or max_iter corrections.  *iters and *rel_res (optional)
 * receive the corrections made and the final relative residual; a result above tol is not an
 * error.  Uses a context workspace of batch fields (allocated on first use, grown as needed).
 * Blocking.  rhs and sol must be different buffers. */
int hh_solve_refined(hh_plan *plan, const double *rhs_dev, double *sol_dev, int batch, double tol, int max_iter,
                     int *iters, double *rel_res);

/* Stencil coefficients the Helmholtz plans use (host arrays of n complex values each):
 * 2D order in bp,ap,b,a,bm,am order; 3D in a..dm order (12 arrays). */
int hh_coefficients2d(int n, int order, double k_re, double k_im, double *const out[6]);
int hh_coefficients3d(int n, int order, double k_re, double k_im, double *const out[12]);

/* ---------------------------------------------------------------- serving ---- */
/* A request loop over one device (no counterpart in the reference, whose Direct_Solver solves
 * one problem per process).  hh_server_submit queues a request and returns at once; a
 * dispatcher thread solves it asynchronously:
 *  - one plan per (dim, n, order, k) stays resident (least recently used plans are evicted
 *    when the HBM budget needs the room); new plans take the tuning cache's settings for their
 *    shape (hh_plan_apply_tuning), so tune one plan per served shape beforehand;
 *  - continuous batching: queued requests of the same shape (dim, n, order) at any k (up to 64
 *    right-hand sides, each request at most 4M points) run as one batched solve over their plans
 *    (hh_solve_source_multi);
 *  - admission: a batch starts while plans plus in-flight staging fit the HBM budget, otherwise
 *    it waits for running batches; a request that can never fit fails with HH_ERR_NOMEM;
 *  - batches go round-robin to `streams` CUDA streams, so requests overlap on the device;
 *  - memory: the server's stream-ordered pool reserves min(budget, 64 GB) of device memory when
 *    the server is created and keeps it until hh_server_destroy (a fresh pool growing under load
 *    stalls the dispatcher).
 * Each result is bitwise the result of hh_solve_source on a plan of the same problem.  Host
 * buffers should be pinned for copies to overlap; device buffers (on_device = 1) are used
 * directly when a request runs alone.  Buffers must stay valid until hh_server_wait returns. */
typedef struct hh_server hh_server;
typedef struct {
    int           dim, n, order; /* 2 or 3; interior points per direction; 2, 4 or 6 */
    double        k_re, k_im;    /* constant wavenumber                               */
    int           nrhs;          /* right-hand sides (1..65535)                       */
    int           on_device;     /* 0: f and u are host memory, 1: device memory      */
    const double *f;             /* nrhs * n^dim complex source samples (interior)    */
    double       *u;             /* nrhs * n^dim complex solution                     */
} hh_request;
typedef struct {
    int    status;                  /* HH_OK or the failure code                      */
    double t_submit, t_start, t_done; /* seconds on hh_server_clock                   */
    int    batch_rhs;               /* right-hand sides of the batch it ran in        */
} hh_request_info;
int    hh_server_create(int device, size_t hbm_budget_bytes, int streams, hh_server **out);
int    hh_server_submit(hh_server *s, const hh_request *r, long long *id);
int    hh_server_wait(hh_server *s, long long id, hh_request_info *info); /* blocks; frees the id */
int    hh_server_stats(hh_server *s, long long *completed, size_t *bytes_in_use, int *plans);
double hh_server_clock(hh_server *s);
int    hh_server_destroy(hh_server *s); /* finishes every submitted request first */
/* Host-side failure injection (no counterpart in the reference, which only prints CUDA errors,
 * 3D_Program/solver_functions/cuda_helper.h:33-48): the next `batches` batches the loop starts
 * run their solves unchanged but complete with HH_ERR_DEVICE, exactly as if one of their kernels
 * had reported an expired bounded wait.  Each stream has its own device error word, cleared
 * before every batch, so a failure is charged to its own batch only and later batches succeed. */
int    hh_server_inject_error(hh_server *s, int batches);
/* The device form: arms hh_ctx_inject_wait_expiry on the loop's context, so that the next batch
 * that runs such a rows transform fails with HH_ERR_DEVICE through its own stream's error word. */
int    hh_server_inject_wait_expiry(hh_server *s);

#ifdef __cplusplus
}
#endif

#endif /* HH_H */
