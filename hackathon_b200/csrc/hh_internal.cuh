// Internal declarations shared by the sm_100a kernels and the C-ABI layer.
//
// Data layout: complex double stored as interleaved (re, im) double2, x fastest, exactly as
// the reference's `double _Complex` arrays (2D_Program/headers/structs.h:9,
// 3D_Program/headers/structs.h:36) so host buffers cross the boundary without repacking.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hh.h"

namespace hh {

// ------------------------------------------------------------------ errors ------
void set_error(const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define HH_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t hh_e_ = (call);                                                    \
        if (hh_e_ != cudaSuccess) return ::hh::cuda_fail(hh_e_, #call, __FILE__, __LINE__); \
    } while (0)

#define HH_TRY(call)                        \
    do {                                    \
        int hh_rc_ = (call);                \
        if (hh_rc_ != HH_OK) return hh_rc_; \
    } while (0)

// ------------------------------------------------------------ complex math ------
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// a - b*c
__host__ __device__ __forceinline__ double2 cfms(double2 a, double2 b, double2 c) {
    return make_double2(a.x - (b.x * c.x - b.y * c.y), a.y - (b.x * c.y + b.y * c.x));
}
// a + b*c
__host__ __device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
    return make_double2(a.x + (b.x * c.x - b.y * c.y), a.y + (b.x * c.y + b.y * c.x));
}
// 1/z by the textbook formula conj(z)/|z|^2 (inputs are O(1) Thomas pivots)
__host__ __device__ __forceinline__ double2 crcp(double2 z) {
    double d = 1.0 / (z.x * z.x + z.y * z.y);
    return make_double2(z.x * d, -z.y * d);
}
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) { return cmul(a, crcp(b)); }

// ---------------------------------------------------------------- context -------
struct Plan;

struct Ctx {
    int          device = 0;
    cudaStream_t stream = nullptr;
    bool         own_stream = false;
    // device twiddle tables keyed by transform length M (= n + 1):
    //   tw[M]  : exp(-2 pi i t / M), t = 0..M-1                 (double2)
    //   sn[M]  : sin(pi t / M),      t = 0..M-1                 (double)
    std::map<int, double2 *> tw;
    std::map<int, double *>  sn;
    std::map<int, double *>  dense; // n*n sine matrices for the direct DST (n+1 not a power of two)
    std::mutex               mu;
    std::vector<Plan *>      plans;
    long long                launches = 0;       // kernels launched through this context
    int                     *err_word = nullptr; // set by kernels whose bounded waits expire
    int                     *inject_word = nullptr; // armed by hh_ctx_inject_wait_expiry, taken by one launch
    size_t                   l2_bytes = 0;        // the device's L2 size (3D transform slabs)
    std::string              dev_name;            // the device's model name (tuning-cache key)
    // stage timing (hh_ctx_set_stage_timing)
    bool                     timing = false;
    std::vector<cudaEvent_t> ev_pending;          // groups of 4 events per timed solve
    double                   stage_ms[3] = {0, 0, 0};
    long long                timed_solves = 0;
    // host-buffer solves: copy streams and per-chunk events (created on first use)
    cudaStream_t             copy_in = nullptr, copy_out = nullptr;
    // plan memory pool (set by the request loop; null = cudaMalloc/cudaFree, synchronous set-up)
    cudaMemPool_t            pool = nullptr;
    std::vector<cudaEvent_t> chunk_ev;
    // residual maxima (max |res|, max |rhs| as double bit patterns) and the refined form's
    // workspace (one residual / correction field per right-hand side), made on first use
    unsigned long long      *norms = nullptr;
    double2                 *refine_work = nullptr;
    long                     refine_elems = 0;
    // the chunk table of multi-plan solves (hh_solve_source_multi), grown on demand
    void                    *multi_tab = nullptr;
    size_t                   multi_tab_bytes = 0;
    // the right-hand-side assembly's workspace (extended-grid derivative fields) and tables
    double2                 *rhs_work = nullptr;
    long                     rhs_elems = 0;
    void                    *rhs_tab = nullptr;
    size_t                   rhs_tab_bytes = 0;
};

int tables_for(Ctx *c, int m, const double2 **tw, const double **sn);
int dense_for(Ctx *c, int n, const double **mat);
// builds (once per context) the tables that DSTs of length n use
int prepare_dst(Ctx *c, int n);

// Plan: one (dim, sizes, stencil coefficients) problem with its device-resident setup.
struct Plan {
    Ctx   *ctx = nullptr;
    int    dim = 2;
    int    nx = 0, ny = 0, nz = 1;
    int    order = 6;
    // line-solve geometry: `lines` independent lines of `rows` points; element (row r, line q)
    // at offset r*row_stride + q inside one right-hand side.
    int    lines = 0, rows = 0;
    int    prow = 0;                // rows of the (zero-padded) per-row tables
    long   row_stride = 0;
    long   field = 0;               // complex elements per right-hand side
    // reciprocal Thomas pivot of the row before each 16-row segment, [segment][line]
    double2 *Pv = nullptr;
    bool     const_rows = false; // stencil row tables constant along the line
    int      variant = 0;        // line-solve kernel: 0/1 general (512x1, 256x2), 2..6 symmetric
    long     slab = 0;           // 3D: planes per slab of the transform passes (0: the whole batch)
    int      col_kernel = 0;     // 3D column DST: 0 CTA tiles of 8 swizzled columns, 1 per-warp tiles
    int      rows_kernel = 0;    // rows DST (n + 1 = 64 .. 1024): 0 default, 1 CTA ring, 2 per-warp buffers;
                                 // (n + 1 = 2048): 0, 1 two warps per line, 2 the Stockham kernel
    bool     sym = false;        // const_rows and sub == super on every line (constant k)
    bool     pf_ok = false;      // order-6 partial fractions well conditioned on every line
    double2 *subt = nullptr, *diagt = nullptr; // sub/diagonal row tables (4 * rows each)
    // super-diagonal(row, line) = rowc[0][row] mu[0][line] + rowc[1][row] mu[1][line] + rowc[2][row] mu[2][line] + rowc[3][row]
    double2 *rowc = nullptr;        // 4 * rows complex
    double  *mu = nullptr;          // 3 * lines real
    // fused source operator (homogeneous Dirichlet, constant k): 0 = off
    int      src_order = 0;
    double  *pade_l = nullptr, *pade_u = nullptr; // [1 10 1] factors along the line (rows each)
    double   pade_linf = 0.0, pade_uinf = 0.0;     // their common limit (reached from row 9 on)
    double   h = 0.0;
    double2  k2 = {0.0, 0.0};
    // 3D line-range plans (a rank's pencil of a slab/pencil solve): the plan holds lines
    // [line0, line0 + lines) of the nx * ny lines and only solves lines (hh_solve_lines)
    long     line0 = 0;
    bool     lines_only = false;
};

// lp: single-precision arithmetic (the refined solve's corrections) where the persistent-warp
// kernels serve (n + 1 = 64 .. 2048); FP64 otherwise
// rows_kernel (n + 1 = 64 .. 1024): 0 the length's default, 1 the CTA ring of line buffers, 2
// per-warp line buffers; (n + 1 = 2048): 0 and 1 two warps per line, 2 the Stockham kernel
int launch_dst_rows(Ctx *c, int n, long rows, const double2 *in, long in_ld, double2 *out, long out_ld,
                    bool lp = false, int rows_kernel = 0);
// The refined solve's correction: the single-precision rows transform of `in` subtracted from
// `out` (out <- out - DST(in)), for the lengths rows_update_supported admits (n + 1 = 64 .. 1024,
// and 2048 unless rows_kernel is 2); HH_ERR_UNSUPPORTED, before any launch, otherwise.
bool rows_update_supported(int n, int rows_kernel);
int  launch_dst_rows_update(Ctx *c, int n, long rows, const double2 *in, long in_ld, double2 *out, long out_ld,
                            int rows_kernel);
// kern: 0 = CTA tiles of 8 swizzled columns where the length allows, 1 = per-warp tiles of LPW columns
int launch_dst_cols(Ctx *c, int n, long ncols, long planes, const double2 *in, long ld, long plane_stride,
                    double2 *out, bool lp = false, int kern = 0);
int launch_factor(Plan *p, const double2 *subt, const double2 *diagt, const double2 *supt);
int launch_line_solve(Plan *p, const double2 *in, double2 *out, int batch, int src_order);
// slab [batch][planes][nlines] <-> the ranks' line parts of a slab/pencil solve (hh_lines_pack)
int launch_lines_pack(Ctx *c, const double2 *in, double2 *out, long batch, long planes, long nlines, int world,
                      bool unpack);
// one symmetric line-solve launch over several plans of one shape (plan i: nrhs[i] consecutive
// fields); table_dev holds line_solve_multi_table_bytes(nplans, total) bytes; HH_ERR_UNSUPPORTED
// (nothing launched) when the plans do not all take the same symmetric kernel variant
size_t line_solve_multi_table_bytes(int nplans, int total);
int launch_line_solve_multi(Plan *const *plans, const int *nrhs, int nplans, const double2 *in, double2 *out,
                            int src_order, void *table_dev);
// res = A_h u - rhs (FP64, zero Dirichlet ring); norms (optional, zeroed by the caller) receive
// max |res| and max |rhs| over the batch as double bit patterns
int launch_residual(Plan *p, const double2 *u, const double2 *rhs, double2 *res, int batch,
                    unsigned long long *norms);
int launch_axpy(Ctx *c, double2 *u, const double2 *v, double s, long n); // u += s v
int read_device_error(Ctx *c, int *val);
long slab_planes(const Plan &p, long planes); // 3D transform slab in planes (the plan's or the default)
// the fused-source solve of several plans of one shape in one pass (hh_solve_source_multi);
// table: device memory of line_solve_multi_table_bytes, or nullptr for the context's own
int solve_source_multi(Plan *const *plans, const int *nrhs, int nplans, const double2 *f, double2 *u, void *table);
// the reference's rhs() on the device for plans of any stencil (hh_rhs2d / hh_rhs3d)
int assemble_rhs2d(Plan *p, const hh_rhs2d_data *d, double2 *rhs);
int assemble_rhs3d(Plan *p, const hh_rhs3d_data *d, double2 *rhs);
int segment_count(int rows);
int sym_default_variant(int rows);
int padded_rows(int rows);
int solve_variant_count();


} // namespace hh
