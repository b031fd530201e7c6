// C ABI (include/hh.h): contexts, plans and the solve pipeline on sm_100a.
//
// Pipeline for one batch of right-hand sides (all on the plan's stream, no host round trip):
//   2D  rhs --DST-I along x (rows)--> F^ --line solves along y--> U^ --DST-I along x--> u
//   3D  rhs --DST-I x (rows), y (columns)--> F^ --line solves along z--> U^ --DST-I y, x--> u
// which is the reference's solver() (2D_Program/solver_functions/solver.c:66-90,
// 3D_Program/solver_functions/solver.c:465-515).  Every stage works in place on the output
// buffer, so the solve needs no scratch beyond the output itself.
#include "hh_internal.cuh"

#include <algorithm>
#include <cmath>

#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <string>

// Device staging for hh_solve_source_host_noalloc: one file-scope array per device, 32 MiB
// (2^21 complex values: e.g. two 1023^2 right-hand sides or one 127^3).  Nothing in it has to
// start at zero: every call writes each element it reads.  Calls that overlap in time on one
// device share it and race; they must be serialized.
constexpr long kNoAllocElems = 1L << 21;
static __device__ __align__(256) double2 g_noalloc_stage[kNoAllocElems];

struct hh_ctx {
    hh::Ctx c;
    // device address of g_noalloc_stage on the context's device, looked up when the context is
    // created (that lookup also loads this file's device code, so a later call allocates nothing)
    double2 *noalloc_stage = nullptr;
    // device staging for hh_solve_host / hh_solve_source_host, shared by the context's plans
    // (host-buffer solves are synchronous, so one call uses it at a time)
    double2 *stage = nullptr;
    long     stage_elems = 0;
};
struct hh_plan {
    hh::Plan p;
};

namespace hh {

static thread_local std::string g_err;

void set_error(const char *fmt, ...) {
    char    buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    set_error("%s failed: %s (%d) at %s:%d", what, cudaGetErrorString(e), (int)e, file, line);
    return e == cudaErrorMemoryAllocation ? HH_ERR_NOMEM : HH_ERR_CUDA;
}

static int upload(Ctx *c, void *dst, const void *src, size_t bytes) {
    HH_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    return HH_OK;
}

// Plan memory: from the context's pool in stream order when it has one (the request loop's
// contexts: no device-wide synchronization on allocation or release), else cudaMalloc/cudaFree.
static int dalloc(Ctx *c, void **p, size_t bytes) {
    if (c->pool) HH_CUDA(cudaMallocFromPoolAsync(p, bytes, c->pool, c->stream));
    else HH_CUDA(cudaMalloc(p, bytes));
    return HH_OK;
}
static void dfree(Ctx *c, void *p) {
    if (!p) return;
    if (c->pool) cudaFreeAsync(p, c->stream);
    else cudaFree(p);
}

} // namespace hh

using namespace hh;

static void drain_events(Ctx &c);
static int stage_mark(Ctx &c, int k);

// ------------------------------------------------------------------ library ------
extern "C" const char *hh_last_error(void) { return g_err.c_str(); }
extern "C" int hh_version(void) { return 100; }

// ----------------------------------------------------------------- contexts ------
extern "C" int hh_ctx_create(int device, void *stream, hh_ctx **out) {
    if (!out) { set_error("hh_ctx_create: null out"); return HH_ERR_INVALID; }
    *out = nullptr;
    int ndev = 0;
    HH_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) { set_error("hh_ctx_create: device %d of %d", device, ndev); return HH_ERR_INVALID; }
    HH_CUDA(cudaSetDevice(device));
    int l2 = 0;
    HH_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device));
    cudaDeviceProp prop;
    HH_CUDA(cudaGetDeviceProperties(&prop, device)); // once per context: the query is slow
    hh_ctx *x = new hh_ctx();
    x->c.device = device;
    x->c.l2_bytes = l2 > 0 ? (size_t)l2 : (size_t)(50u << 20);
    x->c.dev_name = prop.name;
    if (stream) {
        x->c.stream = (cudaStream_t)stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&x->c.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete x; return cuda_fail(e, "cudaStreamCreateWithFlags", __FILE__, __LINE__); }
        x->c.own_stream = true;
    }
    cudaError_t e = cudaMalloc(&x->c.err_word, 2 * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(x->c.err_word, 0, 2 * sizeof(int));
    if (e == cudaSuccess) x->c.inject_word = x->c.err_word + 1;
    if (e == cudaSuccess) e = cudaGetSymbolAddress((void **)&x->noalloc_stage, g_noalloc_stage);
    if (e != cudaSuccess) {
        if (x->c.own_stream) cudaStreamDestroy(x->c.stream);
        delete x;
        return cuda_fail(e, "error word", __FILE__, __LINE__);
    }
    *out = x;
    return HH_OK;
}

static void plan_free(hh_plan *pl);

extern "C" int hh_ctx_destroy(hh_ctx *x) {
    if (!x) return HH_OK;
    cudaSetDevice(x->c.device);
    cudaStreamSynchronize(x->c.stream);
    drain_events(x->c);
    // plans still alive belong to this context: release them with it
    for (Plan *p : x->c.plans) {
        hh_plan *pl = reinterpret_cast<hh_plan *>(p); // Plan is the first member of hh_plan
        plan_free(pl);
        delete pl;
    }
    x->c.plans.clear();
    for (auto &kv : x->c.tw) cudaFree(kv.second);
    for (auto &kv : x->c.sn) cudaFree(kv.second);
    for (auto &kv : x->c.dense) cudaFree(kv.second);
    cudaFree(x->c.err_word);
    cudaFree(x->c.norms);
    cudaFree(x->c.refine_work);
    cudaFree(x->c.multi_tab);
    cudaFree(x->c.rhs_work);
    cudaFree(x->c.rhs_tab);
    cudaFree(x->stage);
    for (cudaEvent_t e : x->c.chunk_ev) cudaEventDestroy(e);
    if (x->c.copy_in) cudaStreamDestroy(x->c.copy_in);
    if (x->c.copy_out) cudaStreamDestroy(x->c.copy_out);
    if (x->c.own_stream) cudaStreamDestroy(x->c.stream);
    delete x;
    return HH_OK;
}

extern "C" int hh_ctx_set_stream(hh_ctx *x, void *stream) {
    if (!x) return HH_ERR_INVALID;
    if (x->c.own_stream) { cudaStreamDestroy(x->c.stream); x->c.own_stream = false; }
    x->c.stream = (cudaStream_t)stream;
    return HH_OK;
}

extern "C" int hh_ctx_synchronize(hh_ctx *x) {
    if (!x) return HH_ERR_INVALID;
    HH_CUDA(cudaSetDevice(x->c.device));
    HH_CUDA(cudaStreamSynchronize(x->c.stream));
    int flag = 0;
    HH_CUDA(cudaMemcpy(&flag, x->c.err_word, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        HH_CUDA(cudaMemset(x->c.err_word, 0, sizeof(int)));
        set_error("a kernel reported an expired bounded wait (code %d)", flag);
        return HH_ERR_DEVICE;
    }
    return HH_OK;
}

extern "C" long long hh_ctx_launch_count(const hh_ctx *x) { return x ? x->c.launches : 0; }

extern "C" int hh_ctx_inject_wait_expiry(hh_ctx *x) {
    if (!x) { set_error("hh_ctx_inject_wait_expiry: null context"); return HH_ERR_INVALID; }
    HH_CUDA(cudaSetDevice(x->c.device));
    const int one = 1;
    HH_CUDA(cudaMemcpyAsync(x->c.inject_word, &one, sizeof(int), cudaMemcpyHostToDevice, x->c.stream));
    HH_CUDA(cudaStreamSynchronize(x->c.stream));
    return HH_OK;
}

static void drain_events(Ctx &c) {
    if (!c.ev_pending.empty()) cudaEventSynchronize(c.ev_pending.back()); // all recorded events complete
    for (size_t g = 0; g + 4 <= c.ev_pending.size(); g += 4) {
        float t;
        for (int s = 0; s < 3; s++) {
            if (cudaEventElapsedTime(&t, c.ev_pending[g + s], c.ev_pending[g + s + 1]) == cudaSuccess)
                c.stage_ms[s] += t;
        }
        for (int s = 0; s < 4; s++) cudaEventDestroy(c.ev_pending[g + s]);
    }
    c.ev_pending.clear();
}

extern "C" int hh_ctx_set_stage_timing(hh_ctx *x, int on) {
    if (!x) return HH_ERR_INVALID;
    x->c.timing = on != 0;
    return HH_OK;
}

extern "C" int hh_ctx_stage_times(hh_ctx *x, double ms[HH_NUM_STAGES], long long *solves) {
    if (!x || !ms) return HH_ERR_INVALID;
    HH_CUDA(cudaStreamSynchronize(x->c.stream));
    drain_events(x->c);
    for (int s = 0; s < 3; s++) {
        ms[s] = x->c.stage_ms[s];
        x->c.stage_ms[s] = 0.0;
    }
    if (solves) *solves = x->c.timed_solves;
    x->c.timed_solves = 0;
    return HH_OK;
}

// records event `k` (0..3) of the current timed solve
static int stage_mark(Ctx &c, int k) {
    if (!c.timing) return HH_OK;
    if (k == 0 && c.ev_pending.size() >= 4 * 64) drain_events(c); // bound the backlog
    cudaEvent_t e;
    HH_CUDA(cudaEventCreate(&e));
    HH_CUDA(cudaEventRecord(e, c.stream));
    c.ev_pending.push_back(e);
    if (k == 3) c.timed_solves++;
    return HH_OK;
}

extern "C" int hh_malloc(hh_ctx *x, size_t bytes, void **p) {
    if (!x || !p) return HH_ERR_INVALID;
    HH_CUDA(cudaSetDevice(x->c.device));
    HH_CUDA(cudaMalloc(p, bytes));
    return HH_OK;
}
extern "C" int hh_free(hh_ctx *x, void *p) {
    if (!x) return HH_ERR_INVALID;
    HH_CUDA(cudaFree(p));
    return HH_OK;
}
extern "C" int hh_memcpy_h2d(hh_ctx *x, void *d, const void *s, size_t n) {
    if (!x) return HH_ERR_INVALID;
    HH_CUDA(cudaMemcpyAsync(d, s, n, cudaMemcpyHostToDevice, x->c.stream));
    HH_CUDA(cudaStreamSynchronize(x->c.stream));
    return HH_OK;
}
extern "C" int hh_memcpy_d2h(hh_ctx *x, void *d, const void *s, size_t n) {
    if (!x) return HH_ERR_INVALID;
    HH_CUDA(cudaMemcpyAsync(d, s, n, cudaMemcpyDeviceToHost, x->c.stream));
    HH_CUDA(cudaStreamSynchronize(x->c.stream));
    return HH_OK;
}

// --------------------------------------------------------------- transforms ------
extern "C" int hh_dst1_rows(hh_ctx *x, int n, long rows, const double *in, long in_ld, double *out, long out_ld) {
    if (!x || !in || !out || n < 1 || rows < 0 || in_ld < n || out_ld < n) {
        set_error("hh_dst1_rows: invalid arguments");
        return HH_ERR_INVALID;
    }
    return launch_dst_rows(&x->c, n, rows, (const double2 *)in, in_ld, (double2 *)out, out_ld);
}

extern "C" int hh_dst1_cols(hh_ctx *x, int n, long ncols, long planes, const double *in, long ld, long plane_stride,
                            double *out) {
    if (!x || !in || !out || n < 1 || ncols < 0 || planes < 0 || ld < ncols || planes > 65535) {
        set_error("hh_dst1_cols: invalid arguments");
        return HH_ERR_INVALID;
    }
    return launch_dst_cols(&x->c, n, ncols, planes, (const double2 *)in, ld, plane_stride, (double2 *)out);
}

extern "C" int hh_lines_pack(hh_ctx *x, const double *in, double *out, long batch, long planes, long nlines, int world,
                             int unpack) {
    if (!x || !in || !out || in == out || (unpack != 0 && unpack != 1)) {
        set_error("hh_lines_pack: invalid arguments");
        return HH_ERR_INVALID;
    }
    HH_CUDA(cudaSetDevice(x->c.device));
    return launch_lines_pack(&x->c, (const double2 *)in, (double2 *)out, batch, planes, nlines, world, unpack == 1);
}

extern "C" int hh_dst2_planes(hh_ctx *x, int nx, int ny, long nplanes, const double *in, double *out) {
    if (!x || !in || !out || nx < 1 || ny < 1 || nplanes < 0) {
        set_error("hh_dst2_planes: invalid arguments");
        return HH_ERR_INVALID;
    }
    const long plane = (long)nx * ny;
    HH_TRY(launch_dst_rows(&x->c, nx, (long)ny * nplanes, (const double2 *)in, nx, (double2 *)out, nx));
    for (long p0 = 0; p0 < nplanes; p0 += 65535) {
        const long np = (nplanes - p0 < 65535) ? nplanes - p0 : 65535;
        double2   *o = (double2 *)out + p0 * plane;
        HH_TRY(launch_dst_cols(&x->c, ny, nx, np, o, nx, plane, o));
    }
    return HH_OK;
}

// -------------------------------------------------------------------- plans ------
static int plan_alloc(hh_plan *pl) {
    Plan &p = pl->p;
    p.ctx->plans.push_back(&p);
    Ctx *c = p.ctx;
    HH_TRY(dalloc(c, (void **)&p.Pv, sizeof(double2) * (size_t)segment_count(p.rows) * p.lines));
    p.prow = padded_rows(p.rows);
    HH_TRY(dalloc(c, (void **)&p.rowc, sizeof(double2) * 4 * (size_t)p.prow));
    HH_TRY(dalloc(c, (void **)&p.subt, sizeof(double2) * 4 * (size_t)p.prow));
    HH_TRY(dalloc(c, (void **)&p.diagt, sizeof(double2) * 4 * (size_t)p.prow));
    HH_TRY(dalloc(c, (void **)&p.mu, sizeof(double) * 3 * (size_t)p.lines));
    // the context's transform tables for this plan's lengths are made here, at set-up, so that
    // solving never allocates
    HH_TRY(prepare_dst(c, p.nx));
    if (p.dim == 3) HH_TRY(prepare_dst(c, p.ny));
    return HH_OK;
}

static void plan_free(hh_plan *pl) {
    Plan &p = pl->p;
    if (p.ctx) {
        auto &v = p.ctx->plans;
        for (size_t i = 0; i < v.size(); i++)
            if (v[i] == &p) { v.erase(v.begin() + (long)i); break; }
    }
    Ctx *c = p.ctx;
    dfree(c, p.Pv);
    dfree(c, p.rowc);
    dfree(c, p.subt);
    dfree(c, p.diagt);
    dfree(c, p.mu);
    dfree(c, p.pade_l);
    dfree(c, p.pade_u);
}

// [1 10 1] Pade factors along the line direction (the reference's constant-coefficient solves,
// 2D_Program/partial_derivatives/4th_order_second_derivative.c:19-24,
// 3D_Program/partial_derivatives/4th_order_partials.c:118-123): U_0 = 10, L_r = 1/U_{r-1},
// U_r = 10 - L_r; the device keeps L_r (L_0 = 0) and 1/U_r.
static int plan_pade(hh_plan *pl) {
    Plan &p = pl->p;
    std::vector<double> L(p.prow, 0.0), Ui(p.prow, 0.0); // zero past the line (neutral rows)
    double U = 10.0;
    L[0] = 0.0;
    Ui[0] = 1.0 / U;
    for (int r = 1; r < p.rows; r++) {
        L[r] = 1.0 / U;
        U = 10.0 - L[r];
        Ui[r] = 1.0 / U;
    }
    // the kernel replaces rows >= 9 by the limit; it is an exact fixed point in double
    {
        double u = 10.0, lim_l = 0.0, lim_u = 0.0;
        for (int r = 1; r < 64; r++) {
            lim_l = 1.0 / u;
            u = 10.0 - lim_l;
            lim_u = 1.0 / u;
        }
        p.pade_linf = lim_l;
        p.pade_uinf = lim_u;
        for (int r = 9; r < p.rows; r++)
            if (L[r] != lim_l || Ui[r] != lim_u) {
                set_error("Pade factors not converged at row %d", r);
                return HH_ERR_UNSUPPORTED;
            }
    }
    HH_TRY(dalloc(p.ctx, (void **)&p.pade_l, sizeof(double) * (size_t)p.prow));
    HH_TRY(dalloc(p.ctx, (void **)&p.pade_u, sizeof(double) * (size_t)p.prow));
    HH_TRY(upload(p.ctx, p.pade_l, L.data(), sizeof(double) * (size_t)p.prow));
    HH_TRY(upload(p.ctx, p.pade_u, Ui.data(), sizeof(double) * (size_t)p.prow));
    return HH_OK;
}

// Build factors from host tables: sub/diag/sup are 4*rows complex each (see hh_tridiag.cu).
static int plan_factor(hh_plan *pl, const std::vector<double2> &sub, const std::vector<double2> &dia,
                       const std::vector<double2> &sup, const std::vector<double> &mu) {
    Plan &p = pl->p;
    Ctx  *c = p.ctx;
    // constant-coefficient lines (constant k): every row of the three tables equals row 0
    auto constant = [&](const std::vector<double2> &t) {
        for (int k = 0; k < 4; k++)
            for (int r = 1; r < p.rows; r++) {
                const double2 a0 = t[(size_t)k * p.rows], ar = t[(size_t)k * p.rows + r];
                if (a0.x != ar.x || a0.y != ar.y) return false;
            }
        return true;
    };
    p.const_rows = constant(sub) && constant(dia) && constant(sup);
    // symmetric constant lines (sub == super): the specialised solve; for order 6 it also needs
    // |10 s - d| well away from zero on every line (partial fractions of A^-1 T^-1), and s not
    // negligible beside d (the kernel re-forms 1/P as (1/s) (s / P))
    p.sym = p.const_rows;
    for (int k = 0; k < 4 && p.sym; k++) {
        const double2 a = sub[(size_t)k * p.rows], b = sup[(size_t)k * p.rows];
        p.sym = a.x == b.x && a.y == b.y;
    }
    p.pf_ok = p.sym;
    for (int q = 0; q < p.lines && p.pf_ok; q++) {
        auto line_value = [&](const std::vector<double2> &tb) {
            const double m0 = mu[q], m1 = mu[(size_t)p.lines + q], m2 = mu[2 * (size_t)p.lines + q];
            const double2 a = tb[0], b = tb[(size_t)p.rows], c = tb[2 * (size_t)p.rows], d = tb[3 * (size_t)p.rows];
            return make_double2(((a.x * m0 + b.x * m1) + c.x * m2) + d.x, ((a.y * m0 + b.y * m1) + c.y * m2) + d.y);
        };
        // |10 s - d| >= |s|, |d| / 4 and |s| > 1e-6 |d|, on squared moduli (one line of a 255^3
        // plan is one of 65025: three hypot calls per line cost milliseconds of set-up)
        const double2 s = line_value(sub), d = line_value(dia);
        const double  ex = 10.0 * s.x - d.x, ey = 10.0 * s.y - d.y;
        const double  num2 = ex * ex + ey * ey;
        const double  as2 = s.x * s.x + s.y * s.y, ad2 = d.x * d.x + d.y * d.y;
        p.pf_ok = num2 >= 0.0625 * std::max(as2, ad2) && as2 > 1e-12 * ad2;
    }
    if (p.sym) p.variant = sym_default_variant(p.rows);
    // tables are [4][prow], zero past the last row (neutral rows in the solve)
    auto padded = [&](const std::vector<double2> &t) {
        std::vector<double2> o(4 * (size_t)p.prow, make_double2(0.0, 0.0));
        for (int k = 0; k < 4; k++)
            for (int r = 0; r < p.rows; r++) o[(size_t)k * p.prow + r] = t[(size_t)k * p.rows + r];
        return o;
    };
    const std::vector<double2> psub = padded(sub), pdia = padded(dia), psup = padded(sup);
    const size_t tb = sizeof(double2) * 4 * (size_t)p.prow;
    int rc = upload(c, p.subt, psub.data(), tb);
    if (rc == HH_OK) rc = upload(c, p.diagt, pdia.data(), tb);
    if (rc == HH_OK) rc = upload(c, p.rowc, psup.data(), tb);
    if (rc == HH_OK) rc = upload(c, p.mu, mu.data(), sizeof(double) * 3 * (size_t)p.lines);
    if (rc == HH_OK) rc = launch_factor(&p, p.subt, p.diagt, p.rowc);
    // contexts with a pool (the request loop) keep set-up asynchronous: its failures surface at
    // the next synchronization of the stream
    cudaError_t e = c->pool ? cudaGetLastError() : cudaStreamSynchronize(c->stream);
    if (rc != HH_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "factorisation", __FILE__, __LINE__);
    return HH_OK;
}

static inline double2 cget(const double *a, int j) { return make_double2(a[2 * j], a[2 * j + 1]); }

extern "C" int hh_plan2d_create(hh_ctx *x, int nx, int ny, const double *bp, const double *ap, const double *b,
                                const double *a, const double *bm, const double *am, hh_plan **out) {
    if (!x || !out || nx < 1 || ny < 1 || !bp || !ap || !b || !a || !bm || !am) {
        set_error("hh_plan2d_create: invalid arguments");
        return HH_ERR_INVALID;
    }
    *out = nullptr;
    HH_CUDA(cudaSetDevice(x->c.device));
    hh_plan *pl = new hh_plan();
    Plan    &p = pl->p;
    p.ctx = &x->c;
    p.dim = 2;
    p.nx = nx;
    p.ny = ny;
    p.lines = nx;
    p.rows = ny;
    p.row_stride = nx;
    p.field = (long)nx * ny;
    int rc = plan_alloc(pl);
    if (rc != HH_OK) { plan_free(pl); delete pl; return rc; }
    // eigenvalues of the x second difference, as 2D LU.c:12-14
    std::vector<double> mu(3 * (size_t)nx, 0.0);
    for (int i = 0; i < nx; i++) mu[nx + i] = 2.0 * cos((i + 1) * M_PI / (nx + 1));
    std::vector<double2> sub(4 * (size_t)ny), dia(4 * (size_t)ny), sup(4 * (size_t)ny);
    const double2 z = make_double2(0.0, 0.0);
    for (int j = 0; j < ny; j++) {
        sub[j] = z; sub[ny + j] = cget(bm, j); sub[2 * ny + j] = z; sub[3 * ny + j] = cget(am, j);
        dia[j] = z; dia[ny + j] = cget(b, j);  dia[2 * ny + j] = z; dia[3 * ny + j] = cget(a, j);
        sup[j] = z; sup[ny + j] = cget(bp, j); sup[2 * ny + j] = z; sup[3 * ny + j] = cget(ap, j);
    }
    rc = plan_factor(pl, sub, dia, sup, mu);
    if (rc != HH_OK) { plan_free(pl); delete pl; return rc; }
    *out = pl;
    return HH_OK;
}

// A 3D plan over lines [q0, q1) of the nx * ny (i, j) lines, q = i + j nx: the whole field for
// hh_plan3d_create, one rank's pencil for hh_plan3d_create_helmholtz_lines.
static int plan3d_create_lines(hh_ctx *x, int nx, int ny, int nz, const double *const coef[12], long q0, long q1,
                               hh_plan **out) {
    if (!x || !out || nx < 1 || ny < 1 || nz < 1 || !coef || q0 < 0 || q1 <= q0 || q1 > (long)nx * ny) {
        set_error("hh_plan3d_create: invalid arguments");
        return HH_ERR_INVALID;
    }
    for (int t = 0; t < 12; t++)
        if (!coef[t]) { set_error("hh_plan3d_create: null coefficient %d", t); return HH_ERR_INVALID; }
    *out = nullptr;
    HH_CUDA(cudaSetDevice(x->c.device));
    hh_plan *pl = new hh_plan();
    Plan    &p = pl->p;
    p.ctx = &x->c;
    p.dim = 3;
    p.nx = nx;
    p.ny = ny;
    p.nz = nz;
    p.line0 = q0;
    p.lines_only = q0 > 0 || q1 < (long)nx * ny;
    p.lines = (int)(q1 - q0);
    p.rows = nz;
    p.row_stride = p.lines;
    p.field = (long)p.lines * nz;
    int rc = plan_alloc(pl);
    if (rc != HH_OK) { plan_free(pl); delete pl; return rc; }
    // eigenvalue products per (i,j) line, as 3D LU.c:31-44
    std::vector<double> mu(3 * (size_t)p.lines), exs((size_t)nx), eys((size_t)ny);
    for (int i = 0; i < nx; i++) exs[(size_t)i] = 2.0 * cos((i + 1) * M_PI / (nx + 1));
    for (int j = 0; j < ny; j++) eys[(size_t)j] = 2.0 * cos((j + 1) * M_PI / (ny + 1));
    for (long q = q0; q < q1; q++) {
        const int    i = (int)(q % nx), j = (int)(q / nx);
        const double ey = eys[(size_t)j], ex = exs[(size_t)i];
        const long   t = q - q0;
        mu[(size_t)t] = ex * ey;
        mu[p.lines + (size_t)t] = ex;
        mu[2 * (size_t)p.lines + (size_t)t] = ey;
    }
    // coef order a,b,c,d,ap,bp,cp,dp,am,bm,cm,dm -> (corner, x-neighbour, y-neighbour, centre)
    std::vector<double2> sub(4 * (size_t)nz), dia(4 * (size_t)nz), sup(4 * (size_t)nz);
    for (int l = 0; l < nz; l++)
        for (int t = 0; t < 4; t++) {
            dia[t * (size_t)nz + l] = cget(coef[t], l);
            sup[t * (size_t)nz + l] = cget(coef[4 + t], l);
            sub[t * (size_t)nz + l] = cget(coef[8 + t], l);
        }
    rc = plan_factor(pl, sub, dia, sup, mu);
    if (rc != HH_OK) { plan_free(pl); delete pl; return rc; }
    *out = pl;
    return HH_OK;
}

extern "C" int hh_plan3d_create(hh_ctx *x, int nx, int ny, int nz, const double *const coef[12], hh_plan **out) {
    return plan3d_create_lines(x, nx, ny, nz, coef, 0, (long)nx * ny, out);
}

extern "C" int hh_plan2d_create_helmholtz(hh_ctx *x, int n, int order, double kr, double ki, hh_plan **out) {
    std::vector<double> buf(6 * 2 * (size_t)n);
    double *arr[6];
    for (int t = 0; t < 6; t++) arr[t] = buf.data() + t * 2 * (size_t)n;
    int rc = hh_coefficients2d(n, order, kr, ki, arr);
    if (rc != HH_OK) { set_error("hh_plan2d_create_helmholtz: order must be 2, 4 or 6"); return rc; }
    HH_TRY(hh_plan2d_create(x, n, n, arr[0], arr[1], arr[2], arr[3], arr[4], arr[5], out));
    Plan &p = (*out)->p;
    p.order = order;
    p.src_order = order;
    p.h = 1.0 / (n + 1);
    p.k2 = make_double2(kr * kr - ki * ki, 2.0 * kr * ki);
    int rc2 = plan_pade(*out);
    if (rc2 != HH_OK) { hh_plan_destroy(*out); *out = nullptr; return rc2; }
    return HH_OK;
}

extern "C" int hh_plan3d_create_helmholtz_lines(hh_ctx *x, int n, int order, double kr, double ki, long q0, long q1,
                                                hh_plan **out) {
    if (n < 1) { set_error("hh_plan3d_create_helmholtz: n = %d", n); return HH_ERR_INVALID; }
    std::vector<double> buf(12 * 2 * (size_t)n);
    double *arr[12];
    for (int t = 0; t < 12; t++) arr[t] = buf.data() + t * 2 * (size_t)n;
    int rc = hh_coefficients3d(n, order, kr, ki, arr);
    if (rc != HH_OK) { set_error("hh_plan3d_create_helmholtz: order must be 2, 4 or 6"); return rc; }
    const double *carr[12];
    for (int t = 0; t < 12; t++) carr[t] = arr[t];
    HH_TRY(plan3d_create_lines(x, n, n, n, carr, q0, q1, out));
    Plan &p = (*out)->p;
    p.order = order;
    p.src_order = order;
    p.h = 1.0 / (n + 1);
    p.k2 = make_double2(kr * kr - ki * ki, 2.0 * kr * ki);
    int rc2 = plan_pade(*out);
    if (rc2 != HH_OK) { hh_plan_destroy(*out); *out = nullptr; return rc2; }
    return HH_OK;
}

extern "C" int hh_plan3d_create_helmholtz(hh_ctx *x, int n, int order, double kr, double ki, hh_plan **out) {
    return hh_plan3d_create_helmholtz_lines(x, n, order, kr, ki, 0, (long)n * n, out);
}

extern "C" int hh_plan_destroy(hh_plan *pl) {
    if (!pl) return HH_OK;
    cudaSetDevice(pl->p.ctx->device);
    if (!pl->p.ctx->pool) cudaStreamSynchronize(pl->p.ctx->stream); // pool frees are stream-ordered
    plan_free(pl);
    delete pl;
    return HH_OK;
}

extern "C" long hh_plan_field_size(const hh_plan *pl) { return pl ? pl->p.field : 0; }

static int check_batch(hh_plan *pl, int batch);

extern "C" int hh_plan_set_variant(hh_plan *pl, int variant) {
    if (!pl || variant < 0 || variant >= solve_variant_count()) {
        set_error("invalid plan or line-solve variant %d", variant);
        return HH_ERR_INVALID;
    }
    pl->p.variant = variant;
    return HH_OK;
}

extern "C" int hh_plan_variant(const hh_plan *pl) { return pl ? pl->p.variant : -1; }

static int transform_forward(Plan &p, const double2 *in, double2 *out, int batch, bool lp = false);
static int transform_inverse(Plan &p, double2 *buf, int batch, bool lp = false);

// Times every line-solve variant on `batch` zero right-hand sides (the solve does the same work
// for any values) and keeps the fastest.  Blocks; must not run inside a stream capture.
static int tune_measure(hh_plan *pl, int batch) {
    Plan &p = pl->p;
    Ctx  *c = p.ctx;
    HH_CUDA(cudaSetDevice(c->device));
    double2 *buf = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = HH_OK, best = p.variant;
    float best_ms = 1e30f;
    const int src = p.src_order;
    auto run = [&]() -> int {
        if (cudaMalloc(&buf, sizeof(double2) * (size_t)p.field * batch) != cudaSuccess ||
            cudaMemsetAsync(buf, 0, sizeof(double2) * (size_t)p.field * batch, c->stream) != cudaSuccess ||
            cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
            set_error("hh_plan_tune: %s", cudaGetErrorString(cudaGetLastError()));
            return HH_ERR_CUDA;
        }
        for (int v = 0; v < solve_variant_count(); v++) {
            p.variant = v;
            HH_TRY(launch_line_solve(&p, buf, buf, batch, src)); // warm-up
            HH_CUDA(cudaEventRecord(e0, c->stream));
            for (int r = 0; r < 3; r++) HH_TRY(launch_line_solve(&p, buf, buf, batch, src));
            HH_CUDA(cudaEventRecord(e1, c->stream));
            HH_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            HH_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best_ms) {
                best_ms = ms;
                best = v;
            }
        }
        return HH_OK;
    };
    rc = run();
    p.variant = best;
    // the rows transform: the CTA ring or per-warp line buffers (lengths n + 1 = 64 .. 1024), the
    // two-warp line kernel or the Stockham kernel (2048), timed as one forward and one inverse
    // transform of the batch
    const int mx = p.nx + 1;
    if (rc == HH_OK && mx >= 64 && mx <= 2048 && (mx & (mx - 1)) == 0) {
        int   best_rk = p.rows_kernel;
        float best_t = 1e30f;
        for (int rk = 1; rk <= 2 && rc == HH_OK; rk++) {
            p.rows_kernel = rk;
            auto pass = [&]() -> int {
                HH_TRY(transform_forward(p, buf, buf, batch));
                return transform_inverse(p, buf, batch);
            };
            if ((rc = pass()) != HH_OK) break;
            if (cudaEventRecord(e0, c->stream) != cudaSuccess) { rc = HH_ERR_CUDA; break; }
            for (int r = 0; r < 3 && rc == HH_OK; r++) rc = pass();
            if (rc != HH_OK) break;
            float ms = 0.f;
            if (cudaEventRecord(e1, c->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = HH_ERR_CUDA;
                break;
            }
            if (ms < best_t) {
                best_t = ms;
                best_rk = rk;
            }
        }
        p.rows_kernel = best_rk;
    }
    // 3D plans: the slab of the transform passes, over candidates from a sixteenth of L2 to the
    // whole batch, timed as one forward and one inverse transform
    if (rc == HH_OK && p.dim == 3) {
        const long planes = (long)p.nz * batch, plane_bytes = 16L * p.nx * p.ny;
        std::vector<long> cand = {planes};
        for (long div : {16L, 8L, 4L, 3L, 2L}) {
            const long sp = std::max(1L, (long)(c->l2_bytes / div) / plane_bytes);
            if (sp < planes && std::find(cand.begin(), cand.end(), sp) == cand.end()) cand.push_back(sp);
        }
        long  best_slab = p.slab;
        int   best_ck = p.col_kernel;
        float best_t = 1e30f;
        for (int trial = 0; trial < 2 * (int)cand.size(); trial++) {
            const long sp = cand[(size_t)trial / 2];
            p.slab = sp;
            p.col_kernel = trial % 2;
            auto pass = [&]() -> int {
                HH_TRY(transform_forward(p, buf, buf, batch));
                return transform_inverse(p, buf, batch);
            };
            if ((rc = pass()) != HH_OK) break;
            if (cudaEventRecord(e0, c->stream) != cudaSuccess) { rc = HH_ERR_CUDA; break; }
            for (int r = 0; r < 3 && rc == HH_OK; r++) rc = pass();
            if (rc != HH_OK) break;
            float ms = 0.f;
            if (cudaEventRecord(e1, c->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
                rc = HH_ERR_CUDA;
                break;
            }
            if (ms < best_t) {
                best_t = ms;
                best_slab = sp;
                best_ck = p.col_kernel;
            }
        }
        p.slab = best_slab;
        p.col_kernel = best_ck;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (buf) {
        cudaStreamSynchronize(c->stream);
        cudaFree(buf);
    }
    if (rc == HH_OK) rc = hh_ctx_synchronize(reinterpret_cast<hh_ctx *>(c)); // Ctx is hh_ctx's first member
    return rc;
}

// ------------------------------------------------------------------ tuning cache ------
// The kernel settings hh_plan_tune measures (line-solve variant; for 3D plans also the column
// transform kernel and the transform slab), remembered per device model and problem shape: dim,
// sizes, the fused source order and which line-solve kernels the plan's stencil admits.  The
// wavenumber does not change which kernel is fastest (every variant does the same work for any
// coefficients), so plans of one shape at different k share an entry.  Process-wide, guarded by a
// mutex; hh_tune_cache_save / _load keep it in a text file (one tab-separated entry per line).
namespace {
struct TuneEntry {
    int  variant = 0, col_kernel = 0, rows_kernel = 0;
    long slab = 0;
};
std::mutex                       g_tune_mu;
std::map<std::string, TuneEntry> g_tune;
long long                        g_tune_hits = 0, g_tune_misses = 0;

std::string tune_key(const Plan &p) {
    char      buf[512];
    const int kinds = p.sym ? (p.pf_ok ? 2 : 1) : 0;
    snprintf(buf, sizeof buf, "%s\t%d\t%d\t%d\t%d\t%d\t%d", p.ctx->dev_name.c_str(), p.dim, p.nx, p.ny, p.nz,
             p.src_order, kinds);
    return buf;
}

bool tune_apply(Plan &p, const TuneEntry &e) {
    if (e.variant < 0 || e.variant >= solve_variant_count() || (e.variant >= 2 && !p.sym) || e.col_kernel < 0 ||
        e.col_kernel > 1 || e.rows_kernel < 0 || e.rows_kernel > 2 || e.slab < 0)
        return false;
    p.variant = e.variant;
    p.col_kernel = e.col_kernel;
    p.rows_kernel = e.rows_kernel;
    p.slab = e.slab;
    return true;
}
} // namespace

// Applies the cached settings of the plan's shape; *found = 0 (plan unchanged) when there are none.
extern "C" int hh_plan_apply_tuning(hh_plan *pl, int *found) {
    if (!pl || !found) { set_error("hh_plan_apply_tuning: invalid arguments"); return HH_ERR_INVALID; }
    const std::string key = tune_key(pl->p);
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(key);
    *found = it != g_tune.end() && tune_apply(pl->p, it->second);
    return HH_OK;
}

extern "C" int hh_plan_tune(hh_plan *pl, int batch) {
    HH_TRY(check_batch(pl, batch));
    if (batch == 0) return HH_OK;
    int found = 0;
    HH_TRY(hh_plan_apply_tuning(pl, &found));
    if (found) {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune_hits++;
        return HH_OK;
    }
    HH_TRY(tune_measure(pl, batch));
    TuneEntry e;
    e.variant = pl->p.variant;
    e.col_kernel = pl->p.col_kernel;
    e.rows_kernel = pl->p.rows_kernel;
    e.slab = pl->p.slab;
    const std::string key = tune_key(pl->p);
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune[key] = e;
    g_tune_misses++;
    return HH_OK;
}

extern "C" int hh_tune_cache_stats(long long *hits, long long *misses, long long *entries) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    if (hits) *hits = g_tune_hits;
    if (misses) *misses = g_tune_misses;
    if (entries) *entries = (long long)g_tune.size();
    return HH_OK;
}

extern "C" int hh_tune_cache_clear(void) {
    std::lock_guard<std::mutex> g(g_tune_mu);
    g_tune.clear();
    g_tune_hits = g_tune_misses = 0;
    return HH_OK;
}

extern "C" int hh_tune_cache_save(const char *path) {
    if (!path) { set_error("hh_tune_cache_save: null path"); return HH_ERR_INVALID; }
    std::lock_guard<std::mutex> g(g_tune_mu);
    FILE *f = fopen(path, "w");
    if (!f) { set_error("hh_tune_cache_save: cannot write %s", path); return HH_ERR_INVALID; }
    fprintf(f, "# hackathon_b200 tuning cache: device, dim, nx, ny, nz, source order, kernels, variant, column kernel, "
               "slab, rows kernel\n");
    for (auto &kv : g_tune)
        fprintf(f, "%s\t%d\t%d\t%ld\t%d\n", kv.first.c_str(), kv.second.variant, kv.second.col_kernel, kv.second.slab,
                kv.second.rows_kernel);
    const bool ok = fclose(f) == 0;
    if (!ok) { set_error("hh_tune_cache_save: write error on %s", path); return HH_ERR_INVALID; }
    return HH_OK;
}

// Adds the entries of a file written by hh_tune_cache_save (malformed lines are skipped);
// *loaded (optional) receives the number of entries read.
extern "C" int hh_tune_cache_load(const char *path, long long *loaded) {
    if (!path) { set_error("hh_tune_cache_load: null path"); return HH_ERR_INVALID; }
    FILE *f = fopen(path, "r");
    if (!f) { set_error("hh_tune_cache_load: cannot read %s", path); return HH_ERR_INVALID; }
    char      line[1024];
    long long n = 0;
    std::lock_guard<std::mutex> g(g_tune_mu);
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '#') continue;
        // the last four tab-separated fields are the settings, the rest is the key
        std::string l(line);
        while (!l.empty() && (l.back() == '\n' || l.back() == '\r')) l.pop_back();
        size_t cut[4];
        size_t pos = l.size();
        bool   ok = true;
        for (int t = 0; t < 4 && ok; t++) {
            pos = l.rfind('\t', pos == 0 ? 0 : pos - 1);
            ok = pos != std::string::npos && pos > 0;
            cut[t] = pos;
        }
        if (!ok) continue;
        TuneEntry e;
        char     *end = nullptr;
        e.variant = (int)strtol(l.c_str() + cut[3] + 1, &end, 10);
        e.col_kernel = (int)strtol(l.c_str() + cut[2] + 1, &end, 10);
        e.slab = strtol(l.c_str() + cut[1] + 1, &end, 10);
        e.rows_kernel = (int)strtol(l.c_str() + cut[0] + 1, &end, 10);
        g_tune[l.substr(0, cut[3])] = e;
        n++;
    }
    fclose(f);
    if (loaded) *loaded = n;
    return HH_OK;
}

// -------------------------------------------------------------------- solve ------
// 3D transforms can run slab by slab: the rows pass over a slab of planes, then the columns
// pass over the same slab, which then finds the rows pass's output in L2, so that a value crosses
// HBM once per direction instead of twice (the reference's per-plane DST(),
// 3D_Program/solver_functions/DST.c:148-204 inside solver.c:338-350, makes both passes over one
// plane at a time in host memory).  Measured at 255^3 x 4: both passes are bound by latency, not
// by HBM, so the extra launches cost more than the saved traffic (2.73 ms per solve over the
// whole batch, 2.82 ms with slabs of 128 planes, 5.34 ms with 8); the default is therefore the
// whole batch in one slab, and hh_plan_tune keeps a smaller slab only where it measures faster.
long hh::slab_planes(const Plan &p, long planes) {
    const long s = p.slab > 0 ? p.slab : planes;
    return std::max(1L, std::min(std::min(s, planes), 65535L));
}

// lp: single-precision transform arithmetic (the refined solve's low-precision solves)
static int transform_forward(Plan &p, const double2 *in, double2 *out, int batch, bool lp) {
    Ctx *c = p.ctx;
    if (p.dim == 2) return launch_dst_rows(c, p.nx, (long)p.ny * batch, in, p.nx, out, p.nx, lp, p.rows_kernel);
    const long plane = (long)p.nx * p.ny, planes = (long)p.nz * batch, sp = slab_planes(p, planes);
    for (long p0 = 0; p0 < planes; p0 += sp) {
        const long np = std::min(sp, planes - p0);
        HH_TRY(launch_dst_rows(c, p.nx, (long)p.ny * np, in + p0 * plane, p.nx, out + p0 * plane, p.nx, lp,
                               p.rows_kernel));
        HH_TRY(launch_dst_cols(c, p.ny, p.nx, np, out + p0 * plane, p.nx, plane, out + p0 * plane, lp, p.col_kernel));
    }
    return HH_OK;
}

static int transform_inverse(Plan &p, double2 *buf, int batch, bool lp) {
    Ctx *c = p.ctx;
    if (p.dim == 2) return launch_dst_rows(c, p.nx, (long)p.ny * batch, buf, p.nx, buf, p.nx, lp, p.rows_kernel);
    const long plane = (long)p.nx * p.ny, planes = (long)p.nz * batch, sp = slab_planes(p, planes);
    for (long p0 = 0; p0 < planes; p0 += sp) {
        const long np = std::min(sp, planes - p0);
        HH_TRY(launch_dst_cols(c, p.ny, p.nx, np, buf + p0 * plane, p.nx, plane, buf + p0 * plane, lp, p.col_kernel));
        HH_TRY(launch_dst_rows(c, p.nx, (long)p.ny * np, buf + p0 * plane, p.nx, buf + p0 * plane, p.nx, lp,
                               p.rows_kernel));
    }
    return HH_OK;
}

extern "C" int hh_plan_set_slab(hh_plan *pl, long planes) {
    if (!pl || planes < 0) {
        set_error("hh_plan_set_slab: invalid plan or slab (%ld)", planes);
        return HH_ERR_INVALID;
    }
    pl->p.slab = planes;
    return HH_OK;
}

extern "C" long hh_plan_slab(const hh_plan *pl) { return pl ? pl->p.slab : -1; }

extern "C" int hh_plan_set_dst_variant(hh_plan *pl, int v) {
    if (!pl || v < 0 || v > 1) {
        set_error("hh_plan_set_dst_variant: invalid plan or variant (%d)", v);
        return HH_ERR_INVALID;
    }
    pl->p.col_kernel = v;
    return HH_OK;
}

extern "C" int hh_plan_dst_variant(const hh_plan *pl) { return pl ? pl->p.col_kernel : -1; }

extern "C" int hh_plan_set_rows_variant(hh_plan *pl, int v) {
    if (!pl || v < 0 || v > 2) {
        set_error("hh_plan_set_rows_variant: invalid plan or variant (%d)", v);
        return HH_ERR_INVALID;
    }
    pl->p.rows_kernel = v;
    return HH_OK;
}

extern "C" int hh_plan_rows_variant(const hh_plan *pl) { return pl ? pl->p.rows_kernel : -1; }

static int check_batch(hh_plan *pl, int batch) {
    if (!pl || batch < 0 || batch > 65535) {
        set_error("invalid plan or batch (%d)", batch);
        return HH_ERR_INVALID;
    }
    if (pl->p.lines_only) {
        set_error("a line-range plan solves lines only (hh_solve_lines)");
        return HH_ERR_INVALID;
    }
    return HH_OK;
}

// The line solve alone, on right-hand sides already transformed along the other axes: the
// middle step of hh_solve (fused = 0) or of hh_solve_source (fused = 1, Helmholtz plans), with
// element (row r, line q) of right-hand side b at b field + r row_stride + q.
extern "C" int hh_solve_lines_strided(hh_plan *pl, const double *in, double *out, int batch, int fused, long row_stride,
                                      long field) {
    if (!pl || batch < 0 || batch > 65535 || (fused != 0 && fused != 1)) {
        set_error("hh_solve_lines: invalid plan, batch (%d) or fused (%d)", batch, fused);
        return HH_ERR_INVALID;
    }
    if (batch == 0) return HH_OK;
    if (!in || !out) { set_error("hh_solve_lines: null buffer"); return HH_ERR_INVALID; }
    Plan &p = pl->p;
    if (fused && p.src_order == 0) {
        set_error("hh_solve_lines: the fused operator needs a Helmholtz plan");
        return HH_ERR_INVALID;
    }
    // the fields either follow each other (field >= rows row_stride) or interleave row by row
    // (row_stride >= batch field); lines are contiguous either way
    const bool rhs_major = row_stride >= p.lines && field >= (long)p.rows * row_stride;
    const bool row_major = field >= p.lines && row_stride >= (long)batch * field;
    if (!rhs_major && !row_major) {
        set_error("hh_solve_lines: overlapping layout (row stride %ld, field %ld, %d lines of %d rows, batch %d)",
                  row_stride, field, p.lines, p.rows, batch);
        return HH_ERR_INVALID;
    }
    HH_CUDA(cudaSetDevice(p.ctx->device));
    Plan q = p; // the same factors and tables over another layout of the fields
    q.row_stride = row_stride;
    q.field = field;
    return launch_line_solve(&q, (const double2 *)in, (double2 *)out, batch, fused ? p.src_order : 0);
}

extern "C" int hh_solve_lines(hh_plan *pl, const double *in, double *out, int batch, int fused) {
    if (!pl) { set_error("hh_solve_lines: invalid plan"); return HH_ERR_INVALID; }
    return hh_solve_lines_strided(pl, in, out, batch, fused, pl->p.row_stride, pl->p.field);
}

extern "C" int hh_solve(hh_plan *pl, const double *rhs, double *sol, int batch) {
    HH_TRY(check_batch(pl, batch));
    if (batch == 0) return HH_OK;
    if (!rhs || !sol) { set_error("hh_solve: null buffer"); return HH_ERR_INVALID; }
    Plan &p = pl->p;
    HH_CUDA(cudaSetDevice(p.ctx->device));
    double2 *u = (double2 *)sol;
    HH_TRY(stage_mark(*p.ctx, 0));
    HH_TRY(transform_forward(p, (const double2 *)rhs, u, batch));
    HH_TRY(stage_mark(*p.ctx, 1));
    HH_TRY(launch_line_solve(&p, u, u, batch, 0));
    HH_TRY(stage_mark(*p.ctx, 2));
    HH_TRY(transform_inverse(p, u, batch));
    return stage_mark(*p.ctx, 3);
}

// The residual maxima buffer of a context (two words, made on first use).
static int ctx_norms(Ctx *c, unsigned long long **out) {
    if (!c->norms) HH_CUDA(cudaMalloc(&c->norms, 2 * sizeof(unsigned long long)));
    *out = c->norms;
    return HH_OK;
}

extern "C" int hh_residual(hh_plan *pl, const double *sol, const double *rhs, double *res, int batch,
                           double *max_res, double *max_rhs) {
    HH_TRY(check_batch(pl, batch));
    if (batch == 0) return HH_OK;
    if (!sol || !rhs || !res) { set_error("hh_residual: null buffer"); return HH_ERR_INVALID; }
    if (res == sol) { set_error("hh_residual: res must not be the solution buffer"); return HH_ERR_INVALID; }
    Plan &p = pl->p;
    Ctx  *c = p.ctx;
    HH_CUDA(cudaSetDevice(c->device));
    unsigned long long *norms = nullptr;
    const bool          want = max_res || max_rhs;
    if (want) {
        HH_TRY(ctx_norms(c, &norms));
        HH_CUDA(cudaMemsetAsync(norms, 0, 2 * sizeof(unsigned long long), c->stream));
    }
    HH_TRY(launch_residual(&p, (const double2 *)sol, (const double2 *)rhs, (double2 *)res, batch, norms));
    if (want) {
        unsigned long long h[2];
        HH_CUDA(cudaMemcpyAsync(h, norms, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
        HH_CUDA(cudaStreamSynchronize(c->stream));
        double v[2];
        memcpy(v, h, sizeof(v));
        if (max_res) *max_res = v[0];
        if (max_rhs) *max_rhs = v[1];
    }
    return HH_OK;
}

// Mixed-precision refined solve of assembled right-hand sides: each solve of the loop runs its
// transforms in single-precision arithmetic and its line solves in FP64; the residual and the
// update are FP64.  u_0 = S(rhs); u_{k+1} = u_k - S(A_h u_k - rhs) until max|A_h u - rhs| /
// max|rhs| <= tol or max_iter corrections.
extern "C" int hh_solve_refined(hh_plan *pl, const double *rhs, double *sol, int batch, double tol, int max_iter,
                                int *iters, double *rel_res) {
    HH_TRY(check_batch(pl, batch));
    if (batch == 0) return HH_OK;
    if (!rhs || !sol) { set_error("hh_solve_refined: null buffer"); return HH_ERR_INVALID; }
    if (rhs == sol) { set_error("hh_solve_refined: rhs and sol must be different buffers"); return HH_ERR_INVALID; }
    if (!(tol > 0.0) || max_iter < 0) { set_error("hh_solve_refined: tol must be > 0, max_iter >= 0"); return HH_ERR_INVALID; }
    Plan &p = pl->p;
    Ctx  *c = p.ctx;
    HH_CUDA(cudaSetDevice(c->device));
    const long need = p.field * (long)batch;
    if (c->refine_elems < need) { // the workspace grows to the largest batch seen
        HH_CUDA(cudaStreamSynchronize(c->stream));
        cudaFree(c->refine_work);
        c->refine_work = nullptr;
        c->refine_elems = 0;
        HH_CUDA(cudaMalloc(&c->refine_work, sizeof(double2) * (size_t)need));
        c->refine_elems = need;
    }
    unsigned long long *norms = nullptr;
    HH_TRY(ctx_norms(c, &norms));
    double2       *u = (double2 *)sol, *w = c->refine_work;
    const double2 *f = (const double2 *)rhs;
    auto low_solve = [&](const double2 *in, double2 *out) -> int {
        HH_TRY(transform_forward(p, in, out, batch, true));
        HH_TRY(launch_line_solve(&p, out, out, batch, 0));
        return transform_inverse(p, out, batch, true);
    };
    // a correction u <- u - S(w): the last (rows) pass of the inverse transform subtracts its
    // result from u as it stores, where the rows kernel has that form; else a separate update
    auto correct = [&]() -> int {
        if (!rows_update_supported(p.nx, p.rows_kernel)) {
            HH_TRY(low_solve(w, w));
            return launch_axpy(c, u, w, -1.0, need);
        }
        HH_TRY(transform_forward(p, w, w, batch, true));
        HH_TRY(launch_line_solve(&p, w, w, batch, 0));
        if (p.dim == 2) return launch_dst_rows_update(c, p.nx, (long)p.ny * batch, w, p.nx, u, p.nx, p.rows_kernel);
        const long plane = (long)p.nx * p.ny, planes = (long)p.nz * batch, sp = slab_planes(p, planes);
        for (long p0 = 0; p0 < planes; p0 += sp) {
            const long np = std::min(sp, planes - p0);
            HH_TRY(launch_dst_cols(c, p.ny, p.nx, np, w + p0 * plane, p.nx, plane, w + p0 * plane, true, p.col_kernel));
            HH_TRY(launch_dst_rows_update(c, p.nx, (long)p.ny * np, w + p0 * plane, p.nx, u + p0 * plane, p.nx,
                                          p.rows_kernel));
        }
        return HH_OK;
    };
    HH_TRY(low_solve(f, u));
    int    k = 0;
    double rr = 0.0;
    for (;;) {
        HH_CUDA(cudaMemsetAsync(norms, 0, 2 * sizeof(unsigned long long), c->stream));
        HH_TRY(launch_residual(&p, u, f, w, batch, norms));
        unsigned long long h[2];
        HH_CUDA(cudaMemcpyAsync(h, norms, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
        HH_CUDA(cudaStreamSynchronize(c->stream));
        double v[2];
        memcpy(v, h, sizeof(v));
        rr = v[1] > 0.0 ? v[0] / v[1] : 0.0;
        if (rr <= tol || k >= max_iter) break;
        HH_TRY(correct());
        k++;
    }
    if (iters) *iters = k;
    if (rel_res) *rel_res = rr;
    return hh_ctx_synchronize(reinterpret_cast<hh_ctx *>(c)); // kernel-reported failures
}

extern "C" int hh_solve_source(hh_plan *pl, const double *f, double *u, int batch) {
    HH_TRY(check_batch(pl, batch));
    if (batch == 0) return HH_OK;
    if (!f || !u) { set_error("hh_solve_source: null buffer"); return HH_ERR_INVALID; }
    Plan &p = pl->p;
    if (p.src_order == 0) {
        set_error("hh_solve_source needs a plan from hh_plan{2,3}d_create_helmholtz");
        return HH_ERR_INVALID;
    }
    HH_CUDA(cudaSetDevice(p.ctx->device));
    double2 *w = (double2 *)u;
    HH_TRY(stage_mark(*p.ctx, 0));
    HH_TRY(transform_forward(p, (const double2 *)f, w, batch));
    HH_TRY(stage_mark(*p.ctx, 1));
    HH_TRY(launch_line_solve(&p, w, w, batch, p.src_order));
    HH_TRY(stage_mark(*p.ctx, 2));
    HH_TRY(transform_inverse(p, w, batch));
    return stage_mark(*p.ctx, 3);
}

// Several wavenumbers in one solve: plans of one shape (dim, sizes, fused order) on one context,
// plan i taking nrhs[i] consecutive fields of f and u.  The transforms do not depend on k, so each
// direction is one launch over the whole batch; the line solves are one launch with a table of
// which right-hand sides use which plan's factors (or one launch per plan where the plans do not
// share a symmetric kernel variant).  table: device memory for that table (nullptr: the context's
// own, grown on demand, which orders the solve behind earlier work on the context's stream).
int hh::solve_source_multi(Plan *const *plans, const int *nrhs, int nplans, const double2 *f, double2 *u,
                           void *table) {
    Plan &p0 = *plans[0];
    Ctx  *c = p0.ctx;
    int   total = 0;
    for (int i = 0; i < nplans; i++) total += nrhs[i];
    if (total == 0) return HH_OK;
    HH_TRY(stage_mark(*c, 0));
    HH_TRY(transform_forward(p0, f, u, total));
    HH_TRY(stage_mark(*c, 1));
    if (!table) {
        const size_t need = line_solve_multi_table_bytes(nplans, total);
        if (c->multi_tab_bytes < need) {
            HH_CUDA(cudaStreamSynchronize(c->stream));
            cudaFree(c->multi_tab);
            c->multi_tab = nullptr;
            c->multi_tab_bytes = 0;
            HH_CUDA(cudaMalloc(&c->multi_tab, need));
            c->multi_tab_bytes = need;
        }
        table = c->multi_tab;
    }
    int rc = nplans > 1 ? launch_line_solve_multi(plans, nrhs, nplans, u, u, p0.src_order, table) : HH_ERR_UNSUPPORTED;
    if (rc == HH_ERR_UNSUPPORTED) { // one launch per plan
        rc = HH_OK;
        long off = 0;
        for (int i = 0; i < nplans && rc == HH_OK; i++) {
            if (nrhs[i]) rc = launch_line_solve(plans[i], u + off, u + off, nrhs[i], p0.src_order);
            off += p0.field * nrhs[i];
        }
    }
    HH_TRY(rc);
    HH_TRY(stage_mark(*c, 2));
    HH_TRY(transform_inverse(p0, u, total));
    return stage_mark(*c, 3);
}

extern "C" int hh_solve_source_multi(hh_plan *const *plans, const int *nrhs, int nplans, const double *f, double *u) {
    if (!plans || !nrhs || nplans < 1 || !f || !u) {
        set_error("hh_solve_source_multi: invalid arguments");
        return HH_ERR_INVALID;
    }
    long total = 0;
    std::vector<Plan *> ps((size_t)nplans);
    for (int i = 0; i < nplans; i++) {
        if (!plans[i] || nrhs[i] < 0) { set_error("hh_solve_source_multi: plan %d or its count is invalid", i); return HH_ERR_INVALID; }
        ps[(size_t)i] = &plans[i]->p;
        const Plan &a = plans[0]->p, &b = plans[i]->p;
        if (b.src_order == 0 || b.lines_only || b.ctx != a.ctx || b.dim != a.dim || b.nx != a.nx || b.ny != a.ny ||
            b.nz != a.nz || b.src_order != a.src_order) {
            set_error("hh_solve_source_multi: plan %d is not a Helmholtz plan of plan 0's shape and context", i);
            return HH_ERR_INVALID;
        }
        total += nrhs[i];
    }
    if (total > 65535) { set_error("hh_solve_source_multi: %ld right-hand sides", total); return HH_ERR_INVALID; }
    HH_CUDA(cudaSetDevice(ps[0]->ctx->device));
    return solve_source_multi(ps.data(), nrhs, nplans, (const double2 *)f, (double2 *)u, nullptr);
}

extern "C" int hh_rhs2d(hh_plan *pl, const hh_rhs2d_data *d, double *rhs) {
    if (!pl || !d || !rhs || !d->f_ext || pl->p.dim != 2 || (d->order != 2 && d->order != 4 && d->order != 6) ||
        (d->order == 6 && !d->k_ext) || pl->p.nx < 3 || pl->p.ny < 3 || !(d->hx > 0.0) || !(d->hy > 0.0)) {
        set_error("hh_rhs2d: invalid arguments (a 2D plan of at least 3 x 3 points, order 2/4/6, f_ext, k_ext "
                  "for order 6, positive spacings)");
        return HH_ERR_INVALID;
    }
    HH_CUDA(cudaSetDevice(pl->p.ctx->device));
    return assemble_rhs2d(&pl->p, d, (double2 *)rhs);
}

extern "C" int hh_rhs3d(hh_plan *pl, const hh_rhs3d_data *d, double *rhs) {
    if (!pl || !d || !rhs || !d->f_ext || pl->p.dim != 3 || pl->p.lines_only ||
        (d->order != 2 && d->order != 4 && d->order != 6) ||
        (d->order == 6 && !d->k2_ext) || pl->p.nx < 3 || pl->p.ny < 3 || pl->p.nz < 3 || !(d->hx > 0.0) ||
        !(d->hy > 0.0) || !(d->hz > 0.0)) {
        set_error("hh_rhs3d: invalid arguments (a 3D plan of at least 3^3 points, order 2/4/6, f_ext, k2_ext "
                  "for order 6, positive spacings)");
        return HH_ERR_INVALID;
    }
    HH_CUDA(cudaSetDevice(pl->p.ctx->device));
    return assemble_rhs3d(&pl->p, d, (double2 *)rhs);
}

// Host buffers: the batch goes through in chunks so that the host-to-device copy of chunk i+1,
// the solve of chunk i and the device-to-host copy of chunk i-1 overlap (separate copy streams,
// ordered by events).  Host memory should be pinned for the copies to run asynchronously.
static int solve_host_common(hh_plan *pl, const double *in_host, double *out_host, int batch, bool source) {
    HH_TRY(check_batch(pl, batch));
    if (batch == 0) return HH_OK;
    if (!in_host || !out_host) { set_error("host solve: null buffer"); return HH_ERR_INVALID; }
    Plan &p = pl->p;
    Ctx  *c = p.ctx;
    HH_CUDA(cudaSetDevice(c->device));
    hh_ctx    *owner = reinterpret_cast<hh_ctx *>(c); // Ctx is the first member of hh_ctx
    const long need = p.field * batch;
    if (owner->stage_elems < need) {
        HH_CUDA(cudaStreamSynchronize(c->stream));
        cudaFree(owner->stage);
        owner->stage = nullptr;
        owner->stage_elems = 0;
        HH_CUDA(cudaMalloc(&owner->stage, sizeof(double2) * (size_t)need));
        owner->stage_elems = need;
    }
    // chunks of at least 4 MB of field data, at most kMaxChunks: more chunks shorten the
    // pipeline's fill (first copy in) and drain (last copy out)
    constexpr int kMaxChunks = 16;
    int nchunk = (int)std::min<long>(kMaxChunks, std::max<long>(1, (long)(sizeof(double2) * need) / (4L << 20)));
    nchunk = std::min(nchunk, batch);
    if (!c->copy_in) {
        HH_CUDA(cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking));
        HH_CUDA(cudaStreamCreateWithFlags(&c->copy_out, cudaStreamNonBlocking));
    }
    while ((int)c->chunk_ev.size() < 2 * kMaxChunks + 1) {
        cudaEvent_t e;
        HH_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->chunk_ev.push_back(e);
    }
    // copies start after the work already queued on the context stream
    HH_CUDA(cudaEventRecord(c->chunk_ev[2 * kMaxChunks], c->stream));
    HH_CUDA(cudaStreamWaitEvent(c->copy_in, c->chunk_ev[2 * kMaxChunks], 0));
    const int per = (batch + nchunk - 1) / nchunk;
    for (int i = 0, b0 = 0; b0 < batch; i++, b0 += per) {
        const int    nb = std::min(per, batch - b0);
        const size_t off = (size_t)p.field * b0, bytes = sizeof(double2) * (size_t)p.field * nb;
        double2     *d = owner->stage + off;
        HH_CUDA(cudaMemcpyAsync(d, in_host + 2 * off, bytes, cudaMemcpyHostToDevice, c->copy_in));
        HH_CUDA(cudaEventRecord(c->chunk_ev[2 * i], c->copy_in));
        HH_CUDA(cudaStreamWaitEvent(c->stream, c->chunk_ev[2 * i], 0));
        HH_TRY(source ? hh_solve_source(pl, (const double *)d, (double *)d, nb)
                      : hh_solve(pl, (const double *)d, (double *)d, nb));
        HH_CUDA(cudaEventRecord(c->chunk_ev[2 * i + 1], c->stream));
        HH_CUDA(cudaStreamWaitEvent(c->copy_out, c->chunk_ev[2 * i + 1], 0));
        HH_CUDA(cudaMemcpyAsync(out_host + 2 * off, d, bytes, cudaMemcpyDeviceToHost, c->copy_out));
    }
    // the context stream sees the copies complete before anything queued after this call
    HH_CUDA(cudaEventRecord(c->chunk_ev[2 * kMaxChunks], c->copy_out));
    HH_CUDA(cudaStreamWaitEvent(c->stream, c->chunk_ev[2 * kMaxChunks], 0));
    return hh_ctx_synchronize(owner);
}

extern "C" int hh_solve_host(hh_plan *pl, const double *rhs, double *sol, int batch) {
    return solve_host_common(pl, rhs, sol, batch, false);
}
extern "C" int hh_solve_source_host(hh_plan *pl, const double *f, double *u, int batch) {
    return solve_host_common(pl, f, u, batch, true);
}

// ------------------------------------------------------ allocation-free host solve ------

extern "C" int hh_solve_source_host_noalloc(hh_plan *pl, const double *f_host, double *u_host, int batch) {
    HH_TRY(check_batch(pl, batch));
    if (batch == 0) return HH_OK;
    if (!f_host || !u_host) { set_error("hh_solve_source_host_noalloc: null buffer"); return HH_ERR_INVALID; }
    Plan &p = pl->p;
    if (p.src_order == 0) {
        set_error("hh_solve_source_host_noalloc needs a plan from hh_plan{2,3}d_create_helmholtz");
        return HH_ERR_INVALID;
    }
    if (p.field * (long)batch > kNoAllocElems) {
        set_error("hh_solve_source_host_noalloc: %ld complex values exceed the %ld-value staging area",
                  p.field * (long)batch, kNoAllocElems);
        return HH_ERR_UNSUPPORTED;
    }
    Ctx *c = p.ctx;
    HH_CUDA(cudaSetDevice(c->device));
    // the array's address on this device, looked up when the context was created
    double2 *d = reinterpret_cast<hh_ctx *>(c)->noalloc_stage; // Ctx is the first member of hh_ctx
    const size_t bytes = sizeof(double2) * (size_t)p.field * batch;
    HH_CUDA(cudaMemcpyAsync(d, f_host, bytes, cudaMemcpyHostToDevice, c->stream));
    HH_TRY(hh_solve_source(pl, (const double *)d, (double *)d, batch));
    HH_CUDA(cudaMemcpyAsync(u_host, d, bytes, cudaMemcpyDeviceToHost, c->stream));
    return hh_ctx_synchronize(reinterpret_cast<hh_ctx *>(c)); // Ctx is the first member of hh_ctx
}
