// The reference's right-hand-side assembly rhs() on the device, for plans of any stencil
// (variable k, Dirichlet data): 2D_Program/main_functions/rhs.c:4-150 and
// 3D_Program/main_functions/rhs.c:13-194 with the compact derivatives of
// 2D_Program/partial_derivatives/*.c and 3D_Program/partial_derivatives/*.c.
//
// The Helmholtz plans apply the constant-k operator in the mode basis inside the line solve
// (hh_tridiag.cu); this file is the general form, used where k varies along the line direction
// or the boundary data is not zero.  Its pieces:
//  * Pade derivatives: each line of the extended grid along one axis gets its compact
//    right-hand side (12 (f_- - 2 f_0 + f_+) / h^2 for [1 10 1], 3 (f_+ - f_-) / h for [1 4 1]),
//    the boundary values subtracted at its two ends, and the Thomas recurrence of
//    tridiag(1, diag, 1) with the reference's factors (L_j = 1/U_{j-1}, U_j = diag - L_j,
//    division by U_j) -- one thread per line, sequential along it;
//  * the pointwise combination of rhs.c (2D :78-86, 3D :149-166) with the second-order
//    differences of 2nd_order*.c inline;
//  * the Dirichlet corrections of the edges (2D rhs.c:126-148) or z faces (3D rhs.c:167-174).
// Arithmetic follows the reference's expression order (complex throughout: where the reference's
// 3D rhs.c:149 keeps its partial sums in real doubles, here they stay complex; the two agree for
// real data, which is what the reference's own problems have).
#include "hh_internal.cuh"

#include <string.h>

#include <algorithm>
#include <vector>

namespace hh {

namespace {

// lines along one axis of the extended grid: line t has interior cross coordinates
// c1 = t % n1 + 1, c2 = t / n1 + 1; its point m (0..n-1) is at c1 s1 + c2 s2 + (m + 1) sa
struct AxisLines {
    int  n, n1;
    long nlines;
    long s1, s2, sa;
    long b2;    // boundary-array stride of the second cross coordinate (the first has stride 1)
    int  bsh;   // added to c1 when indexing the boundary array (fy_yb is indexed by interior x)
    long bface; // offset of the far end's boundary values
};

__global__ void k_pade_lines(const double2 *__restrict__ f, double2 *__restrict__ out, AxisLines g, int first,
                             int plus_first, double h, const double2 *__restrict__ bc, const double *__restrict__ Lf,
                             const double *__restrict__ Uf) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= g.nlines) return;
    const long c1 = t % g.n1 + 1, c2 = t / g.n1 + 1;
    const long base = c1 * g.s1 + c2 * g.s2;
    const int  n = g.n;
    for (int m = 0; m < n; m++) {
        const long    e = base + (long)(m + 1) * g.sa;
        const double2 lo = f[e - g.sa], c = f[e], hi = f[e + g.sa];
        double2       v;
        if (first) {
            v = make_double2(3.0 * (hi.x - lo.x) / h, 3.0 * (hi.y - lo.y) / h);
        } else if (plus_first) { // 12 (f_+ - 2 f_0 + f_-) / h / h
            v = make_double2(12.0 * (hi.x - 2.0 * c.x + lo.x) / h / h, 12.0 * (hi.y - 2.0 * c.y + lo.y) / h / h);
        } else { // 12 (f_- - 2 f_0 + f_+) / h / h
            v = make_double2(12.0 * (lo.x - 2.0 * c.x + hi.x) / h / h, 12.0 * (lo.y - 2.0 * c.y + hi.y) / h / h);
        }
        if (bc && (m == 0 || m == n - 1)) {
            const long    bi = c1 + g.bsh + c2 * g.b2 + (m == 0 ? 0 : g.bface);
            const double2 b = bc[bi];
            v = make_double2(v.x - b.x, v.y - b.y);
            if (n == 1) { // a one-point line subtracts both ends
                const double2 b1 = bc[c1 + g.bsh + c2 * g.b2 + g.bface];
                v = make_double2(v.x - b1.x, v.y - b1.y);
            }
        }
        out[e] = v;
    }
    // tridiag(1, diag, 1): v_m -= L_m v_{m-1};  v_{n-1} /= U_{n-1};  v_m = (v_m - v_{m+1}) / U_m
    double2 prev = out[base + g.sa];
    for (int m = 1; m < n; m++) {
        const long e = base + (long)(m + 1) * g.sa;
        double2    v = out[e];
        v = make_double2(v.x - Lf[m] * prev.x, v.y - Lf[m] * prev.y);
        out[e] = v;
        prev = v;
    }
    {
        const long e = base + (long)n * g.sa;
        const double2 v = out[e];
        prev = make_double2(v.x / Uf[n - 1], v.y / Uf[n - 1]);
        out[e] = prev;
    }
    for (int m = n - 2; m >= 0; m--) {
        const long e = base + (long)(m + 1) * g.sa;
        const double2 v = out[e];
        prev = make_double2((v.x - prev.x) / Uf[m], (v.y - prev.y) / Uf[m]);
        out[e] = prev;
    }
}

// values of an extended-grid array on two opposite faces: face value (c1, c2) of the near face
// (index c1 + c2 * b2 of src) at c1 s1 + c2 s2 (+ far * sa), for c1 < n1, c2 < n2
__global__ void k_fill_faces(double2 *__restrict__ dst, const double2 *__restrict__ src, int n1, int n2, long s1,
                             long s2, long far_off, long b2, long bface) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)n1 * n2) return;
    const long c1 = t % n1, c2 = t / n1;
    const double2 z = make_double2(0.0, 0.0);
    dst[c1 * s1 + c2 * s2] = src ? src[c1 + c2 * b2] : z;
    dst[c1 * s1 + c2 * s2 + far_off] = src ? src[c1 + c2 * b2 + bface] : z;
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 rmul(double a, double2 b) { return make_double2(a * b.x, a * b.y); }
__device__ __forceinline__ double2 rdiv(double2 a, double b) { return make_double2(a.x / b, a.y / b); }
// (a - 2 b + c) / h / h
__device__ __forceinline__ double2 d2h(double2 a, double2 b, double2 c, double h) {
    return make_double2((a.x - 2.0 * b.x + c.x) / h / h, (a.y - 2.0 * b.y + c.y) / h / h);
}

// 2D combination, rhs.c:78-86 (order 6); orders 4 and 2, rhs.c:4-38
__global__ void k_rhs2d_combine(int nx, int ny, int order, double hx, double hy, const double2 *__restrict__ fe,
                                const double2 *__restrict__ fxx, const double2 *__restrict__ fyy,
                                const double2 *__restrict__ fy, const double2 *__restrict__ k2c,
                                const double2 *__restrict__ k2y, double2 *__restrict__ rhs) {
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= (long)nx * ny) return;
    const int  i = (int)(q % nx), j = (int)(q / nx);
    const long E = nx + 2;
    const long c = (i + 1) + (long)(j + 1) * E;
    const double hy2 = hy * hy;
    if (order == 6) {
        const double  hy4 = hy2 * hy2, hx2 = hx * hx, hyy = hy * hy;
        const double2 fxxxx = rdiv(zadd(zsub(fxx[c - 1], rmul(2.0, fxx[c])), fxx[c + 1]), hx2);
        const double2 fxxyy = rdiv(zadd(zsub(fxx[c - E], rmul(2.0, fxx[c])), fxx[c + E]), hyy);
        const double2 fyyyy = rdiv(zadd(zsub(fyy[c - E], rmul(2.0, fyy[c])), fyy[c + E]), hyy);
        const double2 k2 = k2c[j];
        const double2 t1 = zmul(make_double2(1.0 - k2.x * hy2 / 20.0, -(k2.y * hy2 / 20.0)), fe[c]);
        const double2 t2 = rdiv(rmul(hy2, zadd(fxx[c], fyy[c])), 12.0);
        const double2 t3 = rdiv(rmul(hy4, zadd(fxxxx, fyyyy)), 360.0);
        const double2 t4 = rdiv(rmul(hy4, fxxyy), 90.0);
        const double2 t5 = rdiv(zmul(rmul(hy4, k2y[j]), fy[c]), 60.0);
        rhs[q] = rmul(hy2, zadd(zadd(zadd(zadd(t1, t2), t3), t4), t5));
    } else if (order == 4) {
        const double  a = 2.0 / 3.0, b = 1.0 / 12.0;
        const double2 s = zadd(zadd(zadd(fe[c - E], fe[c + E]), fe[c - 1]), fe[c + 1]);
        rhs[q] = rmul(hy2, zadd(rmul(a, fe[c]), rmul(b, s)));
    } else {
        rhs[q] = rmul(hy * hy, fe[c]);
    }
}

// 2D Dirichlet corrections of the edges and corners, rhs.c:126-148.  t[] are the plan's row
// tables [4][prow]: sub (bm at [1], am at [3]), diag (b at [1]), super (bp at [1], ap at [3]).
__global__ void k_rhs2d_dirichlet(int nx, int ny, int prow, const double2 *__restrict__ subt,
                                  const double2 *__restrict__ diagt, const double2 *__restrict__ supt,
                                  const double *__restrict__ ux, const double *__restrict__ uy, double2 *__restrict__ rhs) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    auto U = [&](const double *a, long i) { return a ? a[i] : 0.0; };
    auto bm = [&](int j) { return subt[prow + j]; };
    auto am = [&](int j) { return subt[3 * prow + j]; };
    auto b = [&](int j) { return diagt[prow + j]; };
    auto bp = [&](int j) { return supt[prow + j]; };
    auto ap = [&](int j) { return supt[3 * prow + j]; };
    auto sub = [&](long q, double2 co, double u) { rhs[q] = make_double2(rhs[q].x - co.x * u, rhs[q].y - co.y * u); };
    const long xb1 = ny + 2, yb1 = nx + 2, top = (long)(ny - 1) * nx;
    if (t == 0) {
        sub(0, bm(0), U(uy, 0)); sub(0, am(0), U(uy, 1)); sub(0, bm(0), U(uy, 2));
        sub(0, b(0), U(ux, 1)); sub(0, bp(0), U(ux, 2));
        const long r = nx - 1;
        sub(r, bm(0), U(uy, nx - 1)); sub(r, am(0), U(uy, nx)); sub(r, bm(0), U(uy, nx + 1));
        sub(r, b(0), U(ux, xb1 + 1)); sub(r, bp(0), U(ux, xb1 + 2));
        const int J = ny - 1;
        sub(top, bm(J), U(ux, ny - 1)); sub(top, b(J), U(ux, ny));
        sub(top, bp(J), U(uy, yb1 + 0)); sub(top, ap(J), U(uy, yb1 + 1)); sub(top, bp(J), U(uy, yb1 + 2));
        const long tr = nx - 1 + top;
        sub(tr, bm(J), U(ux, xb1 + ny - 1)); sub(tr, b(J), U(ux, xb1 + ny));
        sub(tr, bp(J), U(uy, yb1 + nx + 1)); sub(tr, ap(J), U(uy, yb1 + nx)); sub(tr, bp(J), U(uy, yb1 + nx - 1));
    } else if (t - 1 < ny - 2) {
        const int  j = (int)(t - 1) + 1;
        const long my = (long)j * nx;
        sub(my, b(j), U(ux, j + 1)); sub(my, bm(j), U(ux, j)); sub(my, bp(j), U(ux, j + 2));
        const long r = my + nx - 1;
        sub(r, b(j), U(ux, xb1 + j + 1)); sub(r, bm(j), U(ux, xb1 + j)); sub(r, bp(j), U(ux, xb1 + j + 2));
    } else if (t - 1 - (ny - 2) < nx - 2) {
        const int i = (int)(t - 1 - (ny - 2)) + 1;
        sub(i, am(0), U(uy, i + 1)); sub(i, bm(0), U(uy, i)); sub(i, bm(0), U(uy, i + 2));
        const long r = i + top;
        const int  J = ny - 1;
        sub(r, ap(J), U(uy, yb1 + i + 1)); sub(r, bp(J), U(uy, yb1 + i)); sub(r, bp(J), U(uy, yb1 + i + 2));
    }
}

// 3D combination, rhs.c:149-166 (order 6); orders 4 and 2, rhs.c:13-62
__global__ void k_rhs3d_combine(int nx, int ny, int nz, int order, double hx, double hy, double hz,
                                const double2 *__restrict__ f, const double2 *__restrict__ fxx,
                                const double2 *__restrict__ fyy, const double2 *__restrict__ fzz,
                                const double2 *__restrict__ k2_ext, const double2 *__restrict__ kp,
                                double2 *__restrict__ rhs) {
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nxy = (long)nx * ny;
    if (q >= nxy * nz) return;
    const int  i = (int)(q % nx), j = (int)((q / nx) % ny), l = (int)(q / nxy);
    const long Ex = nx + 2, Exy = (long)(nx + 2) * (ny + 2);
    const long C = (i + 1) + (j + 1) * Ex + (l + 1) * Exy;
    const long W = C - 1, E = C + 1, S = C - Ex, N = C + Ex, D = C - Exy, Up = C + Exy;
    if (order == 6) {
        const double2 fxxxx = d2h(fxx[W], fxx[C], fxx[E], hx), fyyyy = d2h(fyy[S], fyy[C], fyy[N], hy);
        const double2 fzzzz = d2h(fzz[D], fzz[C], fzz[Up], hz), fxxyy = d2h(fxx[S], fxx[C], fxx[N], hy);
        const double2 fxxzz = d2h(fxx[D], fxx[C], fxx[Up], hz), fyyzz = d2h(fyy[D], fyy[C], fyy[Up], hz);
        const double2 k2 = k2_ext[l + 1];
        const double2 first = zmul(make_double2(1.0 - k2.x * hz * hz / 20.0, -(k2.y * hz * hz / 20.0)), f[C]);
        const double2 second = rmul(hz * hz / 12.0, zadd(zadd(fxx[C], fyy[C]), fzz[C]));
        const double2 third = rmul(hz * hz * hz * hz / 360.0, zadd(zadd(fxxxx, fyyyy), fzzzz));
        const double2 fourth = rmul(hz * hz * hz * hz / 90.0, zadd(zadd(fxxyy, fxxzz), fyyzz));
        const double2 fifth = zmul(rmul(hz * hz * hz / 120.0, kp[l]), zsub(f[Up], f[D]));
        rhs[q] = zadd(zadd(zadd(zadd(first, second), third), fourth), fifth);
    } else if (order == 4) {
        const double2 nb = zadd(zadd(zadd(zadd(zadd(f[W], f[E]), f[S]), f[N]), f[D]), f[Up]);
        rhs[q] = zadd(f[C], rmul(1.0 / 12.0, zsub(nb, rmul(6.0, f[C]))));
    } else {
        rhs[q] = f[C];
    }
}

// 3D z-face Dirichlet terms, rhs.c:24-29, 55-62, 167-174: layer 0 with the sub-diagonal layer's
// stencil (am, bm, cm, dm of layer 0), layer nz-1 with the super-diagonal one (ap..dp of nz-1)
__global__ void k_rhs3d_zfaces(int nx, int ny, int nz, int order, int prow, const double2 *__restrict__ subt,
                               const double2 *__restrict__ supt, const double2 *__restrict__ ue,
                               double2 *__restrict__ rhs) {
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= (long)nx * ny) return;
    const int  i = (int)(t % nx), j = (int)(t / nx);
    const long Ex = nx + 2, Exy = (long)(nx + 2) * (ny + 2), nxy = (long)nx * ny;
    const long b = t, top = t + (long)(nz - 1) * nxy;
    auto X = [&](int ie, int je, long le) { return ue[ie + je * Ex + le * Exy]; };
    if (order == 2) {
        rhs[b] = zsub(rhs[b], X(i + 1, j + 1, 0));
        rhs[top] = zsub(rhs[top], X(i + 1, j + 1, nz + 1));
        return;
    }
    for (int face = 0; face < 2; face++) {
        const long   le = face ? nz + 1 : 0, q = face ? top : b;
        const double2 *tab = face ? supt : subt;
        const int      row = face ? nz - 1 : 0;
        const double2  a = tab[row], bb = tab[prow + row], cc = tab[2 * prow + row], dd = tab[3 * prow + row];
        double2 r = rhs[q];
        r = zsub(r, zmul(a, zadd(zadd(zadd(X(i, j, le), X(i + 2, j, le)), X(i, j + 2, le)), X(i + 2, j + 2, le))));
        r = zsub(r, zmul(bb, zadd(X(i, j + 1, le), X(i + 2, j + 1, le))));
        r = zsub(r, zmul(cc, zadd(X(i + 1, j, le), X(i + 1, j + 2, le))));
        r = zsub(r, zmul(dd, X(i + 1, j + 1, le)));
        rhs[q] = r;
    }
}

// Pade factors of tridiag(1, diag, 1) over n points, as the reference forms them
void pade_factors(int n, double diag, std::vector<double> &L, std::vector<double> &U) {
    L.assign((size_t)n, 0.0);
    U.assign((size_t)n, 0.0);
    U[0] = diag;
    for (int j = 1; j < n; j++) {
        L[(size_t)j] = 1.0 / U[(size_t)j - 1];
        U[(size_t)j] = diag - L[(size_t)j];
    }
}

// complex line of the reference's Pade recurrence on the host (the O(n) k profiles)
void pade_host(std::vector<double2> &v, double diag) {
    const int           n = (int)v.size();
    std::vector<double> L, U;
    pade_factors(n, diag, L, U);
    for (int j = 1; j < n; j++) v[j] = make_double2(v[j].x - L[j] * v[j - 1].x, v[j].y - L[j] * v[j - 1].y);
    v[n - 1] = make_double2(v[n - 1].x / U[n - 1], v[n - 1].y / U[n - 1]);
    for (int j = n - 2; j >= 0; j--) v[j] = make_double2((v[j].x - v[j + 1].x) / U[j], (v[j].y - v[j + 1].y) / U[j]);
}

double2 hmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

} // namespace

// Workspace of the assembly: `count` complex values, grown on demand (outside stream capture).
static int rhs_work(Ctx *c, long count, double2 **out) {
    if (c->rhs_elems < count) {
        HH_CUDA(cudaStreamSynchronize(c->stream));
        cudaFree(c->rhs_work);
        c->rhs_work = nullptr;
        c->rhs_elems = 0;
        HH_CUDA(cudaMalloc(&c->rhs_work, sizeof(double2) * (size_t)count));
        c->rhs_elems = count;
    }
    *out = c->rhs_work;
    return HH_OK;
}

// a small host table on the device, in the context's table area (stream-ordered upload)
struct TableArea {
    Ctx               *c;
    std::vector<char>  host;
    std::vector<size_t> offs;
    size_t add(const void *p, size_t bytes) {
        const size_t off = (host.size() + 255) / 256 * 256;
        host.resize(off + bytes);
        memcpy(host.data() + off, p, bytes);
        offs.push_back(off);
        return off;
    }
};

static int upload_tables(Ctx *c, TableArea &ta, char **dev) {
    if (c->rhs_tab_bytes < ta.host.size()) {
        HH_CUDA(cudaStreamSynchronize(c->stream));
        cudaFree(c->rhs_tab);
        c->rhs_tab = nullptr;
        c->rhs_tab_bytes = 0;
        HH_CUDA(cudaMalloc(&c->rhs_tab, ta.host.size()));
        c->rhs_tab_bytes = ta.host.size();
    }
    HH_CUDA(cudaMemcpyAsync(c->rhs_tab, ta.host.data(), ta.host.size(), cudaMemcpyHostToDevice, c->stream));
    // the upload reads pageable host memory the caller is about to free: wait for it
    HH_CUDA(cudaStreamSynchronize(c->stream));
    *dev = static_cast<char *>(c->rhs_tab);
    return HH_OK;
}

static unsigned blocks_for(long n, int nt) { return (unsigned)std::max<long>(1, (n + nt - 1) / nt); }

int assemble_rhs2d(Plan *p, const hh_rhs2d_data *d, double2 *rhs) {
    Ctx      *c = p->ctx;
    const int nx = p->nx, ny = p->ny, order = d->order;
    const long E = nx + 2, next = E * (ny + 2);
    const double2 *fe = (const double2 *)d->f_ext;
    if (order == 6) {
        double2 *w;
        HH_TRY(rhs_work(c, 3 * next, &w));
        double2 *fxx = w, *fyy = w + next, *fy = w + 2 * next;
        HH_CUDA(cudaMemsetAsync(w, 0, sizeof(double2) * 3 * (size_t)next, c->stream));
        // host: the k profiles (O(ny)) and the Pade factors
        std::vector<double2> k2c((size_t)ny), k2y((size_t)ny);
        const double2       *ke = (const double2 *)d->k_ext;
        for (int j = 0; j < ny; j++) {
            k2c[(size_t)j] = hmul(ke[j + 1], ke[j + 1]);
            const double2 kp2 = hmul(ke[j + 2], ke[j + 2]), km2 = hmul(ke[j], ke[j]);
            k2y[(size_t)j] = make_double2(3.0 * (kp2.x - km2.x) / d->hy, 3.0 * (kp2.y - km2.y) / d->hy);
        }
        if (d->k2y_bc) {
            const double2 *bc = (const double2 *)d->k2y_bc;
            k2y[0] = make_double2(k2y[0].x - bc[0].x, k2y[0].y - bc[0].y);
            k2y[(size_t)ny - 1] = make_double2(k2y[(size_t)ny - 1].x - bc[1].x, k2y[(size_t)ny - 1].y - bc[1].y);
        }
        pade_host(k2y, 4.0);
        std::vector<double> L4y, U4y, L10y, U10y, L10x, U10x;
        pade_factors(ny, 4.0, L4y, U4y);
        pade_factors(ny, 10.0, L10y, U10y);
        pade_factors(nx, 10.0, L10x, U10x);
        TableArea ta{c, {}, {}};
        const size_t o_k2c = ta.add(k2c.data(), 16 * k2c.size()), o_k2y = ta.add(k2y.data(), 16 * k2y.size());
        const size_t o_l4 = ta.add(L4y.data(), 8 * L4y.size()), o_u4 = ta.add(U4y.data(), 8 * U4y.size());
        const size_t o_l10y = ta.add(L10y.data(), 8 * L10y.size()), o_u10y = ta.add(U10y.data(), 8 * U10y.size());
        const size_t o_l10x = ta.add(L10x.data(), 8 * L10x.size()), o_u10x = ta.add(U10x.data(), 8 * U10x.size());
        char *tab;
        HH_TRY(upload_tables(c, ta, &tab));
        auto T = [&](size_t off) { return reinterpret_cast<const double *>(tab + off); };
        const int nt = 128;
        // f_y: [1 4 1] along y (4th_order_first_derivative.c:60-98), boundary values fy_yb (interior x)
        {
            AxisLines g{ny, nx, (long)nx, 1, 0, E, 0, -1, (long)nx};
            k_pade_lines<<<blocks_for(nx, nt), nt, 0, c->stream>>>(fe, fy, g, 1, 0, d->hy, (const double2 *)d->fy_yb, T(o_l4),
                                                                   T(o_u4));
        }
        // f_yy: [1 10 1] along y (4th_order_second_derivative.c:61-120), then its edge values
        {
            AxisLines g{ny, nx, (long)nx, 1, 0, E, 0, 0, E};
            k_pade_lines<<<blocks_for(nx, nt), nt, 0, c->stream>>>(fe, fyy, g, 0, 1, d->hy, (const double2 *)d->fyy_yb,
                                                                   T(o_l10y), T(o_u10y));
            k_fill_faces<<<blocks_for(E, nt), nt, 0, c->stream>>>(fyy, (const double2 *)d->fyy_yb, (int)E, 1, 1, 0,
                                                                  (long)(ny + 1) * E, 0, E);
            k_fill_faces<<<blocks_for(ny + 2, nt), nt, 0, c->stream>>>(fyy, (const double2 *)d->fyy_xb, ny + 2, 1, E, 0,
                                                                       nx + 1, 0, ny + 2);
        }
        // f_xx: [1 10 1] along x (4th_order_second_derivative.c:4-59), then its edge values
        {
            AxisLines g{nx, ny, (long)ny, E, 0, 1, 0, 0, ny + 2};
            k_pade_lines<<<blocks_for(ny, nt), nt, 0, c->stream>>>(fe, fxx, g, 0, 1, d->hx, (const double2 *)d->fxx_xb,
                                                                   T(o_l10x), T(o_u10x));
            k_fill_faces<<<blocks_for(E, nt), nt, 0, c->stream>>>(fxx, (const double2 *)d->fxx_yb, (int)E, 1, 1, 0,
                                                                  (long)(ny + 1) * E, 0, E);
            k_fill_faces<<<blocks_for(ny + 2, nt), nt, 0, c->stream>>>(fxx, (const double2 *)d->fxx_xb, ny + 2, 1, E, 0,
                                                                       nx + 1, 0, ny + 2);
        }
        k_rhs2d_combine<<<blocks_for((long)nx * ny, 256), 256, 0, c->stream>>>(
            nx, ny, 6, d->hx, d->hy, fe, fxx, fyy, fy, reinterpret_cast<const double2 *>(tab + o_k2c),
            reinterpret_cast<const double2 *>(tab + o_k2y), rhs);
        c->launches += 8;
    } else {
        k_rhs2d_combine<<<blocks_for((long)nx * ny, 256), 256, 0, c->stream>>>(nx, ny, order, d->hx, d->hy, fe, nullptr,
                                                                              nullptr, nullptr, nullptr, nullptr, rhs);
        c->launches++;
    }
    HH_CUDA(cudaGetLastError());
    if (d->u_xb || d->u_yb) {
        k_rhs2d_dirichlet<<<blocks_for(1 + (ny - 2) + (nx - 2), 128), 128, 0, c->stream>>>(
            nx, ny, p->prow, p->subt, p->diagt, p->rowc, d->u_xb, d->u_yb, rhs);
        HH_CUDA(cudaGetLastError());
        c->launches++;
    }
    return HH_OK;
}

int assemble_rhs3d(Plan *p, const hh_rhs3d_data *d, double2 *rhs) {
    Ctx       *c = p->ctx;
    const int  nx = p->nx, ny = p->ny, nz = p->nz, order = d->order;
    const long Ex = nx + 2, Ey = ny + 2, Exy = Ex * Ey, next = Exy * (nz + 2);
    const double2 *f = (const double2 *)d->f_ext;
    const int  nt = 128;
    if (order == 6) {
        double2 *w;
        HH_TRY(rhs_work(c, 3 * next, &w));
        double2 *fxx = w, *fyy = w + next, *fzz = w + 2 * next;
        HH_CUDA(cudaMemsetAsync(w, 0, sizeof(double2) * 3 * (size_t)next, c->stream));
        // host: d(k^2)/dz by the [1 4 1] scheme (4th_order_partials.c:296-340), Pade factors
        const double2       *k2 = (const double2 *)d->k2_ext;
        std::vector<double2> kp((size_t)nz);
        for (int l = 0; l < nz; l++)
            kp[(size_t)l] = make_double2(3.0 * (k2[l + 2].x - k2[l].x) / d->hz, 3.0 * (k2[l + 2].y - k2[l].y) / d->hz);
        if (d->kz_bc) {
            const double2 *bc = (const double2 *)d->kz_bc;
            kp[0] = make_double2(kp[0].x + bc[0].x, kp[0].y + bc[0].y);
            kp[(size_t)nz - 1] = make_double2(kp[(size_t)nz - 1].x + bc[1].x, kp[(size_t)nz - 1].y + bc[1].y);
        }
        pade_host(kp, 4.0);
        std::vector<double> Lx, Ux, Ly, Uy, Lz, Uz;
        pade_factors(nx, 10.0, Lx, Ux);
        pade_factors(ny, 10.0, Ly, Uy);
        pade_factors(nz, 10.0, Lz, Uz);
        TableArea ta{c, {}, {}};
        const size_t o_kp = ta.add(kp.data(), 16 * kp.size()), o_k2 = ta.add(k2, 16 * (size_t)(nz + 2));
        const size_t o_lx = ta.add(Lx.data(), 8 * Lx.size()), o_ux = ta.add(Ux.data(), 8 * Ux.size());
        const size_t o_ly = ta.add(Ly.data(), 8 * Ly.size()), o_uy = ta.add(Uy.data(), 8 * Uy.size());
        const size_t o_lz = ta.add(Lz.data(), 8 * Lz.size()), o_uz = ta.add(Uz.data(), 8 * Uz.size());
        char *tab;
        HH_TRY(upload_tables(c, ta, &tab));
        auto T = [&](size_t off) { return reinterpret_cast<const double *>(tab + off); };
        // f_xx along x (4th_order_partials.c:94-160): lines (j, l), boundary layout j + l (ny+2)
        {
            AxisLines g{nx, ny, (long)ny * nz, Ex, Exy, 1, Ey, 0, Ey * (nz + 2)};
            k_pade_lines<<<blocks_for(g.nlines, nt), nt, 0, c->stream>>>(f, fxx, g, 0, 0, d->hx, (const double2 *)d->fxx_b,
                                                                         T(o_lx), T(o_ux));
            k_fill_faces<<<blocks_for(Ey * (nz + 2), nt), nt, 0, c->stream>>>(fxx, (const double2 *)d->fxx_b, (int)Ey, nz + 2,
                                                                              Ex, Exy, nx + 1, Ey, Ey * (nz + 2));
        }
        // f_yy along y (:162-227): lines (i, l), boundary layout i + l (nx+2)
        {
            AxisLines g{ny, nx, (long)nx * nz, 1, Exy, Ex, Ex, 0, Ex * (nz + 2)};
            k_pade_lines<<<blocks_for(g.nlines, nt), nt, 0, c->stream>>>(f, fyy, g, 0, 0, d->hy, (const double2 *)d->fyy_b,
                                                                         T(o_ly), T(o_uy));
            k_fill_faces<<<blocks_for(Ex * (nz + 2), nt), nt, 0, c->stream>>>(fyy, (const double2 *)d->fyy_b, (int)Ex, nz + 2,
                                                                              1, Exy, (long)(ny + 1) * Ex, Ex, Ex * (nz + 2));
        }
        // f_zz along z (:229-294): lines (i, j), boundary layout i + j (nx+2)
        {
            AxisLines g{nz, nx, (long)nx * ny, 1, Ex, Exy, Ex, 0, Exy};
            k_pade_lines<<<blocks_for(g.nlines, nt), nt, 0, c->stream>>>(f, fzz, g, 0, 0, d->hz, (const double2 *)d->fzz_b,
                                                                         T(o_lz), T(o_uz));
            k_fill_faces<<<blocks_for(Exy, nt), nt, 0, c->stream>>>(fzz, (const double2 *)d->fzz_b, (int)Ex, (int)Ey, 1, Ex,
                                                                    (long)(nz + 1) * Exy, Ex, Exy);
        }
        k_rhs3d_combine<<<blocks_for((long)nx * ny * nz, 256), 256, 0, c->stream>>>(
            nx, ny, nz, 6, d->hx, d->hy, d->hz, f, fxx, fyy, fzz, reinterpret_cast<const double2 *>(tab + o_k2),
            reinterpret_cast<const double2 *>(tab + o_kp), rhs);
        c->launches += 7;
    } else {
        k_rhs3d_combine<<<blocks_for((long)nx * ny * nz, 256), 256, 0, c->stream>>>(
            nx, ny, nz, order, d->hx, d->hy, d->hz, f, nullptr, nullptr, nullptr, nullptr, nullptr, rhs);
        c->launches++;
    }
    HH_CUDA(cudaGetLastError());
    if (d->ue_ext) {
        k_rhs3d_zfaces<<<blocks_for((long)nx * ny, 128), 128, 0, c->stream>>>(nx, ny, nz, order, p->prow, p->subt, p->rowc,
                                                                             (const double2 *)d->ue_ext, rhs);
        HH_CUDA(cudaGetLastError());
        c->launches++;
    }
    return HH_OK;
}

} // namespace hh
