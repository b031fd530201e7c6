// Shifted tridiagonal line solves for sm_100a (FP64 complex).
//
// Replaces the reference's per-mode Thomas solves: 2D_Program/solver_functions/solver.c:71-86
// (per x-mode i along y, factors from main_functions/LU.c:3-46) and
// 3D_Program/solver_functions/solver.c:483-496 / cuda_kernels.cu:208-249 (per (i,j) along z,
// factors from main_functions/LU.c:4-81).
//
// Geometry.  A right-hand side holds `lines` independent lines of `rows` points; point
// (row r, line q) sits at offset r*row_stride + q.  2D: line = x-mode i, row = y index j,
// row_stride = Nx (the DST output layout, no transpose).  3D: line = i + j*Nx, row = z
// layer l, row_stride = Nx*Ny.  Consecutive lines are contiguous, so a warp always reads
// whole row segments (the "interleaved" layout).
//
// Line matrix (row r, line q), with per-row coefficient tables and per-line multipliers mu:
//   sub(r,q)   = subc0[r] mu0[q] + subc1[r] mu1[q] + subc2[r] mu2[q] + subc3[r]
//   diag(r,q)  = same with diagc,   super(r,q) = same with supc
// 2D: mu = (0, lambda_i, 0):   sub = bm lambda + am, diag = b lambda + a, super = bp lambda + ap
// 3D: mu = (lx*ly, lx, ly):    sub = am lx ly + bm lx + cm ly + dm, etc.
// This is the reference's eigenvalue shift (2D LU.c:16-23, 3D LU.c:35-47) evaluated on the fly.
//
// Factorisation (set-up, once per plan): Thomas without pivoting, exactly the reference's
// recurrence  L_0 = 0, P_0 = diag_0,  L_r = sub_r / P_{r-1},  P_r = diag_r - L_r super_{r-1};
// the device keeps L_r and 1/P_r in [row][line] layout.
//
// Solve (per right-hand side): each thread owns a segment of MSEG consecutive rows of one line
// in registers.  Forward substitution y_r = f_r - L_r y_{r-1} and back substitution
// x_r = y_r/P_r - (super_r/P_r) x_{r+1} are first-order linear recurrences; each segment
// applies its rows as an affine map of the value entering it, the maps are composed across the
// segments of a line by a Kogge-Stone scan in shared memory, and every segment then re-runs its
// rows from the exact entering value.  All values stay on chip: one HBM read and one HBM write
// per point.
//
// Fused right-hand-side operator (plans for the constant-k, homogeneous-Dirichlet class).  The
// compact RHS of 2D_Program/main_functions/rhs.c:4-97 and 3D_Program/main_functions/rhs.c:13-166
// is a polynomial in the 1D second-difference and Pade operators of each direction.  In the
// DST basis of the transformed direction(s) those operators are diagonal (second difference ->
// lambda - 2, Pade [1 10 1] -> 10 + lambda), so after the forward DST the RHS of line q is
//     F = h^2 [ alpha g + beta D2 g + gamma (omega/12 + D2 omega/360) ],  omega = T^-1 (12 D2 g)
// where g is the transformed source along the line, D2 the second difference along the line
// (zero boundary values), T = tridiag(1, 10, 1) the Pade matrix of the line direction, and
// alpha, beta, gamma depend on the order and on the line's eigenvalues.  It is applied in
// registers before the Helmholtz solve, so the RHS assembly costs no extra HBM traffic.
#include "hh_internal.cuh"

namespace hh {

struct LineCoef {
    const double2 *c[4]; // four per-row complex tables (rows each)
};

__device__ __forceinline__ double2 shifted(const double2 *__restrict__ tab, int rows, int r, double m0, double m1,
                                           double m2) {
    const double2 a = __ldg(tab + r), b = __ldg(tab + rows + r), c = __ldg(tab + 2 * rows + r),
                  d = __ldg(tab + 3 * rows + r);
    // ((a m0 + b m1) + c m2) + d, as the reference's LU.c:35 orders the 3D sum
    return make_double2(((a.x * m0 + b.x * m1) + c.x * m2) + d.x, ((a.y * m0 + b.y * m1) + c.y * m2) + d.y);
}

// ----------------------------------------------------------------- factors --------
__global__ void k_factor(int lines, int rows, const double *__restrict__ mu, const double2 *__restrict__ subt,
                         const double2 *__restrict__ diagt, const double2 *__restrict__ supt,
                         double2 *__restrict__ Lf, double2 *__restrict__ Ui) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= lines) return;
    const double m0 = mu[q], m1 = mu[lines + q], m2 = mu[2 * lines + q];
    double2 piv = shifted(diagt, rows, 0, m0, m1, m2);
    double2 up_prev = shifted(supt, rows, 0, m0, m1, m2);
    Lf[q] = make_double2(0.0, 0.0);
    Ui[q] = crcp(piv);
    for (int r = 1; r < rows; r++) {
        const double2 sub = shifted(subt, rows, r, m0, m1, m2);
        const double2 dia = shifted(diagt, rows, r, m0, m1, m2);
        const double2 L = cdiv(sub, piv);
        piv = cfms(dia, L, up_prev);
        const long o = (long)r * lines + q;
        Lf[o] = L;
        Ui[o] = crcp(piv);
        up_prev = shifted(supt, rows, r, m0, m1, m2);
    }
}

int launch_factor(Plan *p, const double2 *subt, const double2 *diagt, const double2 *supt) {
    const int nt = 128;
    k_factor<<<(p->lines + nt - 1) / nt, nt, 0, p->ctx->stream>>>(p->lines, p->rows, p->mu, subt, diagt, supt, p->Lf,
                                                                   p->Ui);
    HH_CUDA(cudaGetLastError());
    p->ctx->launches++;
    return HH_OK;
}

// ------------------------------------------------------------------- solve --------
constexpr int kSolveThreads = 512;

// Inclusive scan of affine maps (A, B) over the P segments of each of the CW lines of the CTA.
// Thread (c, s) sits at tid = c + CW*s.  FORWARD combines left-to-right, otherwise right-to-left.
// Returns the value entering this thread's segment (B of the neighbour's inclusive prefix).
template <bool FORWARD>
__device__ __forceinline__ double2 segment_scan(double2 A, double2 B, int c, int s, int CW, int P, double2 *sA,
                                                double2 *sB) {
    const int pos = FORWARD ? s : (P - 1 - s);
    const int me = c + CW * pos;
    sA[me] = A;
    sB[me] = B;
    __syncthreads();
    for (int d = 1; d < P; d <<= 1) {
        double2 Al = make_double2(0.0, 0.0), Bl = make_double2(0.0, 0.0);
        const bool has = pos >= d;
        if (has) {
            Al = sA[me - CW * d];
            Bl = sB[me - CW * d];
        }
        __syncthreads();
        if (has) {
            B = cfma(B, A, Bl); // apply the earlier map first: y = A (Al y0 + Bl) + B
            A = cmul(A, Al);
            sA[me] = A;
            sB[me] = B;
        }
        __syncthreads();
    }
    const double2 in = (pos > 0) ? sB[me - CW] : make_double2(0.0, 0.0);
    __syncthreads(); // buffers are reused by the next scan
    return in;
}

// Values of the rows just before and just after this thread's segment (zero outside the line).
template <int SEG>
__device__ __forceinline__ void segment_neighbours(const double2 (&v)[SEG], int c, int s, int CW, int P,
                                                   double2 *sA, double2 *sB, double2 &before, double2 &after) {
    const int me = c + CW * s;
    sA[me] = v[0];
    sB[me] = v[SEG - 1];
    __syncthreads();
    before = (s > 0) ? sB[me - CW] : make_double2(0.0, 0.0);
    after = (s + 1 < P) ? sA[me + CW] : make_double2(0.0, 0.0);
    __syncthreads();
}

struct SrcParams {
    int     dim;       // 2 or 3
    double  h2;        // h^2
    double2 k2h2_20;   // k^2 h^2 / 20
    const double *pl;  // Pade [1 10 1] multipliers L_r = 1/U_{r-1} (L_0 = 0), rows
    const double *pu;  // Pade reciprocal pivots 1/U_r, rows
};

// SRC = 0: the input already is the transformed RHS.  SRC = 2/4/6: the input is the transformed
// source g and the compact operator of that order is applied first.
template <int SEG, int SRC>
__global__ void __launch_bounds__(kSolveThreads)
    k_line_solve(const double2 *__restrict__ in, double2 *__restrict__ out, int lines, int rows, long row_stride,
                 long field, int CW, int P, const double2 *__restrict__ Lf, const double2 *__restrict__ Ui,
                 const double2 *__restrict__ supt, const double *__restrict__ mu, SrcParams sp) {
    __shared__ double2 sA[kSolveThreads], sB[kSolveThreads];
    const int tid = threadIdx.x;
    const int c = tid % CW, s = tid / CW;
    const int q = blockIdx.x * CW + c;
    const bool live = q < lines;
    const int r0 = s * SEG;
    const long base = (long)blockIdx.y * field;
    const double m0 = live ? mu[q] : 0.0, m1 = live ? mu[lines + q] : 0.0, m2 = live ? mu[2 * lines + q] : 0.0;

    double2 v[SEG];
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int r = r0 + u;
        v[u] = (live && r < rows) ? in[base + (long)r * row_stride + q] : make_double2(0.0, 0.0);
    }

    // ---- compact right-hand-side operator in the transformed basis
    if constexpr (SRC == 2) {
#pragma unroll
        for (int u = 0; u < SEG; u++) v[u] = cscale(v[u], sp.h2);
    } else if constexpr (SRC == 4 || SRC == 6) {
        double2 alpha;
        double  beta;
        if constexpr (SRC == 4) {
            alpha = make_double2(sp.dim == 2 ? (10.0 + m1) / 12.0 : (8.0 + m1 + m2) / 12.0, 0.0);
            beta = 1.0 / 12.0;
        } else {
            if (sp.dim == 2) {
                const double muq = 12.0 * (m1 - 2.0) / (10.0 + m1);
                alpha = make_double2(1.0 + muq / 12.0 + (m1 - 2.0) * muq / 360.0 - sp.k2h2_20.x, -sp.k2h2_20.y);
                beta = muq / 90.0;
            } else {
                const double mx = 12.0 * (m1 - 2.0) / (10.0 + m1), my = 12.0 * (m2 - 2.0) / (10.0 + m2);
                alpha = make_double2(1.0 + (mx + my) / 12.0 + ((m1 - 2.0) * mx + (m2 - 2.0) * my) / 360.0 +
                                         (m2 - 2.0) * mx / 90.0 - sp.k2h2_20.x,
                                     -sp.k2h2_20.y);
                beta = (mx + my) / 90.0;
            }
        }
        double2 before, after;
        segment_neighbours<SEG>(v, c, s, CW, P, sA, sB, before, after);
        double2 d[SEG];
#pragma unroll
        for (int u = 0; u < SEG; u++) {
            const double2 lo = (u == 0) ? before : v[u - 1];
            const double2 hi = (u == SEG - 1) ? after : v[u + 1];
            d[u] = make_double2(lo.x - 2.0 * v[u].x + hi.x, lo.y - 2.0 * v[u].y + hi.y);
        }
#pragma unroll
        for (int u = 0; u < SEG; u++)
            v[u] = make_double2(alpha.x * v[u].x - alpha.y * v[u].y + beta * d[u].x,
                                alpha.x * v[u].y + alpha.y * v[u].x + beta * d[u].y);
        if constexpr (SRC == 6) {
            // omega = T^-1 (12 D2 g): Pade solve along the line (real constant factors)
            double2 zh = make_double2(0.0, 0.0), A = make_double2(1.0, 0.0);
#pragma unroll
            for (int u = 0; u < SEG; u++) {
                const int r = r0 + u;
                if (r < rows) {
                    const double l = __ldg(sp.pl + r);
                    zh = make_double2(12.0 * d[u].x - l * zh.x, 12.0 * d[u].y - l * zh.y);
                    A = make_double2(-l * A.x, -l * A.y);
                }
            }
            double2 z = segment_scan<true>(A, zh, c, s, CW, P, sA, sB);
#pragma unroll
            for (int u = 0; u < SEG; u++) {
                const int r = r0 + u;
                if (r < rows) {
                    const double l = __ldg(sp.pl + r);
                    z = make_double2(12.0 * d[u].x - l * z.x, 12.0 * d[u].y - l * z.y);
                    d[u] = z;
                }
            }
            double2 wh = make_double2(0.0, 0.0);
            A = make_double2(1.0, 0.0);
#pragma unroll
            for (int u = SEG - 1; u >= 0; u--) {
                const int r = r0 + u;
                if (r < rows) {
                    const double iu = __ldg(sp.pu + r);
                    wh = make_double2((d[u].x - wh.x) * iu, (d[u].y - wh.y) * iu);
                    A = make_double2(-iu * A.x, -iu * A.y);
                }
            }
            double2 w = segment_scan<false>(A, wh, c, s, CW, P, sA, sB);
#pragma unroll
            for (int u = SEG - 1; u >= 0; u--) {
                const int r = r0 + u;
                if (r < rows) {
                    const double iu = __ldg(sp.pu + r);
                    w = make_double2((d[u].x - w.x) * iu, (d[u].y - w.y) * iu);
                    d[u] = w;
                } else {
                    d[u] = make_double2(0.0, 0.0);
                }
            }
            segment_neighbours<SEG>(d, c, s, CW, P, sA, sB, before, after);
#pragma unroll
            for (int u = 0; u < SEG; u++) {
                const double2 lo = (u == 0) ? before : d[u - 1];
                const double2 hi = (u == SEG - 1) ? after : d[u + 1];
                const double2 d2w = make_double2(lo.x - 2.0 * d[u].x + hi.x, lo.y - 2.0 * d[u].y + hi.y);
                v[u] = make_double2(v[u].x + d[u].x / 12.0 + d2w.x / 360.0, v[u].y + d[u].y / 12.0 + d2w.y / 360.0);
            }
        }
#pragma unroll
        for (int u = 0; u < SEG; u++) v[u] = (r0 + u < rows) ? cscale(v[u], sp.h2) : make_double2(0.0, 0.0);
    }

    // ---- forward substitution y_r = f_r - L_r y_{r-1}
    double2 yh = make_double2(0.0, 0.0), A = make_double2(1.0, 0.0);
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int r = r0 + u;
        if (live && r < rows) {
            const double2 L = __ldg(Lf + (long)r * lines + q);
            yh = cfms(v[u], L, yh);
            A = make_double2(-(L.x * A.x - L.y * A.y), -(L.x * A.y + L.y * A.x));
        }
    }
    double2 y = segment_scan<true>(A, yh, c, s, CW, P, sA, sB);
#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int r = r0 + u;
        if (live && r < rows) {
            const double2 L = __ldg(Lf + (long)r * lines + q);
            y = cfms(v[u], L, y);
            v[u] = y;
        }
    }

    // ---- back substitution x_r = y_r/P_r - (super_r/P_r) x_{r+1}
    double2 xh = make_double2(0.0, 0.0);
    A = make_double2(1.0, 0.0);
#pragma unroll
    for (int u = SEG - 1; u >= 0; u--) {
        const int r = r0 + u;
        if (live && r < rows) {
            const double2 ui = __ldg(Ui + (long)r * lines + q);
            const double2 tau = cmul(shifted(supt, rows, r, m0, m1, m2), ui); // super_r / P_r
            xh = cfms(cmul(v[u], ui), tau, xh);
            A = make_double2(-(tau.x * A.x - tau.y * A.y), -(tau.x * A.y + tau.y * A.x));
        }
    }
    double2 x = segment_scan<false>(A, xh, c, s, CW, P, sA, sB);
#pragma unroll
    for (int u = SEG - 1; u >= 0; u--) {
        const int r = r0 + u;
        if (live && r < rows) {
            const double2 ui = __ldg(Ui + (long)r * lines + q);
            const double2 tau = cmul(shifted(supt, rows, r, m0, m1, m2), ui);
            x = cfms(cmul(v[u], ui), tau, x);
            v[u] = x;
        }
    }

#pragma unroll
    for (int u = 0; u < SEG; u++) {
        const int r = r0 + u;
        if (live && r < rows) out[base + (long)r * row_stride + q] = v[u];
    }
}

static int solve_geometry(int rows, int seg, int *CW, int *P) {
    int p = 1;
    while (p * seg < rows) p <<= 1;
    if (p > kSolveThreads) {
        set_error("line length %d exceeds %d", rows, kSolveThreads * seg);
        return HH_ERR_UNSUPPORTED;
    }
    *P = p;
    *CW = kSolveThreads / p;
    return HH_OK;
}

template <int SEG, int SRC> static int launch_solve_t(Plan *p, const double2 *in, double2 *out, int batch) {
    int CW, P;
    HH_TRY(solve_geometry(p->rows, SEG, &CW, &P));
    SrcParams sp;
    sp.dim = p->dim;
    sp.h2 = p->h * p->h;
    sp.k2h2_20 = make_double2(p->k2.x * sp.h2 / 20.0, p->k2.y * sp.h2 / 20.0);
    sp.pl = p->pade_l;
    sp.pu = p->pade_u;
    dim3 grid((unsigned)((p->lines + CW - 1) / CW), (unsigned)batch);
    k_line_solve<SEG, SRC><<<grid, kSolveThreads, 0, p->ctx->stream>>>(in, out, p->lines, p->rows, p->row_stride,
                                                                         p->field, CW, P, p->Lf, p->Ui, p->rowc, p->mu,
                                                                         sp);
    HH_CUDA(cudaGetLastError());
    p->ctx->launches++;
    return HH_OK;
}

int launch_line_solve(Plan *p, const double2 *in, double2 *out, int batch, int src_order) {
    switch (src_order) {
    case 0: return launch_solve_t<16, 0>(p, in, out, batch);
    case 2: return launch_solve_t<16, 2>(p, in, out, batch);
    case 4: return launch_solve_t<16, 4>(p, in, out, batch);
    case 6: return launch_solve_t<8, 6>(p, in, out, batch);
    default: set_error("source operator order %d", src_order); return HH_ERR_INVALID;
    }
}

} // namespace hh
