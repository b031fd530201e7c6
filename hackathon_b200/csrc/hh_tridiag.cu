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
// Solve: each thread owns a segment of kSeg = 8 consecutive rows of one line.  Only the
// reciprocal pivot entering each segment is stored by the set-up; the thread re-runs the
// factor recurrence for its own rows into registers (the same arithmetic, so the factors are
// those of the sequential factorisation) and keeps them for every right-hand side of its
// chunk.  Forward substitution y_r = f_r - L_r y_{r-1} and back substitution
// x_r = (y_r - super_r x_{r+1}) / P_r are first-order linear recurrences: each segment applies
// its rows as an affine map y_out = A y_in + B of the value entering it.  A (product of the
// segment's multipliers) depends on the factors only; B comes from a local sweep.  The maps of
// a line are composed across its segments by a warp-shuffle scan plus one cross-warp level in
// shared memory, and every segment then re-runs its rows from the exact entering value.  The
// next right-hand side is prefetched into shared memory with cp.async while the current one
// is solved.  One HBM read and one HBM write per point; no per-point factor traffic.
//
// Fused right-hand-side operator (plans for the constant-k, homogeneous-Dirichlet class).  The
// compact RHS of 2D_Program/main_functions/rhs.c:4-97 and 3D_Program/main_functions/rhs.c:13-166
// is a polynomial in the 1D second-difference and Pade operators of each direction.  In the
// DST basis of the transformed direction(s) those operators are diagonal (second difference ->
// lambda - 2, Pade [1 10 1] -> 10 + lambda), so after the forward DST the RHS of line q is
//     order 6:  F = h^2 [ alpha g + beta D2 g + omega/12 + D2 omega/360 ],  omega = T^-1 (12 D2 g)
// where g is the transformed source along the line, D2 the second difference along the line
// (zero boundary values), T = tridiag(1, 10, 1) = D2 + 12 I the Pade matrix of the line
// direction, and alpha, beta depend on k and on the line's eigenvalues.  Because T = D2 + 12 I,
// omega = 12 g - 144 T^-1 g and D2 omega = 12 D2 g - 144 g + 1728 T^-1 g, so
//     order 6:  F = h^2 [ (alpha + 0.6) g + (beta + 1/30) D2 g - 7.2 T^-1 g ]
//     order 4:  F = h^2 [ alpha g + D2 g / 12 ],    order 2:  F = h^2 g
// It is applied in registers before the Helmholtz solve, so the RHS assembly costs no extra
// HBM traffic.
#include "hh_internal.cuh"
#include "hh_tma.cuh"

#include <algorithm>

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
constexpr int kSeg = 8;          // rows per thread in the solve

// One step of the factor recurrence, shared by the set-up and the solve so both produce the
// same values: L = sub / P_prev (as sub * (1/P_prev)), P = diag - L super_prev, returns 1/P.
__device__ __forceinline__ double2 factor_step(double2 sub, double2 dia, double2 sup_prev, double2 ui_prev,
                                               double2 &L) {
    L = make_double2(fma(sub.x, ui_prev.x, -(sub.y * ui_prev.y)), fma(sub.x, ui_prev.y, sub.y * ui_prev.x));
    const double2 P = make_double2(dia.x - fma(L.x, sup_prev.x, -(L.y * sup_prev.y)),
                                   dia.y - fma(L.x, sup_prev.y, L.y * sup_prev.x));
    const double  d = 1.0 / fma(P.x, P.x, P.y * P.y);
    return make_double2(P.x * d, -P.y * d);
}
__device__ __forceinline__ double2 first_pivot(double2 dia) {
    const double d = 1.0 / fma(dia.x, dia.x, dia.y * dia.y);
    return make_double2(dia.x * d, -dia.y * d);
}

// One thread per line: runs the Thomas recurrence over the whole line (the reference's LU(),
// 2D LU.c:25-40 / 3D LU.c:51-72) and keeps 1/P of the row before each kSeg-row segment.
// CONST_ROWS: the stencil rows are the same along the line, so they are formed once (the same
// values the per-row evaluation gives) and the recurrence runs without memory traffic.
template <bool CONST_ROWS>
__global__ void k_factor(int lines, int rows, int prow, const double *__restrict__ mu,
                         const double2 *__restrict__ subt, const double2 *__restrict__ diagt,
                         const double2 *__restrict__ supt, double2 *__restrict__ Pv) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= lines) return;
    const double m0 = mu[q], m1 = mu[lines + q], m2 = mu[2 * lines + q];
    double2 ui = first_pivot(shifted(diagt, prow, 0, m0, m1, m2));
    double2 up_prev = shifted(supt, prow, 0, m0, m1, m2);
    const double2 sub_c = shifted(subt, prow, 0, m0, m1, m2), dia_c = shifted(diagt, prow, 0, m0, m1, m2);
    Pv[q] = make_double2(0.0, 0.0);
    for (int r = 1; r < rows; r++) {
        if (r % kSeg == 0) Pv[(long)(r / kSeg) * lines + q] = ui;
        double2 L;
        if constexpr (CONST_ROWS) {
            ui = factor_step(sub_c, dia_c, up_prev, ui, L);
        } else {
            ui = factor_step(shifted(subt, prow, r, m0, m1, m2), shifted(diagt, prow, r, m0, m1, m2), up_prev, ui,
                             L);
            up_prev = shifted(supt, prow, r, m0, m1, m2);
        }
    }
}

int launch_factor(Plan *p, const double2 *subt, const double2 *diagt, const double2 *supt) {
    const int nt = 64;
    if (p->const_rows)
        k_factor<true><<<(p->lines + nt - 1) / nt, nt, 0, p->ctx->stream>>>(p->lines, p->rows, p->prow, p->mu, subt,
                                                                             diagt, supt, p->Pv);
    else
        k_factor<false><<<(p->lines + nt - 1) / nt, nt, 0, p->ctx->stream>>>(p->lines, p->rows, p->prow, p->mu, subt,
                                                                              diagt, supt, p->Pv);
    HH_CUDA(cudaGetLastError());
    p->ctx->launches++;
    return HH_OK;
}

// ------------------------------------------------------------------- solve --------
// Thread (c, s): line c of the CTA (fastest), segment s.  A warp holds all CW lines and
// SPW = 32/CW consecutive segments of each, so a line's segments are spread over the warps.
struct Lane {
    int c, s, sl, w, lane, CW, SPW;
};

__device__ __forceinline__ double2 shfl_up2(double2 v, int off) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, off), __shfl_up_sync(0xffffffffu, v.y, off));
}
__device__ __forceinline__ double2 shfl_down2(double2 v, int off) {
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, off), __shfl_down_sync(0xffffffffu, v.y, off));
}

template <int NW> struct ScanSmem {
    double2 A[2][NW][32], B[2][NW][32]; // cross-warp totals / neighbour values (double buffered)
    double2 E[NW][32];                  // value entering each warp's first segment, per line
                                        // (rewritten only after the next scan's barrier)
    double  pl[9], pu[9];               // Pade factors of rows 0..8 (constant from row 9 on)
};

// shuffles within groups of NW lanes (the warps of one line in cross_warp_scan)
template <int NW> __device__ __forceinline__ double2 shfl_up_w(double2 v, int off) {
    return make_double2(__shfl_up_sync(0xffffffffu, v.x, off, NW), __shfl_up_sync(0xffffffffu, v.y, off, NW));
}
template <int NW> __device__ __forceinline__ double2 shfl_down_w(double2 v, int off) {
    return make_double2(__shfl_down_sync(0xffffffffu, v.x, off, NW), __shfl_down_sync(0xffffffffu, v.y, off, NW));
}

// Exclusive scan of the per-warp maps (sm.A, sm.B)[par][w][c] over w, for every line c of the CTA:
// sm.E[w][c] = value entering warp w.  Thread t < NW*CW handles (w = t % NW, c = t / NW); the NW
// warps of a line sit in consecutive lanes, so the scan is a width-NW shuffle scan.  FORWARD
// composes warps left to right, else right to left.
template <int NW, bool FORWARD>
__device__ __forceinline__ void cross_warp_scan(ScanSmem<NW> &sm, int par, int CW) {
    const int t = threadIdx.x;
    if ((t >> 5) < (NW * CW + 31) / 32) { // whole warps take part in the shuffles
        const bool in = t < NW * CW;
        const int  w = t % NW, c = t / NW;
        const int  pos = FORWARD ? w : NW - 1 - w;
        double2 A = make_double2(1.0, 0.0), B = make_double2(0.0, 0.0);
        if (in) {
            A = sm.A[par][w][c];
            B = sm.B[par][w][c];
        }
        for (int off = 1; off < NW; off <<= 1) {
            const double2 Ao = FORWARD ? shfl_up_w<NW>(A, off) : shfl_down_w<NW>(A, off);
            const double2 Bo = FORWARD ? shfl_up_w<NW>(B, off) : shfl_down_w<NW>(B, off);
            if (pos >= off) {
                B = cfma(B, A, Bo);
                A = cmul(A, Ao);
            }
        }
        double2 Ex = FORWARD ? shfl_up_w<NW>(B, 1) : shfl_down_w<NW>(B, 1);
        if (pos == 0) Ex = make_double2(0.0, 0.0);
        if (in) sm.E[w][c] = Ex;
    }
}

// Value entering segment s for the left-to-right composition of maps (A, B): y = A y_in + B.
template <int NW>
__device__ __forceinline__ double2 scan_forward(double2 A, double2 B, const Lane &L, ScanSmem<NW> &sm, int par) {
    for (int off = L.CW; off < 32; off <<= 1) {
        const double2 Al = shfl_up2(A, off), Bl = shfl_up2(B, off);
        if (L.lane >= off) {
            B = cfma(B, A, Bl);
            A = cmul(A, Al);
        }
    }
    double2 Ae = shfl_up2(A, L.CW), Be = shfl_up2(B, L.CW);
    if (L.sl == 0) { Ae = make_double2(1.0, 0.0); Be = make_double2(0.0, 0.0); }
    if (L.sl == L.SPW - 1) { sm.A[par][L.w][L.c] = A; sm.B[par][L.w][L.c] = B; }
    __syncthreads();
    cross_warp_scan<NW, true>(sm, par, L.CW);
    __syncthreads();
    return cfma(Be, Ae, sm.E[L.w][L.c]);
}

// Value entering segment s from the right (maps composed right-to-left).
template <int NW>
__device__ __forceinline__ double2 scan_backward(double2 A, double2 B, const Lane &L, ScanSmem<NW> &sm, int par) {
    for (int off = L.CW; off < 32; off <<= 1) {
        const double2 Ar = shfl_down2(A, off), Br = shfl_down2(B, off);
        if (L.lane + off < 32) {
            B = cfma(B, A, Br);
            A = cmul(A, Ar);
        }
    }
    double2 Ae = shfl_down2(A, L.CW), Be = shfl_down2(B, L.CW);
    if (L.sl == L.SPW - 1) { Ae = make_double2(1.0, 0.0); Be = make_double2(0.0, 0.0); }
    if (L.sl == 0) { sm.A[par][L.w][L.c] = A; sm.B[par][L.w][L.c] = B; }
    __syncthreads();
    cross_warp_scan<NW, false>(sm, par, L.CW);
    __syncthreads();
    return cfma(Be, Ae, sm.E[L.w][L.c]);
}

// Last value of segment s-1 and first value of segment s+1 (zero outside the line).
template <int NW>
__device__ __forceinline__ void neighbours(double2 lo, double2 hi, const Lane &L, ScanSmem<NW> &sm, int par,
                                           double2 &prev_hi, double2 &next_lo) {
    prev_hi = shfl_up2(hi, L.CW);
    next_lo = shfl_down2(lo, L.CW);
    if (L.sl == L.SPW - 1) sm.B[par][L.w][L.c] = hi;
    if (L.sl == 0) sm.A[par][L.w][L.c] = lo;
    __syncthreads();
    if (L.sl == 0) prev_hi = (L.w > 0) ? sm.B[par][L.w - 1][L.c] : make_double2(0.0, 0.0);
    if (L.sl == L.SPW - 1) next_lo = (L.w < NW - 1) ? sm.A[par][L.w + 1][L.c] : make_double2(0.0, 0.0);
}

// 16-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros.
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

struct SrcParams {
    int     dim;      // 2 or 3
    double  h2;       // h^2
    double2 k2h2_20;  // k^2 h^2 / 20
    const double *pl; // Pade [1 10 1] multipliers L_r = 1/U_{r-1} (L_0 = 0); zero past the line
    const double *pu; // Pade reciprocal pivots 1/U_r; zero past the line
    double linf, uinf;// both converge to 1/(5 + sqrt 24) exactly in double from row 9 on
};

// Pade factors of row r: rows 0..8 from shared memory, the fixed point up to the line end, zero
// past it (neutral padded rows).
template <int NW>
__device__ __forceinline__ double pade_l(const ScanSmem<NW> &sm, const SrcParams &sp, int r, int rows) {
    return r < 9 ? sm.pl[r] : (r < rows ? sp.linf : 0.0);
}
template <int NW>
__device__ __forceinline__ double pade_u(const ScanSmem<NW> &sm, const SrcParams &sp, int r, int rows) {
    return r < 9 ? sm.pu[r] : (r < rows ? sp.uinf : 0.0);
}

// SRC = 0: the input already is the transformed RHS.  SRC = 2/4/6: the input is the transformed
// source g and the compact operator of that order is applied first (see the file header).
// CONST_ROWS: the stencil rows do not vary along the line (constant k).
// Rows past the end of a line are neutral: zero data, zero reciprocal pivots, zero Pade factors,
// so the sweeps run without per-row conditions.
template <int SRC, bool CONST_ROWS, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_line_solve(const double2 *__restrict__ in, double2 *__restrict__ out, int lines, int rows, int prow,
                 long row_stride, long field, int batch, int rb, int CW, const double2 *__restrict__ Pv,
                 const double2 *__restrict__ subt, const double2 *__restrict__ diagt, const double2 *__restrict__ supt,
                 const double *__restrict__ mu, SrcParams sp) {
    constexpr int NW = NT / 32;
    __shared__ ScanSmem<NW> sm;
    extern __shared__ double2 pre[]; // [kSeg][NT] prefetch of the next right-hand side,
                                     // then (SRC == 6) [kSeg][NT] Pade scratch
    double2 *wsm = pre + kSeg * NT + threadIdx.x;
    Lane L;
    L.lane = threadIdx.x & 31;
    L.w = threadIdx.x >> 5;
    L.CW = CW;
    L.SPW = 32 / CW;
    L.c = threadIdx.x % CW;
    L.s = threadIdx.x / CW;
    L.sl = L.lane / CW;
    const int  q = blockIdx.x * CW + L.c;
    const bool live = q < lines;
    const int  qq = live ? q : 0;
    const int  r0 = L.s * kSeg;
    const double m0 = live ? mu[q] : 0.0, m1 = live ? mu[lines + q] : 0.0, m2 = live ? mu[2 * lines + q] : 0.0;
    const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);

    // ---- factors of this thread's rows, kept in registers for the whole chunk
    double2 sub_c = zero, sup_c = zero;
    if constexpr (CONST_ROWS) {
        sub_c = shifted(subt, prow, 0, m0, m1, m2);
        sup_c = shifted(supt, prow, 0, m0, m1, m2);
    }
    const double2 ui_in = (live && r0 > 0 && r0 < rows) ? Pv[(long)L.s * lines + q] : zero; // 1/P of row r0-1
    double2 ui[kSeg];
    double2 Af = one, Ab = one;
    {
        double2 uprev = ui_in;
        const double2 dia_c = CONST_ROWS ? shifted(diagt, prow, 0, m0, m1, m2) : zero;
#pragma unroll
        for (int u = 0; u < kSeg; u++) {
            const int r = r0 + u;
            double2   Lr = zero;
            ui[u] = zero;
            if (live && r < rows) {
                const double2 dia = CONST_ROWS ? dia_c : shifted(diagt, prow, r, m0, m1, m2);
                if (r == 0) {
                    ui[u] = first_pivot(dia);
                } else {
                    const double2 sb = CONST_ROWS ? sub_c : shifted(subt, prow, r, m0, m1, m2);
                    const double2 sp_ = CONST_ROWS ? sup_c : shifted(supt, prow, r - 1, m0, m1, m2);
                    ui[u] = factor_step(sb, dia, sp_, uprev, Lr);
                }
            } else if (live && r > 0 && u > 0) {
                const double2 sb = CONST_ROWS ? sub_c : shifted(subt, prow, r, m0, m1, m2);
                Lr = cmul(sb, uprev); // first padded row: L is still formed from the last real pivot
            }
            uprev = ui[u];
            Af = cmul(Af, make_double2(-Lr.x, -Lr.y));
            const double2 sp2 = CONST_ROWS ? sup_c : shifted(supt, prow, r, m0, m1, m2);
            const double2 tau = cmul(sp2, ui[u]);
            Ab = cmul(Ab, make_double2(-tau.x, -tau.y));
        }
    }

    // per-line coefficients of the compact right-hand-side operator
    double2 alpha = one;
    double  beta = 0.0;
    if constexpr (SRC == 4) {
        alpha = make_double2(sp.dim == 2 ? (10.0 + m1) / 12.0 : (8.0 + m1 + m2) / 12.0, 0.0);
        beta = 1.0 / 12.0;
    } else if constexpr (SRC == 6) {
        if (sp.dim == 2) {
            const double muq = 12.0 * (m1 - 2.0) / (10.0 + m1);
            alpha = make_double2(1.6 + muq / 12.0 + (m1 - 2.0) * muq / 360.0 - sp.k2h2_20.x, -sp.k2h2_20.y);
            beta = muq / 90.0 + 1.0 / 30.0;
        } else {
            const double mx = 12.0 * (m1 - 2.0) / (10.0 + m1), my = 12.0 * (m2 - 2.0) / (10.0 + m2);
            alpha = make_double2(1.6 + (mx + my) / 12.0 + ((m1 - 2.0) * mx + (m2 - 2.0) * my) / 360.0 +
                                     (m2 - 2.0) * mx / 90.0 - sp.k2h2_20.x,
                                 -sp.k2h2_20.y);
            beta = (mx + my) / 90.0 + 1.0 / 30.0;
        }
    }
    double pa = 1.0, pb = 1.0; // Pade segment products
    if constexpr (SRC == 6) {
        if (threadIdx.x < 9) {
            sm.pl[threadIdx.x] = sp.pl[threadIdx.x];
            sm.pu[threadIdx.x] = sp.pu[threadIdx.x];
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < kSeg; u++) {
            pa *= -pade_l(sm, sp, r0 + u, rows);
            pb *= -pade_u(sm, sp, r0 + u, rows);
        }
    }

    const int  b_begin = blockIdx.y * rb;
    const int  b_end = min(batch, b_begin + rb);
    const long off0 = (long)r0 * row_stride + qq;
    auto prefetch = [&](int b) {
        const double2 *src = in + (long)b * field + off0;
#pragma unroll
        for (int u = 0; u < kSeg; u++) {
            const bool ok = live && r0 + u < rows;
            cp_async16(&pre[u * NT + threadIdx.x], ok ? src + (long)u * row_stride : in, ok ? 16 : 0);
        }
        cp_async_commit();
    };
    prefetch(b_begin);
    int par = 0;
    for (int b = b_begin; b < b_end; b++) {
        double2 v[kSeg];
        cp_async_wait_all();
#pragma unroll
        for (int u = 0; u < kSeg; u++) v[u] = pre[u * NT + threadIdx.x];
        if (b + 1 < b_end) prefetch(b + 1);

        // ---- compact right-hand-side operator in the transformed basis
        if constexpr (SRC == 2) {
#pragma unroll
            for (int u = 0; u < kSeg; u++) v[u] = cscale(v[u], sp.h2);
        } else if constexpr (SRC == 4 || SRC == 6) {
            double2 before, after;
            neighbours(v[0], v[kSeg - 1], L, sm, par, before, after);
            par ^= 1;
            double2 zh = zero;
            if constexpr (SRC == 6) {
                // forward Pade sweep of g (local part): z_r = g_r - l_r z_{r-1}
#pragma unroll
                for (int u = 0; u < kSeg; u++) {
                    const double l = pade_l(sm, sp, r0 + u, rows);
                    zh = make_double2(v[u].x - l * zh.x, v[u].y - l * zh.y);
                    wsm[u * NT] = zh;
                }
            }
            double2 gprev = before;
#pragma unroll
            for (int u = 0; u < kSeg; u++) {
                const double2 g = v[u];
                const double2 hi = (u == kSeg - 1) ? after : v[u + 1];
                const double2 d2 = make_double2(gprev.x - 2.0 * g.x + hi.x, gprev.y - 2.0 * g.y + hi.y);
                gprev = g;
                v[u] = make_double2(fma(alpha.x, g.x, fma(-alpha.y, g.y, beta * d2.x)),
                                    fma(alpha.x, g.y, fma(alpha.y, g.x, beta * d2.y)));
            }
            if constexpr (SRC == 6) {
                // complete the forward sweep from the exact entering value, then the backward one:
                // w_r = (z_r - w_{r+1}) / U_r;  F += -7.2 w
                const double2 zin = scan_forward(make_double2(pa, 0.0), zh, L, sm, par);
                par ^= 1;
                double2 corr = zin;
#pragma unroll
                for (int u = 0; u < kSeg; u++) {
                    const double l = pade_l(sm, sp, r0 + u, rows);
                    corr = make_double2(-l * corr.x, -l * corr.y);
                    const double2 z = wsm[u * NT];
                    wsm[u * NT] = make_double2(z.x + corr.x, z.y + corr.y);
                }
                double2 wh = zero;
#pragma unroll
                for (int u = kSeg - 1; u >= 0; u--) {
                    const double  iu = pade_u(sm, sp, r0 + u, rows);
                    const double2 z = wsm[u * NT];
                    wh = make_double2((z.x - wh.x) * iu, (z.y - wh.y) * iu);
                }
                const double2 win = scan_backward(make_double2(pb, 0.0), wh, L, sm, par);
                par ^= 1;
                double2 wv = win;
#pragma unroll
                for (int u = kSeg - 1; u >= 0; u--) {
                    const double  iu = pade_u(sm, sp, r0 + u, rows);
                    const double2 z = wsm[u * NT];
                    wv = make_double2((z.x - wv.x) * iu, (z.y - wv.y) * iu);
                    v[u] = make_double2(fma(-7.2, wv.x, v[u].x), fma(-7.2, wv.y, v[u].y));
                }
            }
        }
        if constexpr (SRC == 4 || SRC == 6) {
#pragma unroll
            for (int u = 0; u < kSeg; u++) v[u] = cscale(v[u], sp.h2);
        }

        // ---- forward substitution y_r = f_r - L_r y_{r-1},  L_r = sub_r / P_{r-1}
        double2 yh = zero;
#pragma unroll
        for (int u = 0; u < kSeg; u++) {
            const double2 sb = CONST_ROWS ? sub_c : shifted(subt, prow, r0 + u, m0, m1, m2);
            yh = cfms(v[u], cmul(sb, u == 0 ? ui_in : ui[u - 1]), yh);
        }
        double2 y = scan_forward(Af, yh, L, sm, par);
        par ^= 1;
#pragma unroll
        for (int u = 0; u < kSeg; u++) {
            const double2 sb = CONST_ROWS ? sub_c : shifted(subt, prow, r0 + u, m0, m1, m2);
            y = cfms(v[u], cmul(sb, u == 0 ? ui_in : ui[u - 1]), y);
            v[u] = y;
        }

        // ---- back substitution x_r = (y_r - super_r x_{r+1}) / P_r
        double2 xh = zero;
#pragma unroll
        for (int u = kSeg - 1; u >= 0; u--) {
            const double2 sp2 = CONST_ROWS ? sup_c : shifted(supt, prow, r0 + u, m0, m1, m2);
            xh = cmul(cfms(v[u], sp2, xh), ui[u]);
        }
        double2 x = scan_backward(Ab, xh, L, sm, par);
        par ^= 1;
#pragma unroll
        for (int u = kSeg - 1; u >= 0; u--) {
            const double2 sp2 = CONST_ROWS ? sup_c : shifted(supt, prow, r0 + u, m0, m1, m2);
            x = cmul(cfms(v[u], sp2, x), ui[u]);
            v[u] = x;
        }

        double2 *dst = out + (long)b * field + off0;
#pragma unroll
        for (int u = 0; u < kSeg; u++)
            if (live && r0 + u < rows) dst[(long)u * row_stride] = v[u];
    }
}

// Thread-count variants of the interleaved solve: NT threads per CTA, MINB CTAs per SM.
struct SolveVariant {
    int nt, minb;
};
static const SolveVariant kVariants[] = {{512, 1}, {256, 2}};
constexpr int kNumVariants = 2; // plus variants 2..5: k_line_solve_sym where the plan allows it

// segments per line: a power of two >= NT/32 (so at most 32 lines share a warp)
static int solve_geometry(int rows, int nt, int *CW, int *P) {
    int p = nt / 32;
    while (p * kSeg < rows) p <<= 1;
    if (p > nt) {
        set_error("line length %d exceeds %d", rows, nt * kSeg);
        return HH_ERR_UNSUPPORTED;
    }
    *P = p;
    *CW = nt / p;
    return HH_OK;
}

int padded_rows(int rows) {
    int best = rows;
    for (int v = 0; v < kNumVariants; v++) {
        int CW, P;
        if (solve_geometry(rows, kVariants[v].nt, &CW, &P) == HH_OK && P * kSeg > best) best = P * kSeg;
    }
    return best;
}

int solve_variant_count() { return kNumVariants + 5; }

template <int SRC, bool CR, int NT, int MINB>
static int launch_solve_t(Plan *p, const double2 *in, double2 *out, int batch) {
    int CW, P;
    HH_TRY(solve_geometry(p->rows, NT, &CW, &P));
    SrcParams sp;
    sp.dim = p->dim;
    sp.h2 = p->h * p->h;
    sp.k2h2_20 = make_double2(p->k2.x * sp.h2 / 20.0, p->k2.y * sp.h2 / 20.0);
    sp.pl = p->pade_l;
    sp.pu = p->pade_u;
    sp.linf = p->pade_linf;
    sp.uinf = p->pade_uinf;
    const int shm = (int)(sizeof(double2) * kSeg * NT) * (SRC == 6 ? 2 : 1);
    HH_CUDA(cudaFuncSetAttribute(k_line_solve<SRC, CR, NT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, shm));
    // right-hand sides per CTA: enough CTAs to fill the SMs twice, factors reused within a chunk
    const long groups = (p->lines + CW - 1) / CW;
    int rb = 1;
    while (rb < batch && groups * ((batch + 2 * rb - 1) / (2 * rb)) >= 2L * MINB * 148) rb *= 2;
    const int chunks = (batch + rb - 1) / rb;
    dim3 grid((unsigned)groups, (unsigned)chunks);
    k_line_solve<SRC, CR, NT, MINB><<<grid, NT, shm, p->ctx->stream>>>(in, out, p->lines, p->rows, p->prow,
                                                                       p->row_stride, p->field, batch, rb, CW, p->Pv,
                                                                       p->subt, p->diagt, p->rowc, p->mu, sp);
    HH_CUDA(cudaGetLastError());
    p->ctx->launches++;
    return HH_OK;
}

template <bool CR, int NT, int MINB>
static int launch_solve_v(Plan *p, const double2 *in, double2 *out, int batch, int src) {
    switch (src) {
    case 0: return launch_solve_t<0, CR, NT, MINB>(p, in, out, batch);
    case 2: return launch_solve_t<2, CR, NT, MINB>(p, in, out, batch);
    case 4: return launch_solve_t<4, CR, NT, MINB>(p, in, out, batch);
    case 6: return launch_solve_t<6, CR, NT, MINB>(p, in, out, batch);
    default: set_error("source operator order %d", src); return HH_ERR_INVALID;
    }
}

template <bool CR> static int launch_solve_cr(Plan *p, const double2 *in, double2 *out, int batch, int src) {
    if (p->variant == 1) return launch_solve_v<CR, 256, 2>(p, in, out, batch, src);
    return launch_solve_v<CR, 512, 1>(p, in, out, batch, src);
}

int launch_line_solve_sym(Plan *p, const double2 *in, double2 *out, int batch, int src_order);
bool sym_solve_supported(const Plan *p, int src_order);

int launch_line_solve(Plan *p, const double2 *in, double2 *out, int batch, int src_order) {
    if (p->variant >= 2 && sym_solve_supported(p, src_order)) return launch_line_solve_sym(p, in, out, batch, src_order);
    if (src_order == 6 && !p->pade_l) {
        set_error("order-6 source operator needs a Helmholtz plan");
        return HH_ERR_INVALID;
    }
    return p->const_rows ? launch_solve_cr<true>(p, in, out, batch, src_order)
                         : launch_solve_cr<false>(p, in, out, batch, src_order);
}

int segment_count(int rows) { return (rows + kSeg - 1) / kSeg; }

// ------------------------------------------------------------- slab <-> lines ------
// The cut of transformed planes into the ranks' lines for a slab/pencil solve, and back: element
// (b, z, q) of a slab [batch][planes][nlines] is element (z, b, q - q0_s) of rank s's part
// [planes][batch][cnt_s] of the buffer, the parts in rank order, for the balanced contiguous
// split of [0, nlines) over `world` ranks (cnt_s = base + (s < extra), q0_s = s base +
// min(s, extra)).  One thread per element, consecutive threads on consecutive q.
__global__ void __launch_bounds__(256) k_lines_pack(const double2 *__restrict__ a, double2 *__restrict__ o,
                                                    int batch, int planes, int nlines, int world, int unpack) {
    const long row = blockIdx.y; // b * planes + z
    const long b = row / planes, z = row % planes;
    const int  base = nlines / world, extra = nlines % world, cut = (base + 1) * extra;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nlines; q += gridDim.x * blockDim.x) {
        const int  s = q < cut ? q / (base + 1) : extra + (q - cut) / base;
        const int  q0 = s * base + min(s, extra), cnt = base + (s < extra ? 1 : 0);
        const long si = row * nlines + q;
        const long di = (long)batch * planes * q0 + (z * batch + b) * cnt + (q - q0);
        if (unpack) o[si] = a[di];
        else o[di] = a[si];
    }
}

int launch_lines_pack(Ctx *c, const double2 *in, double2 *out, long batch, long planes, long nlines, int world,
                      bool unpack) {
    if (batch < 0 || planes < 1 || nlines < 1 || world < 1 || world > nlines || batch * planes > 65535 ||
        nlines > (1L << 30) || planes > (1L << 30)) {
        set_error("lines pack: batch %ld, planes %ld, lines %ld, ranks %d", batch, planes, nlines, world);
        return HH_ERR_INVALID;
    }
    if (batch == 0) return HH_OK;
    const long bx = std::min<long>((nlines + 255) / 256, 64);
    dim3 grid((unsigned)bx, (unsigned)(batch * planes));
    k_lines_pack<<<grid, 256, 0, c->stream>>>(in, out, (int)batch, (int)planes, (int)nlines, world, unpack ? 1 : 0);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}


// =====================================================================================
// Symmetric constant-row lines (the Helmholtz plans): k_line_solve_sym
//
// For constant k the line matrix is A = d I + s S with S = tridiag(1, 0, 1), the same s below
// and above the diagonal, and one (d, s) per line.  The kernel specialises the solve above for
// that case:
//  * CW (lines per CTA) is a compile-time constant, so every shuffle offset and loop unrolls;
//  * the segment multipliers of the affine maps depend on the factors only, so their scan
//    coefficients are formed once per chunk of right-hand sides (tables in shared memory) and
//    each right-hand side scans only its B values;
//  * every thread loads the two neighbouring rows of its segment with its own rows, so the
//    second differences of the compact operator need no exchange;
//  * order 6: A and the Pade matrix T = 10 I + S are both polynomials in S, so they commute and
//        A^-1 T^-1 = (s A^-1 - T^-1) / (10 s - d)
//    The order-6 right-hand side  F = h^2 [a6 g + b6 D2 g - 7.2 T^-1 g]  then gives
//        u = A^-1 F = A^-1 G + cT T^-1 g,   G = h^2 [(a6 - 7.2 s/(10s - d)) g + b6 D2 g],
//        cT = 7.2 h^2 / (10 s - d)
//    two independent solves that run side by side and share every scan and barrier.  The plan
//    checks |10 s - d| against |d|, |s| on every line before it selects this path.
// =====================================================================================

// a + b c and a - b c with two fused multiply-adds per component
__device__ __forceinline__ double2 zfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(b.x, c.x, fma(-b.y, c.y, a.x)), fma(b.x, c.y, fma(b.y, c.x, a.y)));
}
__device__ __forceinline__ double2 zfms(double2 a, double2 b, double2 c) {
    return make_double2(fma(-b.x, c.x, fma(b.y, c.y, a.x)), fma(-b.x, c.y, fma(-b.y, c.x, a.y)));
}
__device__ __forceinline__ double2 zaxpy(double2 a, double b, double2 c) { // a + b c, b real
    return make_double2(fma(b, c.x, a.x), fma(b, c.y, a.y));
}

template <int NT> __host__ __device__ constexpr int ilog2_t() { return NT <= 1 ? 0 : 1 + ilog2_t<NT / 2>(); }

template <int NW, int CW, int NR> struct SymSmem {
    uint64_t tbar[2];                 // completion of the tile copies (TMA-tile input)
    double2 AwF[NW][CW], AwB[NW][CW]; // warp totals of the segment multipliers (main solve)
    double  awF[NW][CW], awB[NW][CW]; // the same for the Pade solve (real multipliers)
    double2 BwF[NR][NW][CW], BwB[NR][NW][CW]; // warp totals of the B values, per right-hand side
    double2 EF[NR][NW][CW], EB[NR][NW][CW];   // value entering each warp (order 6)
    double2 bwF[NR][NW][CW], bwB[NR][NW][CW];
    double2 eF[NR][NW][CW], eB[NR][NW][CW];
    double  pl[9], pu[9];
};

// Shared-memory reads of the scan tables that the compiler must not hoist out of the loop over
// right-hand sides (hoisting them would hold every stage multiplier in registers).
__device__ __forceinline__ double2 lds_keep(const double2 *p) {
    double2 v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];"
                 : "=d"(v.x), "=d"(v.y)
                 : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))));
    return v;
}
__device__ __forceinline__ double lds_keep(const double *p) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(static_cast<uint32_t>(__cvta_generic_to_shared(p))));
    return v;
}

// Order 6 with 16-row segments keeps its per-row multipliers tau_k = s ui_k in shared memory,
// one column per thread: in registers they would not fit beside the two solves' rows.
template <int SRC, int KS> struct SymUIS {
    static constexpr bool value = SRC == 6 && KS >= 16;
};
// ... and its per-line constants (tau_0, 1/s, c1, cT, c2) in shared memory [5][NT], each read in
// the sweep that uses it, at the CTA widths where that measured faster with identical bits (line
// solve, TMA-tile input: 3D 127^3 x 16 0.352 -> 0.317 ms, 255^3 x 4 0.756 -> 0.714 ms, 2D
// 1023^2 x 64 0.690 -> 0.684 ms; slower at 2 and 8 lines per CTA: 2047^2 x 16 0.851 -> 0.878 ms,
// 511^2 x 32 0.100 -> 0.103 ms)
template <int SRC, int KS, int CW> struct SymPCS {
    static constexpr bool value = SymUIS<SRC, KS>::value && (CW == 4 || CW >= 16);
};

// Intra-warp inclusive scan of B over the segments of each line in the warp, with the stage
// multipliers tab[j * NT] (the thread's own map product at stage j).  FWD composes left to right.
template <int CW, bool FWD>
__device__ __forceinline__ double2 sym_warp_scan(double2 B, const double2 *tab, int NT_, int sl) {
    constexpr int SPW = 32 / CW;
#pragma unroll
    for (int j = 0; (1 << j) < SPW; j++) {
        const double2 Bo = FWD ? shfl_up2(B, CW << j) : shfl_down2(B, CW << j);
        const double2 m = lds_keep(tab + j * NT_);
        if (FWD ? (sl >= (1 << j)) : (sl + (1 << j) < SPW)) B = zfma(B, m, Bo);
    }
    return B;
}
template <int CW, bool FWD>
__device__ __forceinline__ double2 sym_warp_scan(double2 B, const double *tab, int NT_, int sl) {
    constexpr int SPW = 32 / CW;
#pragma unroll
    for (int j = 0; (1 << j) < SPW; j++) {
        const double2 Bo = FWD ? shfl_up2(B, CW << j) : shfl_down2(B, CW << j);
        const double  m = lds_keep(tab + j * NT_);
        if (FWD ? (sl >= (1 << j)) : (sl + (1 << j) < SPW)) B = zaxpy(B, m, Bo);
    }
    return B;
}

struct SymParams {
    double  h2;        // h^2
    double2 k2h2_20;   // k^2 h^2 / 20
    int     dim;
    double  linf, uinf;
    const double *pl, *pu; // Pade factors (rows >= 9 equal linf, uinf)
};

// TMA-tile input of the symmetric line solve: one right-hand side of the CTA's CW lines arrives
// as a tile [rows][CW] in shared memory, brought by tensor copies over a (re/im, line, row,
// right-hand side) map in boxes of br rows, NBUF right-hand sides ahead.  Thread 0 issues the
// copies; the outputs are stored from registers as in the per-thread prefetch form.
template <int SRC> struct SymTileBufs {
    static constexpr int value = SRC == 6 ? 1 : 2; // order 6 spends the space on its pivots
};

struct SymTio {
    const CUtensorMap *in_map;
    double2           *tin;  // NBUF tiles of `tile` elements
    uint64_t          *bar;  // one per tile
    int               *err;
    int                x0, br, nbox, tile;
    unsigned           tile_bytes;
};

// One chunk of right-hand sides for the thread's segment, NR of them side by side (independent
// dependency chains, shared barriers).  TINT = the warp's rows all lie in [9, rows) (constant
// Pade factors).
template <int SRC, int NT, int CW, bool TINT, int NR, int KS, bool TIO>
__device__ __forceinline__ void sym_chunk(const double2 *__restrict__ in, double2 *__restrict__ out, int rows,
                                          long row_stride, long field, int b_begin, int b_end, long off0,
                                          bool live, int r0, int sl, int w, int c, const double2 (&Lr)[KS],
                                          const double2 (&ui)[KS], const double2 *uis, double2 ui_in, double2 s,
                                          double2 c1, double c2, double2 cT, SymSmem<NT / 32, CW, NR> &sm,
                                          double2 *pre, const double2 *tabF, const double2 *tabB, const double *ttF,
                                          const double *ttB, const SymParams &sp, const SymTio &tio) {
    constexpr int NW = NT / 32, SPW = 32 / CW, LOG = ilog2_t<SPW>();
    constexpr int HALO = (SRC == 4 || SRC == 6) ? 1 : 0;
    constexpr int SLOTS = KS + 2;
    constexpr int  NBUF = SymTileBufs<SRC>::value;
    static_assert(!TIO || NR == 1, "tile I/O moves one right-hand side at a time");
    // order 6: the warps' entering values are composed in sequence (threads [0, CW NR) for the
    // main solve, [128, 128 + CW NR) for the Pade solve)
    constexpr bool SEQ = SRC == 6;
    static_assert(!SEQ || (CW * NR <= 128 && NT >= 256), "cross-warp thread ranges");
    const int     t = threadIdx.x;
    const double2 zero = make_double2(0.0, 0.0);
    // Orders 0-4 keep the forward multipliers L_k and the reciprocal pivots ui_k in registers.
    // Order 6, where the two solves' rows fill the registers, keeps one value per row instead:
    // tau_k = s ui_k (= L_{k+1}), in the ui array or (16-row segments) in shared memory, one
    // column per thread.  The sweeps read their multipliers from it as they are, and the final
    // forward pass re-forms ui_k = (1/s) tau_k off the recurrence.
    constexpr bool UIS = SymUIS<SRC, KS>::value;
    constexpr bool KEEP_L = SRC != 6;
    auto TV = [&](int k) -> double2 {
        if constexpr (UIS) return lds_keep(uis + k * NT + t);
        else return ui[k];
    };
    constexpr bool PCS = SymPCS<SRC, KS, CW>::value;
    const double2 *pcs = reinterpret_cast<const double2 *>(ttB + (ilog2_t<32 / CW>() + 1) * NT);
    auto PC = [&](int j) -> double2 { return lds_keep(pcs + j * NT + t); };
    const double2 tau_in = PCS ? zero : cmul(s, ui_in); // L_0 = s / P of row r0 - 1
    const double2 rs = PCS ? zero : (KEEP_L ? s : crcp(s));
    // forward multiplier of row r0 + k
    auto LF = [&](int k) -> double2 {
        if constexpr (KEEP_L) return Lr[k];
        else if constexpr (PCS) return k == 0 ? PC(0) : TV(k - 1);
        else return k == 0 ? tau_in : TV(k - 1);
    };
    // backward multiplier of row r0 + k, tau_k = s ui_k (= L_{k+1} where that row exists)
    const double2 tau_last = KEEP_L ? cmul(s, ui[KS - 1]) : s;
    auto TAU = [&](int k) -> double2 {
        if constexpr (KEEP_L) return k + 1 < KS ? Lr[k + 1] : tau_last;
        else return TV(k);
    };
    // Pade factors of row r0 + k: the constants in warps whose rows all lie in [9, rows)
    auto PL = [&](int k) -> double {
        if constexpr (TINT) return sp.linf;
        const int r = r0 + k;
        return r < 9 ? sm.pl[r] : (r < rows ? sp.linf : 0.0);
    };
    auto PU = [&](int k) -> double {
        if constexpr (TINT) return sp.uinf;
        const int r = r0 + k;
        return r < 9 ? sm.pu[r] : (r < rows ? sp.uinf : 0.0);
    };

    // the tile copies of right-hand side b into tile buffer u, issued by thread 0
    auto tile_load = [&](int b, int u) {
        double2 *dst = tio.tin + (long)u * tio.tile;
        mbar_expect_tx(tio.bar + u, tio.tile_bytes);
        for (int x = 0; x < tio.nbox; x++)
            tma_tile_load(dst + (long)x * tio.br * CW, tio.in_map, tio.x0, x * tio.br, b, tio.bar + u);
    };
    auto prefetch = [&](int b) {
#pragma unroll
        for (int r = 0; r < NR; r++) {
            const bool     okb = live && b + r < b_end;
            const double2 *src = in + (long)(okb ? b + r : 0) * field + off0;
#pragma unroll
            for (int k = -HALO; k < KS + HALO; k++) {
                const bool ok = okb && r0 + k >= 0 && r0 + k < rows;
                cp_async16(&pre[(r * SLOTS + k + 1) * NT + t], ok ? src + (long)k * row_stride : in, ok ? 16 : 0);
            }
        }
        cp_async_commit();
    };
    if constexpr (!TIO) prefetch(b_begin); // with tile I/O the first tile was requested at kernel start
    int it = 0;
    for (int b = b_begin; b < b_end; b += NR, it++) {
        double2 v[NR][KS], g[NR][KS], gm[NR], gp[NR];
        bool    landed = true;
        if constexpr (TIO) {
            const int u = NBUF == 2 ? (it & 1) : 0;
            landed = mbar_wait_parity(tio.bar + u, NBUF == 2 ? (it >> 1) & 1 : it & 1);
            const double2 *tl = tio.tin + (long)u * tio.tile + c;
#pragma unroll
            for (int k = 0; k < KS; k++) v[0][k] = (r0 + k < rows) ? tl[(r0 + k) * CW] : zero;
            // threads whose segment lies wholly past the end of the line (r0 > rows) read no halo:
            // row r0 - 1 is not in the tile
            gm[0] = (HALO && r0 > 0 && r0 <= rows) ? tl[(r0 - 1) * CW] : zero;
            gp[0] = (HALO && r0 + KS < rows) ? tl[(r0 + KS) * CW] : zero;
            fence_async_smem(); // these reads before the copy that refills the tile
        } else {
            cp_async_wait_all();
#pragma unroll
            for (int r = 0; r < NR; r++) {
#pragma unroll
                for (int k = 0; k < KS; k++) v[r][k] = pre[(r * SLOTS + k + 1) * NT + t];
                gm[r] = zero;
                gp[r] = zero;
                if constexpr (HALO) {
                    gm[r] = pre[(r * SLOTS) * NT + t];
                    gp[r] = pre[(r * SLOTS + KS + 1) * NT + t];
                }
            }
            if (b + NR < b_end) prefetch(b + NR);
        }

        // ---- compact right-hand side (order 6: the A^-1 part; g keeps the source for T^-1)
#pragma unroll
        for (int r = 0; r < NR; r++) {
            if constexpr (SRC == 2) {
#pragma unroll
                for (int k = 0; k < KS; k++) v[r][k] = cscale(v[r][k], sp.h2);
            } else if constexpr (SRC == 4 || SRC == 6) {
                double2 prev = gm[r];
                const double2 c1v = PCS ? PC(2) : c1;
                const double  c2v = PCS ? PC(4).x : c2;
#pragma unroll
                for (int k = 0; k < KS; k++) {
                    const double2 gk = v[r][k], nx = (k == KS - 1) ? gp[r] : v[r][k + 1];
                    const double2 d2 = make_double2(fma(-2.0, gk.x, prev.x + nx.x), fma(-2.0, gk.y, prev.y + nx.y));
                    prev = gk;
                    if constexpr (SRC == 6) g[r][k] = gk;
                    v[r][k] = zfma(make_double2(c2v * d2.x, c2v * d2.y), c1v, gk); // c2 D2 g + c1 g
                }
            }
        }

        // ---- forward elimination: local sweeps from a zero entering value
        double2 yh[NR], zh[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) { yh[r] = zero; zh[r] = zero; }
#pragma unroll
        for (int k = 0; k < KS; k++) {
            const double2 l = LF(k);
#pragma unroll
            for (int r = 0; r < NR; r++) {
                yh[r] = zfms(v[r][k], l, yh[r]);
                if constexpr (SRC == 6)
                    zh[r] = make_double2(fma(-PL(k), zh[r].x, g[r][k].x), fma(-PL(k), zh[r].y, g[r][k].y));
            }
        }
        double2 Bfe[NR], bfe[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) {
            const double2 Bf = sym_warp_scan<CW, true>(yh[r], tabF + t, NT, sl);
            Bfe[r] = shfl_up2(Bf, CW);
            bfe[r] = zero;
            if (sl == SPW - 1) sm.BwF[r][w][c] = Bf;
            if constexpr (SRC == 6) {
                const double2 bf = sym_warp_scan<CW, true>(zh[r], ttF + t, NT, sl);
                bfe[r] = shfl_up2(bf, CW);
                if (sl == SPW - 1) sm.bwF[r][w][c] = bf;
            }
            if (sl == 0) { Bfe[r] = zero; bfe[r] = zero; }
        }
        if constexpr (TIO) {
            if (__syncthreads_or(!landed)) { // a tile copy did not land: report and leave together
                if (t == 0) {
                    atomicExch(tio.err, 1);
                    // copies still in flight get a bounded chance to land before the memory is released
                    for (int j = 0; j < NBUF && b + j < b_end; j++) {
                        const int jt = it + j;
                        mbar_wait_parity(tio.bar + (NBUF == 2 ? (jt & 1) : 0), NBUF == 2 ? (jt >> 1) & 1 : jt & 1);
                    }
                }
                return;
            }
            // every thread has read this tile: it takes the right-hand side NBUF ahead
            if (t == 0 && b + NBUF < b_end) tile_load(b + NBUF, NBUF == 2 ? (it & 1) : 0);
        } else {
            __syncthreads();
        }
        // The value entering each warp's segments of line c: the totals of the warps before it,
        // composed in order.  Orders 0-4: every warp forms its own (the totals stay until the next
        // barrier).  Order 6, whose two solves leave no registers for that: CW threads per solve
        // compose them in sequence into shared memory, behind one more barrier.
        if constexpr (SEQ) {
            if (t < CW * NR) {
                const int r = t / CW, cc = t % CW;
                double2   E = zero;
#pragma unroll
                for (int x = 0; x < NW; x++) {
                    sm.EF[r][x][cc] = E;
                    E = zfma(sm.BwF[r][x][cc], sm.AwF[x][cc], E);
                }
            } else if (t >= 128 && t < 128 + CW * NR) {
                const int r = (t - 128) / CW, cc = (t - 128) % CW;
                double2   E = zero;
#pragma unroll
                for (int x = 0; x < NW; x++) {
                    sm.eF[r][x][cc] = E;
                    E = zaxpy(sm.bwF[r][x][cc], sm.awF[x][cc], E);
                }
            }
            __syncthreads();
        }
        {
            double2 EF[NR];
#pragma unroll
            for (int r = 0; r < NR; r++) EF[r] = zero;
            if constexpr (!SEQ) {
#pragma unroll
                for (int x = 0; x < NW - 1; x++) {
                    if (x < w) {
                        const double2 a = lds_keep(&sm.AwF[x][c]);
#pragma unroll
                        for (int r = 0; r < NR; r++) EF[r] = zfma(sm.BwF[r][x][c], a, EF[r]);
                    }
                }
            }
            const double2 AeF = lds_keep(tabF + LOG * NT + t);
            double        aeF = 0.0;
            if constexpr (SRC == 6) aeF = lds_keep(ttF + LOG * NT + t);
            double2 y[NR], z[NR];
#pragma unroll
            for (int r = 0; r < NR; r++) {
                y[r] = zfma(Bfe[r], AeF, SEQ ? sm.EF[r][w][c] : EF[r]);
                z[r] = zero;
                if constexpr (SRC == 6) z[r] = zaxpy(bfe[r], aeF, sm.eF[r][w][c]);
            }
            // the rows keep ui_k y_k, so that the back substitution is x_k = ui_k y_k - tau_k x_{k+1}
            double2       tp = PCS ? PC(0) : tau_in;
            const double2 rsv = PCS ? PC(1) : rs;
#pragma unroll
            for (int k = 0; k < KS; k++) {
                double2 u, l;
                if constexpr (KEEP_L) {
                    u = ui[k];
                    l = Lr[k];
                } else {
                    const double2 tk = TV(k);
                    u = cmul(rsv, tk);
                    l = tp;
                    tp = tk;
                }
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    y[r] = zfms(v[r][k], l, y[r]);
                    v[r][k] = cmul(u, y[r]);
                    if constexpr (SRC == 6) {
                        z[r] = make_double2(fma(-PL(k), z[r].x, g[r][k].x), fma(-PL(k), z[r].y, g[r][k].y));
                        g[r][k] = z[r];
                    }
                }
            }
        }

        // ---- back substitution x_r = ui_r y_r - tau_r x_{r+1};  Pade: w_r = pu_r (z_r - w_{r+1})
        double2 xh[NR], wh[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) { xh[r] = zero; wh[r] = zero; }
#pragma unroll
        for (int k = KS - 1; k >= 0; k--) {
#pragma unroll
            for (int r = 0; r < NR; r++) {
                xh[r] = zfms(v[r][k], TAU(k), xh[r]);
                if constexpr (SRC == 6)
                    wh[r] = make_double2(PU(k) * (g[r][k].x - wh[r].x), PU(k) * (g[r][k].y - wh[r].y));
            }
        }
        double2 Bbe[NR], bbe[NR];
#pragma unroll
        for (int r = 0; r < NR; r++) {
            const double2 Bb = sym_warp_scan<CW, false>(xh[r], tabB + t, NT, sl);
            Bbe[r] = shfl_down2(Bb, CW);
            bbe[r] = zero;
            if (sl == 0) sm.BwB[r][w][c] = Bb;
            if constexpr (SRC == 6) {
                const double2 bb = sym_warp_scan<CW, false>(wh[r], ttB + t, NT, sl);
                bbe[r] = shfl_down2(bb, CW);
                if (sl == 0) sm.bwB[r][w][c] = bb;
            }
            if (sl == SPW - 1) { Bbe[r] = zero; bbe[r] = zero; }
        }
        __syncthreads();
        // the value entering each warp from the warps after it, composed from the last one down
        // (as in the forward direction)
        if constexpr (SEQ) {
            if (t < CW * NR) {
                const int r = t / CW, cc = t % CW;
                double2   E = zero;
#pragma unroll
                for (int x = NW - 1; x >= 0; x--) {
                    sm.EB[r][x][cc] = E;
                    E = zfma(sm.BwB[r][x][cc], sm.AwB[x][cc], E);
                }
            } else if (t >= 128 && t < 128 + CW * NR) {
                const int r = (t - 128) / CW, cc = (t - 128) % CW;
                double2   E = zero;
#pragma unroll
                for (int x = NW - 1; x >= 0; x--) {
                    sm.eB[r][x][cc] = E;
                    E = zaxpy(sm.bwB[r][x][cc], sm.awB[x][cc], E);
                }
            }
            __syncthreads();
        }
        {
            double2 EB[NR];
#pragma unroll
            for (int r = 0; r < NR; r++) EB[r] = zero;
            if constexpr (!SEQ) {
#pragma unroll
                for (int xw = NW - 1; xw > 0; xw--) {
                    if (xw > w) {
                        const double2 a = lds_keep(&sm.AwB[xw][c]);
#pragma unroll
                        for (int r = 0; r < NR; r++) EB[r] = zfma(sm.BwB[r][xw][c], a, EB[r]);
                    }
                }
            }
            const double2 AeB = lds_keep(tabB + LOG * NT + t);
            double        aeB = 0.0;
            if constexpr (SRC == 6) aeB = lds_keep(ttB + LOG * NT + t);
            double2 x[NR], ww[NR];
            const double2 cTv = PCS ? PC(3) : cT;
#pragma unroll
            for (int r = 0; r < NR; r++) {
                x[r] = zfma(Bbe[r], AeB, SEQ ? sm.EB[r][w][c] : EB[r]);
                ww[r] = zero;
                if constexpr (SRC == 6) ww[r] = zaxpy(bbe[r], aeB, sm.eB[r][w][c]);
            }
#pragma unroll
            for (int k = KS - 1; k >= 0; k--) {
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    x[r] = zfms(v[r][k], TAU(k), x[r]);
                    v[r][k] = x[r];
                    if constexpr (SRC == 6) {
                        ww[r] = make_double2(PU(k) * (g[r][k].x - ww[r].x), PU(k) * (g[r][k].y - ww[r].y));
                        v[r][k] = zfma(v[r][k], cTv, ww[r]);
                    }
                }
            }
        }

#pragma unroll
        for (int r = 0; r < NR; r++) {
            if (b + r >= b_end) break;
            double2 *dst = out + (long)(b + r) * field + off0;
            if constexpr (PCS) {
                // one running address and a row count re-formed here: per-row offsets and
                // conditions hoisted out of the loop over right-hand sides would pin registers
                long rsd = row_stride;
                int  nk = live ? rows - r0 : 0;
                asm volatile("" : "+l"(rsd), "+r"(nk));
#pragma unroll
                for (int k = 0; k < KS; k++) {
                    if (k < nk) *dst = v[r][k];
                    dst += rsd;
                }
            } else {
#pragma unroll
                for (int k = 0; k < KS; k++)
                    if (live && r0 + k < rows) dst[(long)k * row_stride] = v[r][k];
            }
        }
    }
}

// Stage multipliers of the intra-warp scans for one per-segment multiplier a (complex, or real
// for the Pade solve): tab[j * NT] = the thread's map product before stage j, tab[LOG * NT] =
// the exclusive product.  Returns the inclusive product, which at the warp's last (forward) or
// first (backward) segment is the warp total.
__device__ __forceinline__ double shfl_up1(double v, int off) { return __shfl_up_sync(0xffffffffu, v, off); }
__device__ __forceinline__ double shfl_down1(double v, int off) { return __shfl_down_sync(0xffffffffu, v, off); }
__device__ __forceinline__ double2 shfl_up1(double2 v, int off) { return shfl_up2(v, off); }
__device__ __forceinline__ double2 shfl_down1(double2 v, int off) { return shfl_down2(v, off); }
__device__ __forceinline__ double  mul1(double a, double b) { return a * b; }
__device__ __forceinline__ double2 mul1(double2 a, double2 b) { return cmul(a, b); }

template <int CW, bool FWD, typename M>
__device__ __forceinline__ M sym_scan_table(M a, M *tab, int NT_, int sl, M one) {
    constexpr int SPW = 32 / CW;
    int           j = 0;
#pragma unroll
    for (; (1 << j) < SPW; j++) {
        tab[j * NT_] = a;
        const M o = FWD ? shfl_up1(a, CW << j) : shfl_down1(a, CW << j);
        if (FWD ? (sl >= (1 << j)) : (sl + (1 << j) < SPW)) a = mul1(a, o);
    }
    M e = FWD ? shfl_up1(a, CW) : shfl_down1(a, CW);
    if (FWD ? sl == 0 : sl == SPW - 1) e = one;
    tab[j * NT_] = e;
    return a;
}

// Elements of one TMA tile [rows][cw] (whole 128-byte units), and the rows per box.
__host__ __device__ inline int sym_tile_rows_per_box(int rows) { return rows < 256 ? rows : 256; }
__host__ __device__ inline int sym_tile_elems(int rows, int cw) {
    const int br = sym_tile_rows_per_box(rows), nbox = (rows + br - 1) / br;
    return (nbox * br * cw + 7) / 8 * 8;
}

// Several plans of one shape in one launch (hh_solve_source_multi): chunk j of the grid's y
// dimension solves right-hand sides [b0, b1) of the batch with the factors and wavenumber of plan
// `plan`; everything else (eigenvalues, Pade factors, h) is the same for plans of one shape.
struct SymPlanRef {
    const double2 *Pv, *subt, *diagt;
    double2        k2h2_20;
};
struct SymChunk {
    int plan, b0, b1, pad;
};

template <int SRC, int NT, int CW, int MINB, int NR, int KS, bool TIO>
__global__ void __launch_bounds__(NT, MINB)
    k_line_solve_sym(const double2 *__restrict__ in, double2 *__restrict__ out, int lines, int rows, long row_stride,
                     long field, int batch, int rb, const double2 *__restrict__ Pv_one, const double2 *__restrict__ subt_one,
                     const double2 *__restrict__ diagt_one, int prow, const double *__restrict__ mu, SymParams sp,
                     const __grid_constant__ CUtensorMap in_map, int *err, const SymPlanRef *__restrict__ refs,
                     const SymChunk *__restrict__ chunks) {
    constexpr int NW = NT / 32, SPW = 32 / CW, LOG = ilog2_t<SPW>();
    constexpr int HALO = (SRC == 4 || SRC == 6) ? 1 : 0;
    __shared__ SymSmem<NW, CW, NR> sm;
    extern __shared__ __align__(128) unsigned char dyn_raw[];
    // 128-byte aligned start (tensor copies need it; the allocation carries 128 bytes of slack)
    double2 *dyn = reinterpret_cast<double2 *>(dyn_raw + ((128u - (smem_u32(dyn_raw) & 127u)) & 127u));
    // per-thread prefetch slots [NR][KS + 2][NT], or the input tiles
    const int io_elems = TIO ? sym_tile_elems(rows, CW) * SymTileBufs<SRC>::value : NR * (KS + 2) * NT;
    double2  *pre = dyn;
    double2 *tabF = pre + io_elems;                     // [LOG + 1][NT]
    double2 *tabB = tabF + (LOG + 1) * NT;              // [LOG + 1][NT]
    constexpr bool UIS = SymUIS<SRC, KS>::value;
    double2 *uis = tabB + (LOG + 1) * NT;               // [KS][NT] tau_k (UIS)
    double  *ttF = reinterpret_cast<double *>(uis + (UIS ? KS * NT : 0)); // [LOG + 1][NT] (order 6)
    double  *ttB = ttF + (LOG + 1) * NT;
    (void)HALO;

    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int c = t % CW, seg = t / CW, sl = lane / CW;
    const int q = blockIdx.x * CW + c;
    // this CTA's right-hand sides and the plan they belong to
    int            b_begin, b_end;
    const double2 *Pv = Pv_one, *subt = subt_one, *diagt = diagt_one;
    if (chunks) {
        const SymChunk   ch = chunks[blockIdx.y];
        const SymPlanRef pr = refs[ch.plan];
        b_begin = ch.b0;
        b_end = ch.b1;
        Pv = pr.Pv;
        subt = pr.subt;
        diagt = pr.diagt;
        sp.k2h2_20 = pr.k2h2_20;
    } else {
        b_begin = blockIdx.y * rb;
        b_end = min(batch, b_begin + rb);
    }
    SymTio    tio{};
    if constexpr (TIO) {
        constexpr int NBUF = SymTileBufs<SRC>::value;
        tio.in_map = &in_map;
        tio.tin = pre;
        tio.bar = sm.tbar;
        tio.err = err;
        tio.x0 = blockIdx.x * CW;
        tio.br = sym_tile_rows_per_box(rows);
        tio.nbox = (rows + tio.br - 1) / tio.br;
        tio.tile = sym_tile_elems(rows, CW);
        tio.tile_bytes = (unsigned)(tio.nbox * tio.br * CW * 16);
        if (t == 0) { // the first right-hand sides' tiles come in while the factors are set up
            const int b0 = b_begin, b1 = b_end;
            for (int u = 0; u < NBUF; u++) mbar_init(tio.bar + u, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            for (int u = 0; u < NBUF && b0 + u < b1; u++) {
                double2 *dst = tio.tin + (long)u * tio.tile;
                mbar_expect_tx(tio.bar + u, tio.tile_bytes);
                for (int x = 0; x < tio.nbox; x++)
                    tma_tile_load(dst + (long)x * tio.br * CW, tio.in_map, tio.x0, x * tio.br, b0 + u, tio.bar + u);
            }
        }
    }
    const bool live = q < lines;
    const int  qq = live ? q : 0;
    const int  r0 = seg * KS;
    const double m0 = mu[qq], m1 = mu[lines + qq], m2 = mu[2 * lines + qq];
    const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);

    // ---- factors of the thread's rows (the set-up's recurrence, same arithmetic)
    const double2 s = shifted(subt, prow, 0, m0, m1, m2), d = shifted(diagt, prow, 0, m0, m1, m2);
    double2 Lr[KS], ui[KS];
    double2 Af = one, Ab = one;
    const double2 ui_in = (live && r0 > 0 && r0 < rows) ? Pv[(long)(r0 / 8) * lines + q] : zero; // 1/P of row r0-1
    {
        double2 uprev = ui_in;
#pragma unroll
        for (int k = 0; k < KS; k++) {
            const int r = r0 + k;
            Lr[k] = zero;
            ui[k] = zero;
            if (live && r < rows) {
                if (r == 0) ui[k] = first_pivot(d);
                else ui[k] = factor_step(s, d, s, uprev, Lr[k]);
            }
            uprev = ui[k];
            Af = cmul(Af, make_double2(-Lr[k].x, -Lr[k].y));
            const double2 tau = cmul(s, ui[k]);
            Ab = cmul(Ab, make_double2(-tau.x, -tau.y));
            if constexpr (SRC == 6) { // order 6 keeps tau_k in place of ui_k
                if constexpr (UIS) uis[k * NT + t] = tau;
                else ui[k] = tau;
            }
        }
    }

    // ---- per-line coefficients of the compact right-hand side
    double2 c1 = one, cT = zero;
    double  c2 = 0.0;
    if constexpr (SRC == 4) {
        c1 = make_double2(sp.h2 * (sp.dim == 2 ? (10.0 + m1) / 12.0 : (8.0 + m1 + m2) / 12.0), 0.0);
        c2 = sp.h2 / 12.0;
    } else if constexpr (SRC == 6) {
        double2 a6;
        double  b6;
        if (sp.dim == 2) {
            const double muq = 12.0 * (m1 - 2.0) / (10.0 + m1);
            a6 = make_double2(1.6 + muq / 12.0 + (m1 - 2.0) * muq / 360.0 - sp.k2h2_20.x, -sp.k2h2_20.y);
            b6 = muq / 90.0 + 1.0 / 30.0;
        } else {
            const double mx = 12.0 * (m1 - 2.0) / (10.0 + m1), my = 12.0 * (m2 - 2.0) / (10.0 + m2);
            a6 = make_double2(1.6 + (mx + my) / 12.0 + ((m1 - 2.0) * mx + (m2 - 2.0) * my) / 360.0 +
                                  (m2 - 2.0) * mx / 90.0 - sp.k2h2_20.x,
                              -sp.k2h2_20.y);
            b6 = (mx + my) / 90.0 + 1.0 / 30.0;
        }
        const double2 den = crcp(make_double2(10.0 * s.x - d.x, 10.0 * s.y - d.y)); // 1/(10 s - d)
        const double2 sr = cmul(s, den);
        c1 = make_double2(sp.h2 * (a6.x - 7.2 * sr.x), sp.h2 * (a6.y - 7.2 * sr.y));
        c2 = sp.h2 * b6;
        cT = make_double2(7.2 * sp.h2 * den.x, 7.2 * sp.h2 * den.y);
        if constexpr (SymPCS<SRC, KS, CW>::value) {
            double2 *pcs = reinterpret_cast<double2 *>(ttB + (LOG + 1) * NT);
            pcs[t] = cmul(s, ui_in);
            pcs[NT + t] = crcp(s);
            pcs[2 * NT + t] = c1;
            pcs[3 * NT + t] = cT;
            pcs[4 * NT + t] = make_double2(c2, 0.0);
        }
    }

    // ---- scan tables (factor-only, shared by every right-hand side of the chunk)
    {
        const double2 totF = sym_scan_table<CW, true>(Af, tabF + t, NT, sl, one);
        const double2 totB = sym_scan_table<CW, false>(Ab, tabB + t, NT, sl, one);
        if (sl == SPW - 1) sm.AwF[w][c] = totF;
        if (sl == 0) sm.AwB[w][c] = totB;
    }
    if constexpr (SRC == 6) {
        if (t < 9) {
            sm.pl[t] = sp.pl[t];
            sm.pu[t] = sp.pu[t];
        }
        __syncthreads();
        double af = 1.0, ab = 1.0;
#pragma unroll
        for (int k = 0; k < KS; k++) {
            const int r = r0 + k;
            af *= -(r < 9 ? sm.pl[r] : (r < rows ? sp.linf : 0.0));
            ab *= -(r < 9 ? sm.pu[r] : (r < rows ? sp.uinf : 0.0));
        }
        const double totF = sym_scan_table<CW, true>(af, ttF + t, NT, sl, 1.0);
        const double totB = sym_scan_table<CW, false>(ab, ttB + t, NT, sl, 1.0);
        if (sl == SPW - 1) sm.awF[w][c] = totF;
        if (sl == 0) sm.awB[w][c] = totB;
    }
    __syncthreads();

    const long off0 = (long)r0 * row_stride + qq;
    // warps whose rows all lie in [9, rows) use the constant Pade factors
    const bool tint = (w * SPW * KS >= 9) && ((w + 1) * SPW * KS <= rows);
    if (SRC == 6 && tint)
        sym_chunk<SRC, NT, CW, true, NR, KS, TIO>(in, out, rows, row_stride, field, b_begin, b_end, off0, live, r0, sl,
                                                  w, c, Lr, ui, uis, ui_in, s, c1, c2, cT, sm, pre, tabF, tabB, ttF,
                                                  ttB, sp, tio);
    else
        sym_chunk<SRC, NT, CW, false, NR, KS, TIO>(in, out, rows, row_stride, field, b_begin, b_end, off0, live, r0,
                                                   sl, w, c, Lr, ui, uis, ui_in, s, c1, c2, cT, sm, pre, tabF, tabB,
                                                   ttF, ttB, sp, tio);
}

// Right-hand sides per CTA: the chunk whose grid has the smallest wave-quantised cost,
//   ceil(CTAs / resident CTAs) * (rb + 1),
// counting the per-chunk set-up (factors and scan tables) as about one right-hand side.
static int pick_rb(long groups, int batch, int resident, int nr) {
    int  best = nr, rb = nr;
    long best_cost = -1;
    for (; ; rb *= 2) {
        const int  r = rb < batch ? rb : batch;
        const long ctas = groups * ((batch + r - 1) / r);
        const long cost = ((ctas + resident - 1) / resident) * (long)(r + 1);
        if (best_cost < 0 || cost < best_cost) { best_cost = cost; best = r; }
        if (rb >= batch) break;
    }
    return best;
}

// (re/im, line, row, right-hand side) map of a batch of line-solve fields, boxes of cw lines by
// br rows
static int encode_line_map(CUtensorMap *map, const double2 *base, const Plan *p, int batch, int cw, int br) {
    const unsigned long long dims[4] = {2, (unsigned long long)p->lines, (unsigned long long)p->rows,
                                        (unsigned long long)batch};
    const unsigned long long strides[3] = {16, (unsigned long long)p->row_stride * 16,
                                           (unsigned long long)p->field * 16};
    const unsigned           box[4] = {2, (unsigned)cw, (unsigned)br, 1};
    return encode_tensor_map(map, base, 4, dims, strides, box);
}

// A multi-plan launch: the plans' references and the chunk table, in device memory the caller
// provides, and the chunk count (the grid's y extent).
struct SymMulti {
    const SymPlanRef *refs = nullptr;
    const SymChunk   *chunks = nullptr;
    int               nchunks = 0;
};

template <int SRC, int CW, int MINB, int NR, int KS, bool TIO>
static int launch_sym_t(Plan *p, const double2 *in, double2 *out, int batch, const SymMulti *multi) {
    constexpr int NT = 256, SPW = 32 / CW, LOG = ilog2_t<SPW>();
    SymParams sp;
    sp.h2 = p->h * p->h;
    sp.k2h2_20 = make_double2(p->k2.x * sp.h2 / 20.0, p->k2.y * sp.h2 / 20.0);
    sp.dim = p->dim;
    sp.linf = p->pade_linf;
    sp.uinf = p->pade_uinf;
    sp.pl = p->pade_l;
    sp.pu = p->pade_u;
    const int io_elems = TIO ? sym_tile_elems(p->rows, CW) * SymTileBufs<SRC>::value : NR * (KS + 2) * NT;
    const int shm = 128 + (int)(sizeof(double2) * (io_elems + 2 * (LOG + 1) * NT +
                                                   (SymUIS<SRC, KS>::value ? KS * NT : 0) +
                                                   (SymPCS<SRC, KS, CW>::value ? 5 * NT : 0)) +
                                (SRC == 6 ? sizeof(double) * 2 * (LOG + 1) * NT : 0));
    CUtensorMap in_map{};
    if constexpr (TIO) HH_TRY(encode_line_map(&in_map, in, p, batch, CW, sym_tile_rows_per_box(p->rows)));
    HH_CUDA(cudaFuncSetAttribute(k_line_solve_sym<SRC, NT, CW, MINB, NR, KS, TIO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 shm));
    const long groups = (p->lines + CW - 1) / CW;
    int blocks_per_sm = 0, dev = 0, sms = 148;
    HH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, k_line_solve_sym<SRC, NT, CW, MINB, NR, KS, TIO>, NT,
                                                          shm));
    HH_CUDA(cudaGetDevice(&dev));
    HH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int rb = pick_rb(groups, batch, std::max(1, blocks_per_sm) * sms, NR);
    const int chunks = multi ? multi->nchunks : (batch + rb - 1) / rb;
    dim3 grid((unsigned)groups, (unsigned)chunks);
    k_line_solve_sym<SRC, NT, CW, MINB, NR, KS, TIO><<<grid, NT, shm, p->ctx->stream>>>(
        in, out, p->lines, p->rows, p->row_stride, p->field, batch, rb, p->Pv, p->subt, p->diagt, p->prow, p->mu, sp,
        in_map, p->ctx->err_word, multi ? multi->refs : nullptr, multi ? multi->chunks : nullptr);
    HH_CUDA(cudaGetLastError());
    p->ctx->launches++;
    return HH_OK;
}

// TIO: tile I/O where a line group is at least two lines (32-byte row pieces or wider); one-line
// groups keep the per-thread prefetch.
// segments per line of the symmetric kernel: a power of two P >= rows / KS with 8 <= P <= 256
// (CW = 256 / P lines per CTA); P = 8 runs one right-hand side per pass
static int sym_segments(int rows, int ks) {
    int P = 8;
    while (P * ks < rows) P <<= 1;
    return P;
}

template <int SRC, int MINB, int NR, int KS, bool TIO = false>
static int launch_sym_src(Plan *p, const double2 *in, double2 *out, int batch, const SymMulti *multi) {
    switch (sym_segments(p->rows, KS)) {
    case 8: return launch_sym_t<SRC, 32, MINB, 1, KS, TIO>(p, in, out, batch, multi); // per-RHS scan arrays would not fit
    case 16: return launch_sym_t<SRC, 16, MINB, NR, KS, TIO>(p, in, out, batch, multi);
    case 32: return launch_sym_t<SRC, 8, MINB, NR, KS, TIO>(p, in, out, batch, multi);
    case 64: return launch_sym_t<SRC, 4, MINB, NR, KS, TIO>(p, in, out, batch, multi);
    case 128: return launch_sym_t<SRC, 2, MINB, NR, KS, TIO>(p, in, out, batch, multi); // 32-byte row pieces
    case 256: return launch_sym_t<SRC, 1, MINB, NR, KS, false>(p, in, out, batch, multi);
    default: set_error("symmetric line solve: %d rows", p->rows); return HH_ERR_UNSUPPORTED;
    }
}

// Default symmetric variant of a plan: 2, or 5 where the lines are longer than 8-row segments
// reach (more than 256 * 8 rows), so that such plans keep the symmetric kernel untuned.
int sym_default_variant(int rows) { return rows > 256 * kSeg ? 5 : 2; }

bool sym_solve_supported(const Plan *p, int src_order) {
    const int max_rows = 256 * (p->variant >= 5 ? 16 : kSeg);
    return p->sym && p->rows <= max_rows && (src_order != 6 || (p->pf_ok && p->pade_l));
}

// Variants of the symmetric kernel: 2 = two CTAs per SM, 3 = one CTA per SM (no register cap),
// 4 = one CTA per SM with two right-hand sides per pass, 5 = one CTA per SM with 16-row segments
// (twice the lines per CTA: wider contiguous row pieces in global memory, half the scans; at
// order 6 the reciprocal pivots move to shared memory), 6 = variant 5 with each right-hand side
// brought in as a TMA tile where a CTA holds at least four lines.
template <int SRC>
static int launch_sym_variant(Plan *p, const double2 *in, double2 *out, int batch, const SymMulti *multi) {
    switch (p->variant) {
    case 3: return launch_sym_src<SRC, 1, 1, kSeg>(p, in, out, batch, multi);
    case 4: return launch_sym_src<SRC, 1, 2, kSeg>(p, in, out, batch, multi);
    case 5: return launch_sym_src<SRC, 1, 1, 16>(p, in, out, batch, multi);
    case 6: return launch_sym_src<SRC, 1, 1, 16, true>(p, in, out, batch, multi);
    default: return launch_sym_src<SRC, 2, 1, kSeg>(p, in, out, batch, multi);
    }
}

static int launch_sym_order(Plan *p, const double2 *in, double2 *out, int batch, int src_order, const SymMulti *multi) {
    switch (src_order) {
    case 0: return launch_sym_variant<0>(p, in, out, batch, multi);
    case 2: return launch_sym_variant<2>(p, in, out, batch, multi);
    case 4: return launch_sym_variant<4>(p, in, out, batch, multi);
    case 6: return launch_sym_variant<6>(p, in, out, batch, multi);
    default: set_error("source operator order %d", src_order); return HH_ERR_INVALID;
    }
}

int launch_line_solve_sym(Plan *p, const double2 *in, double2 *out, int batch, int src_order) {
    return launch_sym_order(p, in, out, batch, src_order, nullptr);
}

size_t line_solve_multi_table_bytes(int nplans, int total) {
    return sizeof(SymPlanRef) * (size_t)nplans + sizeof(SymChunk) * (size_t)(total + nplans);
}

// One symmetric line-solve launch over the right-hand sides of several plans of one shape: plan i
// solves nrhs[i] consecutive fields of the batch (plans in order).  Every plan must take the
// symmetric kernel with the same variant; table_dev (line_solve_multi_table_bytes) receives the
// plan references and the chunk table in stream order.  Returns HH_ERR_UNSUPPORTED when the plans
// do not qualify, before launching anything.
int launch_line_solve_multi(Plan *const *plans, const int *nrhs, int nplans, const double2 *in, double2 *out,
                            int src_order, void *table_dev) {
    Plan *p0 = plans[0];
    for (int i = 0; i < nplans; i++) {
        const Plan *pi = plans[i];
        if (pi->variant < 2 || pi->variant != p0->variant || !sym_solve_supported(pi, src_order)) {
            set_error("multi-plan line solve: plan %d does not take the symmetric kernel variant %d", i, p0->variant);
            return HH_ERR_UNSUPPORTED;
        }
    }
    int total = 0;
    for (int i = 0; i < nplans; i++) total += nrhs[i];
    if (total == 0) return HH_OK;
    // right-hand sides per chunk: the single-plan choice for the whole batch, chunks never
    // crossing a plan boundary
    const int ks = (p0->variant >= 5) ? 16 : kSeg;
    const int P = sym_segments(p0->rows, ks), CW = 256 / P, nr = (p0->variant == 4 && P > 8) ? 2 : 1;
    const long groups = (p0->lines + CW - 1) / CW;
    int dev = 0, sms = 148;
    HH_CUDA(cudaGetDevice(&dev));
    HH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int rb = pick_rb(groups, total, (p0->variant == 2 ? 2 : 1) * sms, nr);
    std::vector<SymPlanRef> refs((size_t)nplans);
    std::vector<SymChunk>   chunks;
    for (int i = 0, b = 0; i < nplans; b += nrhs[i], i++) {
        const Plan *pi = plans[i];
        const double h2 = pi->h * pi->h;
        refs[(size_t)i] = SymPlanRef{pi->Pv, pi->subt, pi->diagt, make_double2(pi->k2.x * h2 / 20.0, pi->k2.y * h2 / 20.0)};
        for (int b0 = b; b0 < b + nrhs[i]; b0 += rb) chunks.push_back(SymChunk{i, b0, std::min(b + nrhs[i], b0 + rb), 0});
    }
    if (chunks.size() > 65535) {
        set_error("multi-plan line solve: %zu chunks", chunks.size());
        return HH_ERR_UNSUPPORTED;
    }
    char *tab = static_cast<char *>(table_dev);
    HH_CUDA(cudaMemcpyAsync(tab, refs.data(), sizeof(SymPlanRef) * refs.size(), cudaMemcpyHostToDevice, p0->ctx->stream));
    HH_CUDA(cudaMemcpyAsync(tab + sizeof(SymPlanRef) * refs.size(), chunks.data(), sizeof(SymChunk) * chunks.size(),
                            cudaMemcpyHostToDevice, p0->ctx->stream));
    SymMulti m;
    m.refs = reinterpret_cast<const SymPlanRef *>(tab);
    m.chunks = reinterpret_cast<const SymChunk *>(tab + sizeof(SymPlanRef) * refs.size());
    m.nchunks = (int)chunks.size();
    return launch_sym_order(p0, in, out, total, src_order, &m);
}

} // namespace hh
