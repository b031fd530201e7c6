// FP64 residual of the compact operator, and the update step of the refined form.
//
// k_residual computes res = A_h u - rhs for a plan's stencil with a zero Dirichlet ring, as the
// reference's residual() does on the host:
//   2D  2D_Program/main_functions/residual.c:3-34  (9-point stencil, per-row
//       coefficients [bm am bm; b a b; bp ap bp] of the centre row j),
//   3D  3D_Program/main_functions/residual.c:42-96 (27-point stencil, per-layer coefficients
//       a..dm of the centre layer l: corners, x-neighbours, y-neighbours, centre).
// The plan keeps those coefficients as its line-solve tables: subt / diagt / rowc hold, for the
// layer below / the same layer / the layer above, [corner, x-neighbour, y-neighbour, centre]
// at [t * prow + row].  In 2D the corner and y-neighbour entries are zero.
//
// A block takes whole rows of n0 points (x fastest, so the loads of a warp are contiguous), with
// its layer's coefficients loaded once per row and no division per point; neighbours come
// through L1/L2.  The pass is bound by HBM: 48 bytes per point (read u and rhs, write res),
// plus the neighbour re-reads the caches absorb.
#include "hh_internal.cuh"

#include <algorithm>

namespace hh {

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *a, double v) {
    // non-negative doubles order as their bit patterns
    atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

template <bool D3>
__global__ void __launch_bounds__(256)
    k_residual(const double2 *__restrict__ u, const double2 *__restrict__ rhs, double2 *__restrict__ res, int n0,
               int n1, int n2, long field, int prow, const double2 *__restrict__ subt,
               const double2 *__restrict__ diagt, const double2 *__restrict__ supt, unsigned long long *norms) {
    const long     b = blockIdx.y;
    const double2 *ub = u + b * field;
    const double2  zero = make_double2(0.0, 0.0);
    const long     plane = (long)n0 * n1;
    const long     nrows = D3 ? (long)n1 * n2 : (long)n2; // rows of n0 points (x fastest)
    double         mr = 0.0, mf = 0.0; // squared moduli; the root is taken once per block
    auto ld = [&](const double2 *q, bool ok) { return ok ? __ldg(q) : zero; };
    // one row of n0 points per pass of the block: its layer's coefficients once, no division per point
    for (long R = blockIdx.x; R < nrows; R += gridDim.x) {
        const int  j = D3 ? (int)(R % n1) : 0;
        const int  r = D3 ? (int)(R / n1) : (int)R;
        const long row0 = (long)r * plane + (long)j * n0;
        const bool yl = D3 && j > 0, yr = D3 && j + 1 < n1;
        double2    cf[3][4]; // layer below / same / above: corner, x-neighbour, y-neighbour, centre
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double2 *T = d == 0 ? subt : (d == 1 ? diagt : supt);
#pragma unroll
            for (int q = 0; q < 4; q++) cf[d][q] = __ldg(T + q * prow + r);
        }
        for (int i = threadIdx.x; i < n0; i += blockDim.x) {
            const long p = row0 + i;
            const bool xl = i > 0, xr = i + 1 < n0;
            double2    acc = zero;
#pragma unroll
            for (int dr = -1; dr <= 1; dr++) {
                if (r + dr < 0 || r + dr >= n2) continue; // the zero Dirichlet layer
                const double2(&T)[4] = cf[dr + 1];
                const double2 *c = ub + p + dr * plane;    // the neighbour (i, j, r + dr)
                const double2  xs = cadd(ld(c - 1, xl), ld(c + 1, xr));
                acc = cadd(acc, cmul(T[3], __ldg(c)));
                acc = cadd(acc, cmul(T[1], xs));
                if constexpr (D3) {
                    const double2 ys = cadd(ld(c - n0, yl), ld(c + n0, yr));
                    const double2 corners = cadd(cadd(ld(c - n0 - 1, yl && xl), ld(c - n0 + 1, yl && xr)),
                                                 cadd(ld(c + n0 - 1, yr && xl), ld(c + n0 + 1, yr && xr)));
                    acc = cadd(acc, cmul(T[0], corners));
                    acc = cadd(acc, cmul(T[2], ys));
                }
            }
            const double2 f = __ldg(rhs + b * field + p);
            const double2 rv = csub(acc, f);
            res[b * field + p] = rv;
            if (norms) {
                mr = fmax(mr, fma(rv.x, rv.x, rv.y * rv.y));
                mf = fmax(mf, fma(f.x, f.x, f.y * f.y));
            }
        }
    }
    if (norms) {
        // block maxima, then one atomic per block
        __shared__ double sr[8], sf[8];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, off));
            mf = fmax(mf, __shfl_xor_sync(0xffffffffu, mf, off));
        }
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) { sr[w] = mr; sf[w] = mf; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int x = 1; x < (int)(blockDim.x >> 5); x++) { mr = fmax(mr, sr[x]); mf = fmax(mf, sf[x]); }
            atomic_max_nonneg(norms, sqrt(mr));
            atomic_max_nonneg(norms + 1, sqrt(mf));
        }
    }
}

// 3D, tiled: a block owns a kRTX x kRTY tile of the (x, y) plane over layers [z0, z0 + kRZ) and
// keeps layers r - 1, r, r + 1 of the tile with a one-point halo in shared memory (a ring of
// three, zero outside the field), so that each value of u is read from global memory about once
// instead of through the caches 27 times.  At 32 registers eight blocks share an SM, which hides
// the layer loads; forms that keep neighbourhoods or partial sums in registers to read shared
// memory less ran slower (fewer blocks per SM).  The sum runs in the order of k_residual, term by
// term (a zero-filled neighbour contributes an exact zero).
constexpr int kRTX = 32, kRTY = 8, kRZ = 64;
__global__ void __launch_bounds__(kRTX * kRTY)
    k_residual3d_tiled(const double2 *__restrict__ u, const double2 *__restrict__ rhs, double2 *__restrict__ res,
                       int n0, int n1, int n2, long field, int prow, const double2 *__restrict__ subt,
                       const double2 *__restrict__ diagt, const double2 *__restrict__ supt, int zchunks,
                       unsigned long long *norms) {
    __shared__ double2 ring[3][kRTY + 2][kRTX + 2];
    const int      tx = threadIdx.x % kRTX, ty = threadIdx.x / kRTX;
    const int      x0 = blockIdx.x * kRTX, y0 = blockIdx.y * kRTY;
    const long     b = blockIdx.z / zchunks;
    const int      z0 = (int)(blockIdx.z % zchunks) * kRZ, z1 = min(n2, z0 + kRZ);
    const long     plane = (long)n0 * n1;
    const double2 *ub = u + b * field;
    const double2  zero = make_double2(0.0, 0.0);
    const int      gx = x0 + tx, gy = y0 + ty;
    const bool     mine = gx < n0 && gy < n1;
    double         mr = 0.0, mf = 0.0;
    auto load_layer = [&](int r, int slot) { // tile of layer r with its halo, zeros outside the field
        for (int e = threadIdx.x; e < (kRTY + 2) * (kRTX + 2); e += kRTX * kRTY) {
            const int ly = e / (kRTX + 2), lx = e % (kRTX + 2);
            const int x = x0 + lx - 1, y = y0 + ly - 1;
            ring[slot][ly][lx] = (r >= 0 && r < n2 && x >= 0 && x < n0 && y >= 0 && y < n1)
                                     ? __ldg(ub + (long)r * plane + (long)y * n0 + x)
                                     : zero;
        }
    };
    if (z0 < n2) {
        load_layer(z0 - 1, (z0 + 2) % 3);
        load_layer(z0, z0 % 3);
    }
    for (int r = z0; r < z1; r++) {
        load_layer(r + 1, (r + 1) % 3);
        __syncthreads();
        if (mine) {
            double2 acc = zero;
#pragma unroll
            for (int dr = -1; dr <= 1; dr++) {
                if (r + dr < 0 || r + dr >= n2) continue; // the zero Dirichlet layer
                const double2 *T = dr < 0 ? subt : (dr == 0 ? diagt : supt);
                const double2(&L)[kRTY + 2][kRTX + 2] = ring[(r + dr + 3) % 3];
                const int     cy = ty + 1, cx = tx + 1;
                const double2 xs = cadd(L[cy][cx - 1], L[cy][cx + 1]);
                acc = cadd(acc, cmul(__ldg(T + 3 * prow + r), L[cy][cx]));
                acc = cadd(acc, cmul(__ldg(T + prow + r), xs));
                const double2 ys = cadd(L[cy - 1][cx], L[cy + 1][cx]);
                const double2 corners = cadd(cadd(L[cy - 1][cx - 1], L[cy - 1][cx + 1]), cadd(L[cy + 1][cx - 1], L[cy + 1][cx + 1]));
                acc = cadd(acc, cmul(__ldg(T + r), corners));
                acc = cadd(acc, cmul(__ldg(T + 2 * prow + r), ys));
            }
            const long    pidx = b * field + (long)r * plane + (long)gy * n0 + gx;
            const double2 f = __ldg(rhs + pidx);
            const double2 rv = csub(acc, f);
            res[pidx] = rv;
            if (norms) {
                mr = fmax(mr, fma(rv.x, rv.x, rv.y * rv.y));
                mf = fmax(mf, fma(f.x, f.x, f.y * f.y));
            }
        }
        __syncthreads(); // the slot of layer r - 1 takes layer r + 2 next
    }
    if (norms) {
        __shared__ double sr[8], sf[8];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, off));
            mf = fmax(mf, __shfl_xor_sync(0xffffffffu, mf, off));
        }
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) { sr[w] = mr; sf[w] = mf; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int x = 1; x < (int)(blockDim.x >> 5); x++) { mr = fmax(mr, sr[x]); mf = fmax(mf, sf[x]); }
            atomic_max_nonneg(norms, sqrt(mr));
            atomic_max_nonneg(norms + 1, sqrt(mf));
        }
    }
}

// 2D, tiled: a block owns kR2X consecutive points of the rows [z0, z0 + kRZ) and keeps rows
// r - 1, r, r + 1 of that span with a one-point halo in shared memory (a ring of three, zero
// outside the field), so that each value of u is read from global memory about once.  The sum
// runs in the order of k_residual.
constexpr int kR2X = 256;
__global__ void __launch_bounds__(kR2X)
    k_residual2d_tiled(const double2 *__restrict__ u, const double2 *__restrict__ rhs, double2 *__restrict__ res,
                       int n0, int n2, long field, int prow, const double2 *__restrict__ subt,
                       const double2 *__restrict__ diagt, const double2 *__restrict__ supt, int zchunks,
                       unsigned long long *norms) {
    __shared__ double2 ring[3][kR2X + 2];
    const int      x0 = blockIdx.x * kR2X, gx = x0 + threadIdx.x;
    const long     b = blockIdx.y / zchunks;
    const int      z0 = (int)(blockIdx.y % zchunks) * kRZ, z1 = min(n2, z0 + kRZ);
    const double2 *ub = u + b * field;
    const double2  zero = make_double2(0.0, 0.0);
    const bool     mine = gx < n0;
    double         mr = 0.0, mf = 0.0;
    auto load_row = [&](int r, int slot) { // the span of row r with its halo, zeros outside the field
        for (int e = threadIdx.x; e < kR2X + 2; e += kR2X) {
            const int x = x0 + e - 1;
            ring[slot][e] = (r >= 0 && r < n2 && x >= 0 && x < n0) ? __ldg(ub + (long)r * n0 + x) : zero;
        }
    };
    if (z0 < n2) {
        load_row(z0 - 1, (z0 + 2) % 3);
        load_row(z0, z0 % 3);
    }
    for (int r = z0; r < z1; r++) {
        load_row(r + 1, (r + 1) % 3);
        __syncthreads();
        if (mine) {
            double2 acc = zero;
#pragma unroll
            for (int dr = -1; dr <= 1; dr++) {
                if (r + dr < 0 || r + dr >= n2) continue; // the zero Dirichlet row
                const double2 *T = dr < 0 ? subt : (dr == 0 ? diagt : supt);
                const double2 *L = ring[(r + dr + 3) % 3];
                const int      cx = threadIdx.x + 1;
                const double2  xs = cadd(L[cx - 1], L[cx + 1]);
                acc = cadd(acc, cmul(__ldg(T + 3 * prow + r), L[cx]));
                acc = cadd(acc, cmul(__ldg(T + prow + r), xs));
            }
            const long    pidx = b * field + (long)r * n0 + gx;
            const double2 f = __ldg(rhs + pidx);
            const double2 rv = csub(acc, f);
            res[pidx] = rv;
            if (norms) {
                mr = fmax(mr, fma(rv.x, rv.x, rv.y * rv.y));
                mf = fmax(mf, fma(f.x, f.x, f.y * f.y));
            }
        }
        __syncthreads(); // the slot of row r - 1 takes row r + 2 next
    }
    if (norms) {
        __shared__ double sr[8], sf[8];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, off));
            mf = fmax(mf, __shfl_xor_sync(0xffffffffu, mf, off));
        }
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) { sr[w] = mr; sf[w] = mf; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int x = 1; x < (int)(blockDim.x >> 5); x++) { mr = fmax(mr, sr[x]); mf = fmax(mf, sf[x]); }
            atomic_max_nonneg(norms, sqrt(mr));
            atomic_max_nonneg(norms + 1, sqrt(mf));
        }
    }
}

int launch_residual(Plan *p, const double2 *u, const double2 *rhs, double2 *res, int batch,
                    unsigned long long *norms) {
    if (p->dim == 2) {
        const int zchunks = (p->ny + kRZ - 1) / kRZ;
        if ((long)batch * zchunks <= 65535) {
            dim3 grid((unsigned)((p->nx + kR2X - 1) / kR2X), (unsigned)(batch * zchunks));
            k_residual2d_tiled<<<grid, kR2X, 0, p->ctx->stream>>>(u, rhs, res, p->nx, p->ny, p->field, p->prow, p->subt,
                                                                   p->diagt, p->rowc, zchunks, norms);
            HH_CUDA(cudaGetLastError());
            p->ctx->launches++;
            return HH_OK;
        }
    }
    if (p->dim == 3) {
        const int zchunks = (p->nz + kRZ - 1) / kRZ;
        if ((long)batch * zchunks <= 65535 && (p->ny + kRTY - 1) / kRTY <= 65535) {
            dim3 grid((unsigned)((p->nx + kRTX - 1) / kRTX), (unsigned)((p->ny + kRTY - 1) / kRTY),
                      (unsigned)(batch * zchunks));
            k_residual3d_tiled<<<grid, kRTX * kRTY, 0, p->ctx->stream>>>(u, rhs, res, p->nx, p->ny, p->nz, p->field,
                                                                          p->prow, p->subt, p->diagt, p->rowc, zchunks,
                                                                          norms);
            HH_CUDA(cudaGetLastError());
            p->ctx->launches++;
            return HH_OK;
        }
    }
    const int  n0 = p->nx, n1 = p->dim == 3 ? p->ny : 1, n2 = p->dim == 3 ? p->nz : p->ny;
    const long rows = (long)n1 * n2; // rows of n0 points per field, one per block pass
    const long blocks = std::min<long>(rows, std::max<long>(1, 148L * 8 / std::max(1, batch)) * 4);
    dim3       grid((unsigned)blocks, (unsigned)batch);
    if (p->dim == 3)
        k_residual<true><<<grid, 256, 0, p->ctx->stream>>>(u, rhs, res, n0, n1, n2, p->field, p->prow, p->subt,
                                                          p->diagt, p->rowc, norms);
    else
        k_residual<false><<<grid, 256, 0, p->ctx->stream>>>(u, rhs, res, n0, n1, n2, p->field, p->prow, p->subt,
                                                           p->diagt, p->rowc, norms);
    HH_CUDA(cudaGetLastError());
    p->ctx->launches++;
    return HH_OK;
}

// u += s v over n complex values (s real)
__global__ void __launch_bounds__(256) k_axpy(double2 *__restrict__ u, const double2 *__restrict__ v, double s, long n) {
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
        const double2 a = u[k], b = __ldg(v + k);
        u[k] = make_double2(fma(s, b.x, a.x), fma(s, b.y, a.y));
    }
}

int launch_axpy(Ctx *c, double2 *u, const double2 *v, double s, long n) {
    const long blocks = std::min<long>((n + 255) / 256, 148L * 16);
    k_axpy<<<(unsigned)blocks, 256, 0, c->stream>>>(u, v, s, n);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

} // namespace hh
