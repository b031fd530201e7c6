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
// One thread per point (x fastest, so the loads of a warp are contiguous); neighbours come
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
    double         mr = 0.0, mf = 0.0; // squared moduli; the root is taken once per block
    auto ld = [&](const double2 *q, bool ok) { return ok ? __ldg(q) : zero; };
    for (long p = (long)blockIdx.x * blockDim.x + threadIdx.x; p < field; p += (long)gridDim.x * blockDim.x) {
        const int  i = (int)(p % n0);
        const long rest = p / n0;
        const int  j = D3 ? (int)(rest % n1) : 0;
        const int  r = D3 ? (int)(rest / n1) : (int)rest;
        const bool xl = i > 0, xr = i + 1 < n0, yl = D3 && j > 0, yr = D3 && j + 1 < n1;
        double2    acc = zero;
#pragma unroll
        for (int dr = -1; dr <= 1; dr++) {
            if (r + dr < 0 || r + dr >= n2) continue; // the zero Dirichlet layer
            const double2 *T = dr < 0 ? subt : (dr == 0 ? diagt : supt);
            const double2 *c = ub + p + dr * plane;    // the neighbour (i, j, r + dr)
            const double2  xs = cadd(ld(c - 1, xl), ld(c + 1, xr));
            acc = cadd(acc, cmul(__ldg(T + 3 * prow + r), __ldg(c)));
            acc = cadd(acc, cmul(__ldg(T + prow + r), xs));
            if constexpr (D3) {
                const double2 ys = cadd(ld(c - n0, yl), ld(c + n0, yr));
                const double2 corners = cadd(cadd(ld(c - n0 - 1, yl && xl), ld(c - n0 + 1, yl && xr)),
                                             cadd(ld(c + n0 - 1, yr && xl), ld(c + n0 + 1, yr && xr)));
                acc = cadd(acc, cmul(__ldg(T + r), corners));
                acc = cadd(acc, cmul(__ldg(T + 2 * prow + r), ys));
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

int launch_residual(Plan *p, const double2 *u, const double2 *rhs, double2 *res, int batch,
                    unsigned long long *norms) {
    const int  n0 = p->nx, n1 = p->dim == 3 ? p->ny : 1, n2 = p->dim == 3 ? p->nz : p->ny;
    const long blocks = std::min<long>((p->field + 255) / 256, 148L * 8);
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
