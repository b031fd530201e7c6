// Orthonormal DST-I kernels for sm_100a (FP64 complex).
//
// Replaces the reference's transform step: 2D_Program/solver_functions/DST.c:6-44
// (forwardDST / reverseDST: per row, two zero-padded real FFTs of length 2N+2 through
// FFTW) and 3D_Program/solver_functions/DST.c:148-204 plus cuda_kernels.cu:23-176 (the 3D
// plane transform: cuFFT D2Z batches around six staging kernels).
//
// Algorithm (for M = N + 1 a power of two).  The DST-I of complex x_1..x_{M-1}
//     S_k = sum_j x_j sin(pi j k / M)
// is obtained from ONE complex FFT of length M (instead of the reference's two real FFTs
// of length 2M per row):
//     y_0 = 0,  y_j = sin(pi j/M) (x_j + x_{M-j}) + (x_j - x_{M-j})/2
//     Y   = FFT_M(y)                         (e^{-2 pi i jk/M})
//     S_2k    = (Y_{M-k} - Y_k) / (2i)                     k = 1..M/2-1
//     S_2k+1  = Y_0/2 + sum_{q=1..k} (Y_q + Y_{M-q}) / 2     k = 0..M/2-1
// i.e. the symmetric part of y carries the odd outputs as first differences (recovered by a
// block-wide prefix sum) and the antisymmetric part carries the even outputs directly.
// Result scaled by sqrt(2/M) (orthonormal, self-inverse).
//
// Kernel structure: a "slot" of T threads owns one line of length N; each thread keeps
// R = M/T values in registers.  The line arrives by a TMA bulk copy (cp.async.bulk) into
// shared memory (contiguous rows) or by coalesced cooperative loads (strided columns), the
// first radix-R pass runs straight from the pre-processing in registers, later Stockham
// passes exchange through a padded shared buffer (one 16-byte pad per 16 elements keeps
// the 16-byte accesses of each quarter-warp on distinct banks).  FP64 values are exchanged
// through shared memory rather than warp shuffles: a shuffle moves 32 bits, so a complex
// double costs four shuffles per hop.
#include "hh_internal.cuh"
#include "hh_tma.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <math.h>

#include <algorithm>

namespace hh {

// ----------------------------------------------------------- in-register DFT ------
// cos/sin(2 pi t / 16) as compile-time constants
template <int t> struct Tw16;
#define HH_TW(t, c, s) \
    template <> struct Tw16<t> { static constexpr double C = c; static constexpr double S = s; };
HH_TW(0, 1.0, 0.0)
HH_TW(1, 0.9238795325112867, 0.3826834323650898)
HH_TW(2, 0.7071067811865476, 0.7071067811865476)
HH_TW(3, 0.3826834323650898, 0.9238795325112867)
HH_TW(4, 0.0, 1.0)
HH_TW(5, -0.3826834323650898, 0.9238795325112867)
HH_TW(6, -0.7071067811865476, 0.7071067811865476)
HH_TW(7, -0.9238795325112867, 0.3826834323650898)
#undef HH_TW

// v * exp(-2 pi i t / 16)
template <int t> __device__ __forceinline__ double2 tw16_mul(double2 v) {
    if constexpr (t == 0) return v;
    else if constexpr (t == 4) return make_double2(v.y, -v.x);
    else if constexpr (t == 2) {
        constexpr double r = Tw16<2>::C;
        return make_double2((v.x + v.y) * r, (v.y - v.x) * r);
    } else if constexpr (t == 6) {
        constexpr double r = Tw16<2>::C;
        return make_double2((v.y - v.x) * r, -(v.x + v.y) * r);
    } else {
        constexpr double c = Tw16<t>::C, s = Tw16<t>::S;
        return make_double2(fma(v.x, c, v.y * s), fma(v.y, c, -(v.x * s)));
    }
}

template <int R> __host__ __device__ constexpr int ilog2c() { return R <= 1 ? 0 : 1 + ilog2c<R / 2>(); }
template <int R> __host__ __device__ constexpr int bitrev_c(int i) {
    int r = 0;
    for (int b = 0; b < ilog2c<R>(); b++) r |= ((i >> b) & 1) << (ilog2c<R>() - 1 - b);
    return r;
}

// One radix-2 DIF stage at compile-time span, then recurse.  Output in bit-reversed order.
template <int R, int SPAN, int J> struct DifButterflies {
    __device__ __forceinline__ static void run(double2 (&v)[R], int start) {
        if constexpr (J < SPAN) {
            double2 a = v[start + J], b = v[start + J + SPAN];
            v[start + J] = cadd(a, b);
            // exp(-2 pi i J / (2 SPAN)) = exp(-2 pi i (J * 16/(2 SPAN)) / 16)
            v[start + J + SPAN] = tw16_mul<J * (16 / (2 * SPAN))>(csub(a, b));
            DifButterflies<R, SPAN, J + 1>::run(v, start);
        }
    }
};
template <int R, int SPAN, int START> struct DifStage {
    __device__ __forceinline__ static void run(double2 (&v)[R]) {
        if constexpr (START < R) {
            DifButterflies<R, SPAN, 0>::run(v, START);
            DifStage<R, SPAN, START + 2 * SPAN>::run(v);
        }
    }
};
template <int R, int SPAN> struct DifAll {
    __device__ __forceinline__ static void run(double2 (&v)[R]) {
        if constexpr (SPAN >= 1) {
            DifStage<R, SPAN, 0>::run(v);
            DifAll<R, SPAN / 2>::run(v);
        }
    }
};
// forward DFT of R <= 16 points; result X[q] = v[bitrev_c<R>(q)]
template <int R> __device__ __forceinline__ void dft_reg(double2 (&v)[R]) { DifAll<R, R / 2>::run(v); }

// ------------------------------------------------------------ configuration -------
__host__ __device__ constexpr int pad_idx(int i) { return i + (i >> 4); }

template <int M> struct DstCfg;
// T threads per line, R = M/T values per thread, radix schedule R1 (= R), R2, R3, R4
template <> struct DstCfg<64>   { static constexpr int T = 8,   R2 = 8,  R3 = 1,  R4 = 1; };
template <> struct DstCfg<128>  { static constexpr int T = 16,  R2 = 8,  R3 = 2,  R4 = 1; };
template <> struct DstCfg<256>  { static constexpr int T = 32,  R2 = 8,  R3 = 4,  R4 = 1; };
template <> struct DstCfg<512>  { static constexpr int T = 64,  R2 = 8,  R3 = 8,  R4 = 1; };
template <> struct DstCfg<1024> { static constexpr int T = 64,  R2 = 8,  R3 = 8,  R4 = 1; };
template <> struct DstCfg<2048> { static constexpr int T = 128, R2 = 16, R3 = 8,  R4 = 1; };
template <> struct DstCfg<4096> { static constexpr int T = 256, R2 = 16, R3 = 16, R4 = 1; };
template <> struct DstCfg<8192> { static constexpr int T = 512, R2 = 16, R3 = 16, R4 = 2; };

constexpr int kDstThreads = 256;

template <int M> struct DstGeom {
    static constexpr int T = DstCfg<M>::T;
    static constexpr int R = M / T;
    static constexpr int S = (kDstThreads / T) > 0 ? kDstThreads / T : 1; // lines per CTA
    static constexpr int NT = S * T;                                     // threads per CTA
    static constexpr int PADN = M + M / 16;                              // padded elements
    static constexpr int SLOT_BYTES = PADN * 16 + 16;                    // +16: bank skew
    static constexpr int WARPS = (T + 31) / 32;
    static constexpr int HDR = 16 * S + 16 * S * WARPS;                  // mbarriers + scan
    static constexpr int SMEM = HDR + S * SLOT_BYTES;
};

// ------------------------------------------------------------- primitives ---------
template <int T> __device__ __forceinline__ void slot_sync(int slot) {
    if constexpr (T <= 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(slot + 1), "r"(T) : "memory");
    }
}

// one Stockham pass of radix RAD at stride NS over the padded slot buffer
template <int M, int T, int RAD, int NS>
__device__ __forceinline__ void stockham_pass(double2 *buf, const double2 *__restrict__ tw, int t, int slot) {
    constexpr int NB = (M / RAD) / T; // butterflies per thread
    static_assert(NB >= 1, "radix too large for this thread count");
    double2 v[NB][RAD];
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int b = t + T * u;
#pragma unroll
        for (int q = 0; q < RAD; q++) v[u][q] = buf[pad_idx(b + q * (M / RAD))];
    }
    slot_sync<T>(slot);
#pragma unroll
    for (int u = 0; u < NB; u++) {
        const int b = t + T * u;
        const int bm = b & (NS - 1);
        if constexpr (NS > 1) {
#pragma unroll
            for (int q = 1; q < RAD; q++) v[u][q] = cmul(v[u][q], __ldg(tw + q * bm * (M / (NS * RAD))));
        }
        dft_reg<RAD>(v[u]);
        const int dst = (b - bm) * RAD + bm;
#pragma unroll
        for (int q = 0; q < RAD; q++) buf[pad_idx(dst + q * NS)] = v[u][bitrev_c<RAD>(q)];
    }
    slot_sync<T>(slot);
}

// inclusive scan across the T threads of a slot (complex), using `red` (WARPS entries)
template <int T>
__device__ __forceinline__ double2 slot_scan_inclusive(double2 x, int t, int slot, double2 *red) {
    constexpr int W = (T < 32) ? T : 32;
    const int lane = t & (W - 1);
#pragma unroll
    for (int off = 1; off < W; off <<= 1) {
        double ox = __shfl_up_sync(0xffffffffu, x.x, off, W);
        double oy = __shfl_up_sync(0xffffffffu, x.y, off, W);
        if (lane >= off) { x.x += ox; x.y += oy; }
    }
    if constexpr (T > 32) {
        const int w = t >> 5;
        if (lane == 31) red[w] = x;
        slot_sync<T>(slot);
        double2 pre = make_double2(0.0, 0.0);
        for (int q = 0; q < w; q++) pre = cadd(pre, red[q]);
        x = cadd(x, pre);
        slot_sync<T>(slot);
    }
    return x;
}

// ------------------------------------------------------------------- kernel -------
// Line s of the CTA is line (blockIdx.x*S + s) of plane blockIdx.y.  Its element j lives at
//   IN_STRIDED = false:  in + plane*in_plane + line*in_ld + j        (contiguous rows)
//   IN_STRIDED = true :  in + plane*in_plane + line + j*in_ld        (columns; S neighbouring
//                        lines are loaded together, S*16 contiguous bytes per j)
// and likewise for the output with OUT_STRIDED / out_ld / out_plane.  Rows in + columns out
// writes the transform transposed (each output line contiguous in the other direction).
template <int M, bool IN_STRIDED, bool OUT_STRIDED>
__global__ void __launch_bounds__(DstGeom<M>::NT)
    k_dst1(const double2 *__restrict__ in, double2 *__restrict__ out, long nlines, long in_ld, long out_ld,
           long in_plane, long out_plane, const double2 *__restrict__ tw, const double *__restrict__ sn,
           int *err) {
    using G = DstGeom<M>;
    constexpr int T = G::T, R = G::R, S = G::S, N = M - 1;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
    double2  *red_all = reinterpret_cast<double2 *>(smem + 16 * S);
    const int slot = threadIdx.x / T, t = threadIdx.x % T;
    double2  *buf = reinterpret_cast<double2 *>(smem + G::HDR + slot * G::SLOT_BYTES);
    double2  *red = red_all + slot * G::WARPS;

    const long line = (long)blockIdx.x * S + slot;
    const bool live = line < nlines;
    const long ibase = (long)blockIdx.y * in_plane, obase = (long)blockIdx.y * out_plane;

    // ---- stage the line into shared memory (unpadded, x_j at buf[j-1])
    if constexpr (!IN_STRIDED) {
        if (threadIdx.x < S) mbar_init(&bars[threadIdx.x], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        __syncthreads();
        if (t == 0 && live) {
            mbar_expect_tx(&bars[slot], N * 16);
            tma_bulk_load(buf, in + ibase + line * in_ld, N * 16, &bars[slot]);
        }
        if (live) {
            // A copy that never lands is reported through `err`; the slot keeps going so that
            // every barrier below is still reached by all of its threads.
            if (!mbar_wait0(&bars[slot]) && t == 0) atomicExch(err, 1);
        } else {
            for (int j = t; j < N; j += T) buf[j] = make_double2(0.0, 0.0);
        }
        slot_sync<T>(slot);
    } else {
        const long col0 = (long)blockIdx.x * S;
        for (int idx = threadIdx.x; idx < S * N; idx += G::NT) {
            const int c = idx % S, j = idx / S;
            double2  *b2 = reinterpret_cast<double2 *>(smem + G::HDR + c * G::SLOT_BYTES);
            b2[j] = (col0 + c < nlines) ? in[ibase + col0 + c + (long)j * in_ld] : make_double2(0.0, 0.0);
        }
        __syncthreads();
    }

    // ---- pre-processing fused with the first radix-R pass (butterfly b = t)
    double2 v[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
        const int j = t + q * T;
        if (j == 0) {
            v[q] = make_double2(0.0, 0.0);
        } else {
            const double2 a = buf[j - 1], b = buf[M - j - 1];
            const double  s = __ldg(sn + j);
            v[q] = make_double2(fma(s, a.x + b.x, 0.5 * (a.x - b.x)), fma(s, a.y + b.y, 0.5 * (a.y - b.y)));
        }
    }
    slot_sync<T>(slot); // staging reads done before the buffer is overwritten
    dft_reg<R>(v);
#pragma unroll
    for (int q = 0; q < R; q++) buf[pad_idx(t * R + q)] = v[bitrev_c<R>(q)];
    slot_sync<T>(slot);

    constexpr int R2 = DstCfg<M>::R2, R3 = DstCfg<M>::R3, R4 = DstCfg<M>::R4;
    stockham_pass<M, T, R2, R>(buf, tw, t, slot);
    if constexpr (R3 > 1) stockham_pass<M, T, R3, R * R2>(buf, tw, t, slot);
    if constexpr (R4 > 1) stockham_pass<M, T, R4, R * R2 * R3>(buf, tw, t, slot);

    // ---- post-processing: thread t owns k in [t*K, t*K + K)
    constexpr int K = (M / 2) / T;
    double2 cs[K], ev[K];
    double2 run = make_double2(0.0, 0.0);
#pragma unroll
    for (int u = 0; u < K; u++) {
        const int k = t * K + u;
        const double2 yk = buf[pad_idx(k)];
        const double2 ym = buf[pad_idx(k == 0 ? 0 : M - k)];
        if (k == 0) {
            cs[u] = make_double2(0.5 * yk.x, 0.5 * yk.y);
            ev[u] = make_double2(0.0, 0.0);
        } else {
            cs[u] = make_double2(0.5 * (yk.x + ym.x), 0.5 * (yk.y + ym.y));
            ev[u] = make_double2(0.5 * (ym.y - yk.y), -0.5 * (ym.x - yk.x)); // (Y_{M-k}-Y_k)/(2i)
        }
        run = cadd(run, cs[u]);
        cs[u] = run; // local inclusive prefix
    }
    const double2 incl = slot_scan_inclusive<T>(run, t, slot, red);
    const double2 pre = csub(incl, run); // exclusive prefix of this thread
    const double  coef = sqrt(2.0 / M);
    slot_sync<T>(slot); // all reads of Y done
#pragma unroll
    for (int u = 0; u < K; u++) {
        const int k = t * K + u;
        const double2 odd = cadd(pre, cs[u]);
        buf[pad_idx(2 * k)] = cscale(odd, coef);                // S_{2k+1} -> index 2k
        if (k > 0) buf[pad_idx(2 * k - 1)] = cscale(ev[u], coef); // S_{2k}   -> index 2k-1
    }

    // ---- write back
    if constexpr (!OUT_STRIDED) {
        slot_sync<T>(slot);
        if (live) {
            double2 *dst = out + obase + line * out_ld;
#pragma unroll
            for (int u = 0; u < R; u++) {
                const int i = t + T * u;
                if (i < N) dst[i] = buf[pad_idx(i)];
            }
        }
    } else {
        __syncthreads();
        const long col0 = (long)blockIdx.x * S;
        for (int idx = threadIdx.x; idx < S * N; idx += G::NT) {
            const int c = idx % S, j = idx / S;
            const double2 *b2 = reinterpret_cast<const double2 *>(smem + G::HDR + c * G::SLOT_BYTES);
            if (col0 + c < nlines) out[obase + col0 + c + (long)j * out_ld] = b2[pad_idx(j)];
        }
    }
}

// ------------------------------- persistent warps, one line per TL lanes (rows) ------
// The same transform for contiguous rows, M = TL x R with TL = 8, 16 or 32 lanes per line
// (32/TL lines per warp) and R values per lane:
//   lane l of a line holds x_j and the mirror x_{M-j} for j = l + TL q (read from the line
//   buffer that the TMA filled), forms y_j in registers, runs an R-point DFT over q, twiddles by
//   W_M^{l k1} and exchanges through one padded transpose; TL-point DFTs over l then leave
//   Y_{k1 + R k2} for k1 = l + TL i in the lane.
//   Post-processing runs on blocks (lane l owns k in [KB l, KB l + KB), KB = M/(2 TL)), so the
//   prefix sum of the odd outputs is a sequential sum plus one scan over the line's lanes; the
//   outputs go back through the buffer so that the global stores are coalesced.
// Each warp owns two buffer sets and works through line groups w, w + W, ...: while it
// transforms one group, the TMA brings in the next.

// sin(pi m / 64), m = 0..32
__device__ __forceinline__ constexpr double sinpi64(int m) {
    constexpr double s[33] = {0.0,
                              0.049067674327418014255,
                              0.098017140329560601994,
                              0.14673047445536175166,
                              0.19509032201612826785,
                              0.24298017990326388995,
                              0.29028467725446236764,
                              0.33688985339222005069,
                              0.38268343236508977173,
                              0.42755509343028209432,
                              0.47139673682599764856,
                              0.51410274419322172659,
                              0.55557023301960222474,
                              0.59569930449243334347,
                              0.63439328416364549822,
                              0.67155895484701840063,
                              0.7071067811865475244,
                              0.74095112535495909118,
                              0.77301045336273696081,
                              0.80320753148064490981,
                              0.83146961230254523708,
                              0.8577286100002720699,
                              0.88192126434835502971,
                              0.90398929312344333159,
                              0.92387953251128675613,
                              0.94154406518302077841,
                              0.95694033573220886494,
                              0.9700312531945439926,
                              0.98078528040323044913,
                              0.98917650996478097345,
                              0.99518472667219688624,
                              0.99879545620517239271,
                              1.0};
    return s[m];
}
// sin and cos of pi m / 64 for m = 0..63
__device__ __forceinline__ constexpr double sin_m64(int m) { return m <= 32 ? sinpi64(m) : sinpi64(64 - m); }
__device__ __forceinline__ constexpr double cos_m64(int m) { return m <= 32 ? sinpi64(32 - m) : -sinpi64(m - 32); }

// Radix-2 decimation-in-time butterfly with twiddle w = exp(-2 pi i t / R), R <= 64 (angle
// pi m / 64, m = 128 t / R):  a <- a + w b,  b <- a - w b.  With a non-trivial twiddle the
// difference takes four fused multiply-adds and the sum is 2a minus it, six operations in all.
template <int R, int t> __device__ __forceinline__ void dit_bfly(double2 &a, double2 &b) {
    constexpr int m = t * (128 / R);
    const double2 x = a;
    if constexpr (t == 0) {
        a = cadd(x, b);
        b = csub(x, b);
    } else if constexpr (m == 32) { // w = -i, w b = (b.y, -b.x)
        a = make_double2(x.x + b.y, x.y - b.x);
        b = make_double2(x.x - b.y, x.y + b.x);
    } else {
        constexpr double c = cos_m64(m), sn = sin_m64(m); // w = c - i sn, w b = (c b.x + sn b.y, c b.y - sn b.x)
        const double2 d = make_double2(fma(-c, b.x, fma(-sn, b.y, x.x)), fma(-c, b.y, fma(sn, b.x, x.y)));
        a = make_double2(fma(2.0, x.x, -d.x), fma(2.0, x.y, -d.y));
        b = d;
    }
}
template <int R, int SPAN, int J> struct DitB {
    __device__ __forceinline__ static void run(double2 (&v)[R], int start) {
        if constexpr (J < SPAN) {
            dit_bfly<R, J * (R / (2 * SPAN))>(v[start + J], v[start + J + SPAN]);
            DitB<R, SPAN, J + 1>::run(v, start);
        }
    }
};
template <int R, int SPAN, int START> struct DitS {
    __device__ __forceinline__ static void run(double2 (&v)[R]) {
        if constexpr (START < R) {
            DitB<R, SPAN, 0>::run(v, START);
            DitS<R, SPAN, START + 2 * SPAN>::run(v);
        }
    }
};
template <int R, int SPAN> struct DitA {
    __device__ __forceinline__ static void run(double2 (&v)[R]) {
        if constexpr (SPAN < R) {
            DitS<R, SPAN, 0>::run(v);
            DitA<R, SPAN * 2>::run(v);
        }
    }
};
// forward R-point DFT in registers (R <= 64) of x held in bit-reversed order, v[bitrev(q)] = x_q;
// on return v[k] = X_k
template <int R> __device__ __forceinline__ void dft_dit(double2 (&v)[R]) { DitA<R, 1>::run(v); }

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int M> struct WCfg;
// TL lanes per line, R values per lane, WPC warps per CTA, NBUF line buffers per warp in the rows
// kernel (2: the next line loads while one is transformed; 1: more warps per SM instead), MINB
// CTAs per SM the register budget is sized for; CWPC warps per CTA and CNT tiles per warp in the
// columns kernel (CNT - 1 tiles load while one is transformed); RING: the rows use the CTA-ring
// kernel with RWPC warps per CTA
template <> struct WCfg<1024> { static constexpr int TL = 32, R = 32, WPC = 2, NBUF = 2, MINB = 3, CWPC = 2, CNT = 2, RWPC = 4, RING = 1; };
template <> struct WCfg<512>  { static constexpr int TL = 16, R = 32, WPC = 2, NBUF = 2, MINB = 3, CWPC = 2, CNT = 2, RWPC = 4, RING = 0; };
template <> struct WCfg<256>  { static constexpr int TL = 16, R = 16, WPC = 4, NBUF = 2, MINB = 3, CWPC = 4, CNT = 2, RWPC = 4, RING = 0; };
template <> struct WCfg<128>  { static constexpr int TL = 8,  R = 16, WPC = 4, NBUF = 2, MINB = 3, CWPC = 4, CNT = 2, RWPC = 4, RING = 0; };
template <> struct WCfg<64>   { static constexpr int TL = 8,  R = 8,  WPC = 4, NBUF = 2, MINB = 3, CWPC = 4, CNT = 2, RWPC = 4, RING = 0; };

template <int M> struct WGeom {
    static constexpr int TL = WCfg<M>::TL, R = WCfg<M>::R, WPC = WCfg<M>::WPC;
    static constexpr int LPW = 32 / TL, KB = M / (2 * TL);
    // one line's buffer: raw line, transpose [R][TL + 1], Y (k + k/KB), outputs ((2KB + 1) per 2KB)
    static constexpr int BUF = cmax(R * (TL + 1), cmax(M + M / KB, M + M / (2 * KB))) + 1;
    static constexpr int NBUF = WCfg<M>::NBUF;
    static constexpr int WARP_ELEMS = NBUF * LPW * BUF; // NBUF buffer sets per warp
    static constexpr int SMEM = 16 * WPC + 16 * WARP_ELEMS * WPC;
};

// Per-lane constants of the transform: sin, cos(pi l / M) and the twiddles W_M^{l a} (a < 8),
// W_M^{8 l b} (b < R/8).
template <int M> struct WConst {
    static constexpr int NB = WCfg<M>::R / 8 > 0 ? WCfg<M>::R / 8 : 1;
    double               sb, cb;
    double2              twa[8], twb[NB];
    __device__ __forceinline__ void load(int l, const double2 *__restrict__ tw, const double *__restrict__ sn) {
        sb = __ldg(sn + l);
        cb = __ldg(sn + M / 2 - l);
#pragma unroll
        for (int a = 0; a < 8; a++) twa[a] = __ldg(tw + ((l * a) & (M - 1)));
#pragma unroll
        for (int b = 0; b < NB; b++) twb[b] = __ldg(tw + ((8 * l * b) & (M - 1)));
    }
    // re-formed for every line: an empty asm hides them from loop-invariant hoisting, which would
    // otherwise pin every derived sine and twiddle in registers
    __device__ __forceinline__ void launder() {
        asm volatile("" : "+d"(sb), "+d"(cb));
#pragma unroll
        for (int a = 0; a < 8; a++) asm volatile("" : "+d"(twa[a].x), "+d"(twa[a].y));
#pragma unroll
        for (int b = 0; b < NB; b++) asm volatile("" : "+d"(twb[b].x), "+d"(twb[b].y));
    }
};

// inclusive scan over the TL lanes of a line: contiguous lanes (rows kernel) or lanes c + LPW l
// (columns kernel)
template <int TL, int LPW, bool INTER> __device__ __forceinline__ double2 line_scan(double2 x, int l) {
#pragma unroll
    for (int off = 1; off < TL; off <<= 1) {
        double ox, oy;
        if constexpr (INTER) {
            ox = __shfl_up_sync(0xffffffffu, x.x, off * LPW);
            oy = __shfl_up_sync(0xffffffffu, x.y, off * LPW);
        } else {
            ox = __shfl_up_sync(0xffffffffu, x.x, off, TL);
            oy = __shfl_up_sync(0xffffffffu, x.y, off, TL);
        }
        if (l >= off) { x.x += ox; x.y += oy; }
    }
    return x;
}

// The transform of one line by its TL lanes.  xload(j) returns x_j (1 <= j <= N) from wherever
// the line was staged; `buf` is the line's exchange area (BUF elements, may be that staging
// area: every x_j is read before the first write).  On return the outputs sit in buf at
// (2KB + 1)(p / 2KB) + p % 2KB for output offset p.
template <int M, bool INTER, typename XLoad>
__device__ __forceinline__ void w_transform(XLoad xload, double2 *buf, int l, bool live, WConst<M> &K) {
    using G = WGeom<M>;
    constexpr int TL = G::TL, R = G::R, LPW = G::LPW, KB = G::KB, K2 = 2 * KB;
    const double2 zero = make_double2(0.0, 0.0);
    K.launder();

    // ---- y_j = sin(pi j/M)(x_j + x_{M-j}) + (x_j - x_{M-j})/2 = (s + 1/2) x_j + (s - 1/2) x_{M-j},
    //      j = l + TL q, stored at v[bitrev(q)] for the decimation-in-time DFT
    double2 v[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
        const int j = l + TL * q;
        double2   a = zero, m = zero;
        if (live && (q > 0 || l > 0)) {
            a = xload(j);
            m = xload(M - j);
        }
        const double sp = fma(K.sb, cos_m64(q * (64 / R)), fma(K.cb, sin_m64(q * (64 / R)), 0.5)); // sin(pi j/M) + 1/2
        const double sm = sp - 1.0;
        v[bitrev_c<R>(q)] = make_double2(fma(sp, a.x, sm * m.x), fma(sp, a.y, sm * m.y));
    }
    __syncwarp(); // staged input consumed

    // ---- R-point DFTs over q, twiddle W_M^{l k1}, transpose [k1][l]
    dft_dit<R>(v);
#pragma unroll
    for (int k1 = 0; k1 < R; k1++)
        buf[k1 * (TL + 1) + l] = k1 ? cmul(v[k1], cmul(K.twa[k1 & 7], K.twb[k1 >> 3])) : v[0];
    __syncwarp();
    double2 w2[R / TL][TL]; // lane l takes k1 = l + TL i with all TL values of l', in bit-reversed order
#pragma unroll
    for (int i = 0; i < R / TL; i++)
#pragma unroll
        for (int lp = 0; lp < TL; lp++) w2[i][bitrev_c<TL>(lp)] = buf[(l + TL * i) * (TL + 1) + lp];
    __syncwarp();

    // ---- TL-point DFTs over l': Y_{k1 + R k2} = w2[i][k2]
#pragma unroll
    for (int i = 0; i < R / TL; i++) {
        dft_dit<TL>(w2[i]);
#pragma unroll
        for (int k2 = 0; k2 < TL; k2++) {
            const int k = l + TL * i + R * k2;
            buf[k + k / KB] = w2[i][k2];
        }
    }
    __syncwarp();

    // ---- post-processing on blocks k = KB l + u (the halves of (Y_k + Y_{M-k})/2 and
    //      (Y_{M-k} - Y_k)/(2i) are folded into the output scale)
    double2 cs[KB], ev[KB];
    double2 run = zero;
#pragma unroll
    for (int u = 0; u < KB; u++) {
        const int     k = KB * l + u;
        const double2 yk = buf[k + k / KB];
        if (k == 0) {
            cs[u] = yk;
            ev[u] = zero;
        } else {
            const int     km = M - k;
            const double2 ym = buf[km + km / KB];
            cs[u] = cadd(yk, ym);
            ev[u] = make_double2(ym.y - yk.y, yk.x - ym.x); // (Y_{M-k} - Y_k)/i
        }
        run = cadd(run, cs[u]);
        cs[u] = run;
    }
    const double2 pre = csub(line_scan<TL, LPW, INTER>(run, l), run);
    const double  coef = 0.5 * sqrt(2.0 / M);
    __syncwarp(); // every read of Y is done
#pragma unroll
    for (int u = 0; u < KB; u++) {
        const int k = KB * l + u, po = 2 * k, pe = 2 * k - 1;
        buf[(K2 + 1) * (po / K2) + po % K2] = cscale(cadd(pre, cs[u]), coef); // S_{2k+1} at 2k
        if (k > 0) buf[(K2 + 1) * (pe / K2) + pe % K2] = cscale(ev[u], coef); // S_{2k}   at 2k-1
    }
    __syncwarp();
}

// ---- single-precision arithmetic form of w_transform (the refined solve's correction
// transforms): the same algorithm and data movement, float arithmetic, FP64 in and out.  The
// staged line and the results stay double2 in shared memory; the exchanges in between are
// float2 in the same buffer.
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
template <int R, int t> __device__ __forceinline__ void dit_bfly_f(float2 &a, float2 &b) {
    constexpr int m = t * (128 / R);
    const float2  x = a;
    if constexpr (t == 0) {
        a = fadd2(x, b);
        b = fsub2(x, b);
    } else if constexpr (m == 32) {
        a = make_float2(x.x + b.y, x.y - b.x);
        b = make_float2(x.x - b.y, x.y + b.x);
    } else {
        constexpr float c = (float)cos_m64(m), sn = (float)sin_m64(m);
        const float2    d = make_float2(fmaf(-c, b.x, fmaf(-sn, b.y, x.x)), fmaf(-c, b.y, fmaf(sn, b.x, x.y)));
        a = make_float2(fmaf(2.0f, x.x, -d.x), fmaf(2.0f, x.y, -d.y));
        b = d;
    }
}
template <int R, int SPAN, int J> struct DitBF {
    __device__ __forceinline__ static void run(float2 (&v)[R], int start) {
        if constexpr (J < SPAN) {
            dit_bfly_f<R, J * (R / (2 * SPAN))>(v[start + J], v[start + J + SPAN]);
            DitBF<R, SPAN, J + 1>::run(v, start);
        }
    }
};
template <int R, int SPAN, int START> struct DitSF {
    __device__ __forceinline__ static void run(float2 (&v)[R]) {
        if constexpr (START < R) {
            DitBF<R, SPAN, 0>::run(v, START);
            DitSF<R, SPAN, START + 2 * SPAN>::run(v);
        }
    }
};
template <int R, int SPAN> struct DitAF {
    __device__ __forceinline__ static void run(float2 (&v)[R]) {
        if constexpr (SPAN < R) {
            DitSF<R, SPAN, 0>::run(v);
            DitAF<R, SPAN * 2>::run(v);
        }
    }
};
template <int R> __device__ __forceinline__ void dft_dit_f(float2 (&v)[R]) { DitAF<R, 1>::run(v); }

template <int TL, int LPW, bool INTER> __device__ __forceinline__ float2 line_scan_f(float2 x, int l) {
#pragma unroll
    for (int off = 1; off < TL; off <<= 1) {
        float ox, oy;
        if constexpr (INTER) {
            ox = __shfl_up_sync(0xffffffffu, x.x, off * LPW);
            oy = __shfl_up_sync(0xffffffffu, x.y, off * LPW);
        } else {
            ox = __shfl_up_sync(0xffffffffu, x.x, off, TL);
            oy = __shfl_up_sync(0xffffffffu, x.y, off, TL);
        }
        if (l >= off) { x.x += ox; x.y += oy; }
    }
    return x;
}

template <int M, bool INTER, typename XLoad>
__device__ __forceinline__ void w_transform_lp(XLoad xload, double2 *buf, int l, bool live, WConst<M> &K) {
    using G = WGeom<M>;
    constexpr int TL = G::TL, R = G::R, LPW = G::LPW, KB = G::KB, K2 = 2 * KB;
    constexpr int NB = WConst<M>::NB;
    const float2  zero = make_float2(0.f, 0.f);
    float2       *fb = reinterpret_cast<float2 *>(buf);
    K.launder();
    const float sb = (float)K.sb, cb = (float)K.cb;
    float2      twa[8], twb[NB];
#pragma unroll
    for (int a = 0; a < 8; a++) twa[a] = make_float2((float)K.twa[a].x, (float)K.twa[a].y);
#pragma unroll
    for (int b = 0; b < NB; b++) twb[b] = make_float2((float)K.twb[b].x, (float)K.twb[b].y);

    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
        const int j = l + TL * q;
        double2   a = make_double2(0.0, 0.0), m = a;
        if (live && (q > 0 || l > 0)) {
            a = xload(j);
            m = xload(M - j);
        }
        const float sp = fmaf(sb, (float)cos_m64(q * (64 / R)), fmaf(cb, (float)sin_m64(q * (64 / R)), 0.5f));
        const float sm = sp - 1.0f;
        v[bitrev_c<R>(q)] = make_float2(fmaf(sp, (float)a.x, sm * (float)m.x), fmaf(sp, (float)a.y, sm * (float)m.y));
    }
    __syncwarp();

    dft_dit_f<R>(v);
#pragma unroll
    for (int k1 = 0; k1 < R; k1++)
        fb[k1 * (TL + 1) + l] = k1 ? fmul2(v[k1], fmul2(twa[k1 & 7], twb[k1 >> 3])) : v[0];
    __syncwarp();
    float2 w2[R / TL][TL];
#pragma unroll
    for (int i = 0; i < R / TL; i++)
#pragma unroll
        for (int lp = 0; lp < TL; lp++) w2[i][bitrev_c<TL>(lp)] = fb[(l + TL * i) * (TL + 1) + lp];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < R / TL; i++) {
        dft_dit_f<TL>(w2[i]);
#pragma unroll
        for (int k2 = 0; k2 < TL; k2++) {
            const int k = l + TL * i + R * k2;
            fb[k + k / KB] = w2[i][k2];
        }
    }
    __syncwarp();

    float2 cs[KB], ev[KB];
    float2 run = zero;
#pragma unroll
    for (int u = 0; u < KB; u++) {
        const int    k = KB * l + u;
        const float2 yk = fb[k + k / KB];
        if (k == 0) {
            cs[u] = yk;
            ev[u] = zero;
        } else {
            const int    km = M - k;
            const float2 ym = fb[km + km / KB];
            cs[u] = fadd2(yk, ym);
            ev[u] = make_float2(ym.y - yk.y, yk.x - ym.x);
        }
        run = fadd2(run, cs[u]);
        cs[u] = run;
    }
    const float2 pre = fsub2(line_scan_f<TL, LPW, INTER>(run, l), run);
    const float  coef = (float)(0.5 * sqrt(2.0 / M));
    __syncwarp();
#pragma unroll
    for (int u = 0; u < KB; u++) {
        const int    k = KB * l + u, po = 2 * k, pe = 2 * k - 1;
        const float2 o = fadd2(pre, cs[u]);
        buf[(K2 + 1) * (po / K2) + po % K2] = make_double2((double)(o.x * coef), (double)(o.y * coef));
        if (k > 0) buf[(K2 + 1) * (pe / K2) + pe % K2] = make_double2((double)(ev[u].x * coef), (double)(ev[u].y * coef));
    }
    __syncwarp();
}

// ---- rows: lines g = 0 .. nlines*nplanes-1 at in + (g / nlines) in_plane + (g % nlines) in_ld
// with x_1..x_N at offsets 0..N-1, likewise for the output; in and out may be the same buffer.
// Failure injection (hh_ctx_inject_wait_expiry): when *inj is set, warp 0 of CTA 0 takes it
// (one launch only) and its first line group's barrier expects kInjectBytes more than the copies
// bring, so that wait cannot complete and runs out of a short poll budget (kInjectPolls); the
// kernel then reports through `err` exactly as for a copy that never lands.  The drain counts
// the added bytes as arrived itself and waits, with the full budget, for the real copies.
constexpr uint32_t kInjectBytes = 16;
constexpr long     kInjectPolls = 1L << 12;

// UPD (the refined solve's correction, single-precision transforms): out <- out - result
template <int M, bool LP = false, bool UPD = false>
__global__ void __launch_bounds__(32 * WCfg<M>::WPC, WCfg<M>::MINB)
    k_dst1_w(const double2 *in, double2 *out, long nlines, long nplanes, long in_ld, long out_ld, long in_plane,
             long out_plane, const double2 *__restrict__ tw, const double *__restrict__ sn, int *err, int *inj) {
    using G = WGeom<M>;
    constexpr int      TL = G::TL, LPW = G::LPW, KB = G::KB, BUF = G::BUF, N = M - 1, K2 = 2 * KB;
    constexpr uint32_t kLineBytes = N * 16;
    extern __shared__ __align__(128) unsigned char dsm[];
    const int  lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int  c = lane / TL, l = lane % TL; // line of the warp's group, lane within the line
    uint64_t  *bar = reinterpret_cast<uint64_t *>(dsm) + 2 * wq;
    double2   *sets = reinterpret_cast<double2 *>(dsm + 16 * G::WPC) + wq * G::WARP_ELEMS;
    const long total = nlines * nplanes;
    const long groups = (total + LPW - 1) / LPW;
    const long stride = (long)gridDim.x * G::WPC;
    const long g0 = (long)blockIdx.x * G::WPC + wq;
    if (g0 >= groups) return; // whole warp

    // one plane (all 2D calls): no 64-bit division per line
    auto src_of = [&](long g) {
        return nplanes == 1 ? in + g * in_ld : in + (g / nlines) * in_plane + (g % nlines) * in_ld;
    };
    auto dst_of = [&](long g) {
        return nplanes == 1 ? out + g * out_ld : out + (g / nlines) * out_plane + (g % nlines) * out_ld;
    };
    int injected = 0;
    if (lane == 0 && inj && blockIdx.x == 0 && wq == 0) injected = atomicExch(inj, 0);
    injected = __shfl_sync(0xffffffffu, injected, 0);
    // lane 0: bring in line group `grp` to buffer set `s` (`extra`: injected bytes that never come)
    auto fetch = [&](long grp, int s, uint32_t extra) {
        const long first = grp * LPW;
        const int  nl = (int)((total - first) < LPW ? (total - first) : LPW);
        mbar_expect_tx(&bar[s], (uint32_t)nl * kLineBytes + extra);
        for (int x = 0; x < nl; x++) tma_bulk_load(sets + (s * LPW + x) * BUF, src_of(first + x), kLineBytes, &bar[s]);
    };
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    constexpr int NBUF = G::NBUF;
    if (lane == 0) {
        fetch(g0, 0, injected ? kInjectBytes : 0u);
        if (NBUF == 2 && g0 + stride < groups) fetch(g0 + stride, 1, 0u);
    }
    WConst<M> K;
    K.load(l, tw, sn);

    int  it = 0;
    long failed = -1;
    for (long grp = g0; grp < groups; grp += stride, it++) {
        const int s = NBUF == 2 ? (it & 1) : 0;
        double2  *buf = sets + (s * LPW + c) * BUF;
        const long line = grp * LPW + c;
        const bool live = line < total;
        const uint32_t par = NBUF == 2 ? (it >> 1) & 1 : it & 1;
        if (!(it == 0 && injected ? mbar_wait_parity_n(&bar[s], par, kInjectPolls) : mbar_wait_parity(&bar[s], par))) {
            if (lane == 0) atomicExch(err, 1);
            failed = grp;
            break;
        }
        if constexpr (LP) w_transform_lp<M, false>([&](int j) { return buf[j - 1]; }, buf, l, live, K);
        else w_transform<M, false>([&](int j) { return buf[j - 1]; }, buf, l, live, K);
        if (live) {
            double2 *dst = dst_of(line);
#pragma unroll
            for (int q = 0; q < M / TL; q++) {
                const int p = l + TL * q;
                if (p < N) {
                    const double2 o = buf[(K2 + 1) * (p / K2) + p % K2];
                    dst[p] = UPD ? csub(dst[p], o) : o;
                }
            }
        }
        // the buffer set is free again: bring in the group after next (every lane orders its
        // generic-proxy accesses before the asynchronous copy that overwrites them)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0 && grp + NBUF * stride < groups) fetch(grp + NBUF * stride, s, 0u);
    }
    // after an expired wait, give the copies still in flight a bounded chance to land before the
    // CTA's shared memory is released
    if (failed >= 0 && lane == 0 && injected && it == 0) mbar_complete_tx(&bar[0], kInjectBytes);
    if (failed >= 0 && lane == 0) {
        if (NBUF == 1) {
            mbar_wait_parity(&bar[0], it & 1);
        } else {
            mbar_wait_parity(&bar[it & 1], (it >> 1) & 1);
            if (failed + stride < groups) mbar_wait_parity(&bar[(it + 1) & 1], ((it + 1) >> 1) & 1);
        }
    }
}

// ---- rows, CTA ring: the same transform with the line buffers pooled per CTA.  RWPC warps share
// RNS = RWPC + 2 buffers: ticket t of the CTA (group blockIdx.x + t gridDim.x) lives in buffer
// t % RNS; warp w takes tickets w, w + RWPC, ...; the warp that finishes ticket t brings in
// ticket t + RNS to the buffer it frees.  With fewer buffers per warp than the per-warp double
// buffer (1.5 against 2), more warps fit per SM.  gen[b] counts the copies issued to buffer b, so
// a warp waits on a buffer's mbarrier only once the copy of its ticket has been issued (at most
// one phase ahead of the barrier).
template <int M> struct WRing {
    using G = WGeom<M>;
    static constexpr int WPC = WCfg<M>::RWPC, NS = WPC + 2;
    static constexpr int SLOT = G::LPW * G::BUF;        // elements of one buffer (one line group)
    static constexpr int SMEM = 128 + 16 * NS * SLOT;   // barriers and counters, then the buffers
    static_assert(NS * 8 + NS * 4 <= 128, "barriers and counters fit in front of the buffers");
};

template <int M, bool LP = false, bool UPD = false>
__global__ void __launch_bounds__(32 * WCfg<M>::RWPC, 2)
    k_dst1_wr(const double2 *in, double2 *out, long nlines, long nplanes, long in_ld, long out_ld, long in_plane,
              long out_plane, const double2 *__restrict__ tw, const double *__restrict__ sn, int *err) {
    using G = WGeom<M>;
    using RG = WRing<M>;
    constexpr int      TL = G::TL, LPW = G::LPW, KB = G::KB, BUF = G::BUF, N = M - 1, K2 = 2 * KB;
    constexpr int      NS = RG::NS, WPC = RG::WPC;
    constexpr uint32_t kLineBytes = N * 16;
    extern __shared__ __align__(128) unsigned char dsm[];
    const int          lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int          c = lane / TL, l = lane % TL;
    uint64_t          *bar = reinterpret_cast<uint64_t *>(dsm);
    volatile int      *gen = reinterpret_cast<volatile int *>(dsm + 8 * NS);
    double2           *slots = reinterpret_cast<double2 *>(dsm + 128);
    const long         total = nlines * nplanes;
    const long         groups = (total + LPW - 1) / LPW;
    if ((long)blockIdx.x >= groups) return; // whole CTA
    const int  tickets = (int)((groups - blockIdx.x + gridDim.x - 1) / gridDim.x);
    auto       grp_of = [&](int t) { return (long)blockIdx.x + (long)t * gridDim.x; };
    auto       src_of = [&](long g) { // one plane (all 2D calls): no 64-bit division per line
        return nplanes == 1 ? in + g * in_ld : in + (g / nlines) * in_plane + (g % nlines) * in_ld;
    };
    auto dst_of = [&](long g) {
        return nplanes == 1 ? out + g * out_ld : out + (g / nlines) * out_plane + (g % nlines) * out_ld;
    };
    auto       fetch = [&](int t) { // lane 0: ticket t into buffer t % NS
        const int  b = (int)(t % NS);
        const long first = grp_of(t) * LPW;
        const int  nl = (int)((total - first) < LPW ? (total - first) : LPW);
        mbar_expect_tx(&bar[b], (uint32_t)nl * kLineBytes);
        for (int x = 0; x < nl; x++)
            tma_bulk_load(slots + (long)b * RG::SLOT + x * BUF, src_of(first + x), kLineBytes, &bar[b]);
    };
    if (threadIdx.x == 0) {
        for (int b = 0; b < NS; b++) {
            mbar_init(&bar[b], 1);
            gen[b] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int b = 0; b < NS && b < tickets; b++) {
            fetch(b);
            gen[b] = 1;
        }
    }
    __syncthreads();
    WConst<M> K;
    K.load(l, tw, sn);

    int failed = -1;
    for (int t = wq; t < tickets; t += WPC) {
        const int b = t % NS;
        const int want = t / NS + 1; // the copy of this ticket is buffer b's want-th
        bool      ok = true;
        if (lane == 0) {
            long spin = 0;
            while (gen[b] < want && ++spin < (1L << 26)) {
            }
            ok = gen[b] >= want;
        }
        ok = __shfl_sync(0xffffffffu, ok, 0) && mbar_wait_parity(&bar[b], (uint32_t)((t / NS) & 1));
        if (!ok) {
            if (lane == 0) atomicExch(err, 1);
            failed = t;
            break;
        }
        double2   *buf = slots + (long)b * RG::SLOT + c * BUF;
        const long line = grp_of(t) * LPW + c;
        const bool live = line < total;
        if constexpr (LP) w_transform_lp<M, false>([&](int j) { return buf[j - 1]; }, buf, l, live, K);
        else w_transform<M, false>([&](int j) { return buf[j - 1]; }, buf, l, live, K);
        if (live) {
            double2 *dst = dst_of(line);
#pragma unroll
            for (int q = 0; q < M / TL; q++) {
                const int p = l + TL * q;
                if (p < N) {
                    const double2 o = buf[(K2 + 1) * (p / K2) + p % K2];
                    dst[p] = UPD ? csub(dst[p], o) : o;
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // reads before the refill
        __syncwarp();
        if (lane == 0 && t + NS < tickets) {
            fetch(t + NS);
            __threadfence_block(); // the copy's arrival is registered before its ticket is announced
            gen[b] = want + 1;
        }
    }
    // after an expired wait, copies this warp issued get a bounded chance to land before the
    // CTA's shared memory is released
    if (failed >= 0 && lane == 0)
        for (int t = failed; t < tickets && t < failed + NS; t++) {
            const int b = t % NS;
            if (gen[b] >= t / NS + 1) mbar_wait_parity(&bar[b], (uint32_t)((t / NS) & 1));
        }
}

// ---- rows, M = 2048: two warps per line (a "team" of TL = 64 lanes, R = 32 values per lane; one
// warp would need 64 values per lane).  With j = l + 64 q and k = k1 + 32 k2:
//   Y_k = sum_l W_64^{l k2} [ W_M^{l k1} sum_q y_{l+64q} W_32^{q k1} ]
// Lane l forms y_j (q < 32), runs the 32-point DFT over q and twiddles by W_M^{l k1}; a transpose
// through the line's buffer gives each k1 (< 32) its 64 values over l.  That 64-point DFT is split
// 64 = 2 x 32 over a lane pair of one warp (lanes w and w ^ 16 take the even and the odd l): each
// runs a 32-point DFT and the pair finishes with one radix-2 step, exchanging half of its values
// by shuffles.  Post-processing and the outputs are those of w_transform (KB = 16 per lane), the
// prefix sum carried from the first warp of the team to the second through shared memory.  The
// team synchronises on its own named barrier (64 threads).  A CTA of TPC teams shares a ring of
// NS = TPC + 2 line buffers with the protocol of k_dst1_wr (gen[] counts the copies issued to a
// buffer; the team that frees a buffer loads the CTA's line NS tickets ahead into it).
template <int M> struct W2Geom;
template <> struct W2Geom<2048> {
    static constexpr int TL = 64, R = 32, KB = 16, TPC = 4, NS = 6;
    static constexpr int TP = TL + 1; // transpose pitch: the 8 lanes of a phase read 8 distinct bank groups
    // max(staged line N, transpose R * TP, Y at k + k / KB, outputs at (2KB + 1)(p / 2KB) + p % 2KB),
    // rounded to 8 elements
    static constexpr int BUF = (cmax(cmax(2047, R * TP), cmax(2048 + 2048 / KB, (2 * KB + 1) * (2048 / (2 * KB)))) + 7) / 8 * 8;
    static constexpr int SMEM = 256 + 16 * NS * BUF; // barriers, counters and carries, then the buffers
    static_assert(NS * 8 + NS * 4 <= 128 && TPC * 16 <= 128, "the header fits in 256 bytes");
};

__device__ __forceinline__ void team_sync(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }
// true on every thread of the team if p holds on any of them (a barrier of the team)
__device__ __forceinline__ bool team_any(int id, bool p) {
    int r;
    asm volatile("{\n .reg .pred q, o;\n setp.ne.s32 q, %1, 0;\n bar.red.or.pred o, %2, 64, q;\n selp.s32 %0, 1, 0, o;\n}\n"
                 : "=r"(r)
                 : "r"((int)p), "r"(id)
                 : "memory");
    return r != 0;
}

// One line of the two-warp transform in single-precision arithmetic (the refined solve's correction
// transforms): the staged line x_1..x_N at buf[0..N-1] in, the outputs at
// buf[(2KB + 1)(p / 2KB) + p % 2KB] out, FP64 in and out with float exchanges in the same buffer
// (as w_transform_lp does for one warp per line).  l: lane of the line; h, w: warp of the team and
// lane of the warp; (k1, e): the lane's second-stage DFT and half; tq, bid: the team and its named
// barrier; carry: the team's slot for the prefix sum.  The FP64 form is written out in k_dst1_w2.
template <int M>
__device__ __forceinline__ void w2_transform_lp(double2 *buf, int l, int h, int w, int k1, int e, int tq, int bid,
                                                double sbd, double cbd, const double2 (&twad)[8],
                                                const double2 (&twbd)[W2Geom<M>::R / 8], double2 *carry) {
    using G = W2Geom<M>;
    constexpr int TL = G::TL, R = G::R, KB = G::KB, K2 = 2 * KB, TP = G::TP;
    const float2  zero = make_float2(0.f, 0.f);
    float2       *fb = reinterpret_cast<float2 *>(buf);
    float2       *fcarry = reinterpret_cast<float2 *>(carry);
    const float   sb = (float)sbd, cb = (float)cbd;
    float2        twa[8], twb[R / 8];
#pragma unroll
    for (int a = 0; a < 8; a++) twa[a] = make_float2((float)twad[a].x, (float)twad[a].y);
#pragma unroll
    for (int a = 0; a < R / 8; a++) twb[a] = make_float2((float)twbd[a].x, (float)twbd[a].y);

    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
        const int j = l + TL * q;
        double2   a = make_double2(0.0, 0.0), m = a;
        if (q > 0 || l > 0) {
            a = buf[j - 1];
            m = buf[M - j - 1];
        }
        const float sp = fmaf(sb, (float)cos_m64(q * (64 / R)), fmaf(cb, (float)sin_m64(q * (64 / R)), 0.5f));
        const float sm = sp - 1.0f;
        v[bitrev_c<R>(q)] = make_float2(fmaf(sp, (float)a.x, sm * (float)m.x), fmaf(sp, (float)a.y, sm * (float)m.y));
    }
    team_sync(bid); // the staged line is consumed
    dft_dit_f<R>(v);
#pragma unroll
    for (int k = 0; k < R; k++) fb[k * TP + l] = k ? fmul2(v[k], fmul2(twa[k & 7], twb[k >> 3])) : v[0];
    team_sync(bid);

    float2 u[R];
#pragma unroll
    for (int m = 0; m < R; m++) u[bitrev_c<R>(m)] = fb[k1 * TP + e + 2 * m];
    team_sync(bid);
    dft_dit_f<R>(u);
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const float2 own = e ? u[16 + i] : u[i];
        const float2 snd = e ? u[i] : u[16 + i];
        const float2 rcv = make_float2(__shfl_xor_sync(0xffffffffu, snd.x, 16), __shfl_xor_sync(0xffffffffu, snd.y, 16));
        const float2 a0 = e ? rcv : own, a1 = e ? own : rcv;
        float2       tt = fmul2(a1, make_float2((float)cos_m64(2 * i), -(float)sin_m64(2 * i)));
        if (e) tt = make_float2(tt.y, -tt.x);
        const int klo = k1 + 32 * (16 * e + i), khi = klo + 1024;
        fb[klo + klo / KB] = fadd2(a0, tt);
        fb[khi + khi / KB] = fsub2(a0, tt);
    }
    team_sync(bid);

    float2 cs[KB], ev[KB];
    float2 run = zero;
#pragma unroll
    for (int uu = 0; uu < KB; uu++) {
        const int    k = KB * l + uu;
        const float2 yk = fb[k + k / KB];
        if (k == 0) {
            cs[uu] = yk;
            ev[uu] = zero;
        } else {
            const int    km = M - k;
            const float2 ym = fb[km + km / KB];
            cs[uu] = fadd2(yk, ym);
            ev[uu] = make_float2(ym.y - yk.y, yk.x - ym.x);
        }
        run = fadd2(run, cs[uu]);
        cs[uu] = run;
    }
    const float2 incl = line_scan_f<32, 1, false>(run, w);
    if (h == 0 && w == 31) fcarry[2 * tq] = incl;
    team_sync(bid);
    float2 pre = fsub2(incl, run);
    if (h) pre = fadd2(pre, fcarry[2 * tq]);
    const float coef = (float)(0.5 * sqrt(2.0 / M));
#pragma unroll
    for (int uu = 0; uu < KB; uu++) {
        const int    k = KB * l + uu, po = 2 * k, pe = 2 * k - 1;
        const float2 o = fadd2(pre, cs[uu]);
        buf[(K2 + 1) * (po / K2) + po % K2] = make_double2((double)(o.x * coef), (double)(o.y * coef));
        if (k > 0) buf[(K2 + 1) * (pe / K2) + pe % K2] = make_double2((double)(ev[uu].x * coef), (double)(ev[uu].y * coef));
    }
    team_sync(bid); // outputs complete
}

template <int M, bool LP = false, bool UPD = false>
__global__ void __launch_bounds__(64 * W2Geom<M>::TPC, 1)
    k_dst1_w2(const double2 *in, double2 *out, long nlines, long nplanes, long in_ld, long out_ld, long in_plane,
              long out_plane, const double2 *__restrict__ tw, const double *__restrict__ sn, int *err) {
    using G = W2Geom<M>;
    constexpr int      TL = G::TL, R = G::R, KB = G::KB, K2 = 2 * KB, NS = G::NS, TPC = G::TPC, TP = G::TP;
    constexpr int      N = M - 1, BUF = G::BUF;
    constexpr uint32_t kLineBytes = N * 16;
    extern __shared__ __align__(128) unsigned char dsm[];
    uint64_t          *bar = reinterpret_cast<uint64_t *>(dsm);
    volatile int      *gen = reinterpret_cast<volatile int *>(dsm + 8 * NS);
    double2           *carry = reinterpret_cast<double2 *>(dsm + 128);
    double2           *slots = reinterpret_cast<double2 *>(dsm + 256);
    const int          tq = threadIdx.x >> 6, l = threadIdx.x & 63; // team, lane of the line
    const int          h = l >> 5, w = l & 31;                       // warp of the team, lane of the warp
    const int          k1 = 16 * h + (w & 15), e = w >> 4;           // second stage: DFT k1, even/odd l
    const int          bid = 1 + tq;                                 // the team's named barrier
    const long         total = nlines * nplanes;
    if ((long)blockIdx.x >= total) return; // whole CTA
    const int tickets = (int)((total - blockIdx.x + gridDim.x - 1) / gridDim.x);
    auto      line_of = [&](int t) { return (long)blockIdx.x + (long)t * gridDim.x; };
    auto      src_of = [&](long g) {
        return nplanes == 1 ? in + g * in_ld : in + (g / nlines) * in_plane + (g % nlines) * in_ld;
    };
    auto dst_of = [&](long g) {
        return nplanes == 1 ? out + g * out_ld : out + (g / nlines) * out_plane + (g % nlines) * out_ld;
    };
    auto fetch = [&](int t) { // one thread: ticket t into buffer t % NS
        const int b = t % NS;
        mbar_expect_tx(&bar[b], kLineBytes);
        tma_bulk_load(slots + (long)b * BUF, src_of(line_of(t)), kLineBytes, &bar[b]);
    };
    if (threadIdx.x == 0) {
        for (int b = 0; b < NS; b++) {
            mbar_init(&bar[b], 1);
            gen[b] = 0;
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int b = 0; b < NS && b < tickets; b++) {
            fetch(b);
            gen[b] = 1;
        }
    }
    __syncthreads();
    // per-lane constants: sin, cos(pi l / M); W_M^{l a} (a < 8), W_M^{8 l b} (b < R / 8)
    double  sb = __ldg(sn + l), cb = __ldg(sn + M / 2 - l);
    double2 twa[8], twb[R / 8];
#pragma unroll
    for (int a = 0; a < 8; a++) twa[a] = __ldg(tw + ((l * a) & (M - 1)));
#pragma unroll
    for (int b = 0; b < R / 8; b++) twb[b] = __ldg(tw + ((8 * l * b) & (M - 1)));
    const double2 zero = make_double2(0.0, 0.0);
    const double  coef = 0.5 * sqrt(2.0 / M);

    int failed = -1;
    for (int t = tq; t < tickets; t += TPC) {
        const int b = t % NS;
        const int want = t / NS + 1; // the copy of this ticket is buffer b's want-th
        long      spin = 0;
        while (gen[b] < want && ++spin < (1L << 26)) {
        }
        const bool ok = gen[b] >= want && mbar_wait_parity(&bar[b], (uint32_t)((t / NS) & 1));
        if (team_any(bid, !ok)) {
            if (l == 0) atomicExch(err, 1);
            failed = t;
            break;
        }
        double2 *buf = slots + (long)b * BUF;
        // re-formed for every line (see WConst::launder): hoisted products would pin registers
        asm volatile("" : "+d"(sb), "+d"(cb));
#pragma unroll
        for (int a = 0; a < 8; a++) asm volatile("" : "+d"(twa[a].x), "+d"(twa[a].y));
#pragma unroll
        for (int a = 0; a < R / 8; a++) asm volatile("" : "+d"(twb[a].x), "+d"(twb[a].y));

        if constexpr (LP) {
            w2_transform_lp<M>(buf, l, h, w, k1, e, tq, bid, sb, cb, twa, twb, carry);
        } else {
            // ---- y_j = (s + 1/2) x_j + (s - 1/2) x_{M-j}, s = sin(pi j / M), j = l + TL q, at v[bitrev(q)]
            double2 v[R];
    #pragma unroll
            for (int q = 0; q < R; q++) {
                const int j = l + TL * q;
                double2   a = zero, m = zero;
                if (q > 0 || l > 0) {
                    a = buf[j - 1];
                    m = buf[M - j - 1];
                }
                const double sp = fma(sb, cos_m64(q * (64 / R)), fma(cb, sin_m64(q * (64 / R)), 0.5));
                const double sm = sp - 1.0;
                v[bitrev_c<R>(q)] = make_double2(fma(sp, a.x, sm * m.x), fma(sp, a.y, sm * m.y));
            }
            team_sync(bid); // the staged line is consumed
            dft_dit<R>(v);
    #pragma unroll
            for (int k = 0; k < R; k++) buf[k * TP + l] = k ? cmul(v[k], cmul(twa[k & 7], twb[k >> 3])) : v[0];
            team_sync(bid);

            // ---- k1's 64-point DFT over l: this lane takes l = e + 2 m (m < 32)
            double2 u[R];
    #pragma unroll
            for (int m = 0; m < R; m++) u[bitrev_c<R>(m)] = buf[k1 * TP + e + 2 * m];
            team_sync(bid); // the transposed values are consumed
            dft_dit<R>(u);  // u[k] = A_e[k]
    #pragma unroll
            for (int i = 0; i < 16; i++) {
                // the pair's radix-2 step: Z[k'] = A_0[k'] + W_64^{k'} A_1[k'], Z[k' + 32] = A_0[k'] - W_64^{k'} A_1[k'],
                // this lane at k' = 16 e + i (W_64^{16 + i} = -i W_64^i)
                const double2 own = e ? u[16 + i] : u[i];
                const double2 snd = e ? u[i] : u[16 + i];
                const double2 rcv = make_double2(__shfl_xor_sync(0xffffffffu, snd.x, 16), __shfl_xor_sync(0xffffffffu, snd.y, 16));
                const double2 a0 = e ? rcv : own, a1 = e ? own : rcv;
                double2       tt = cmul(a1, make_double2(cos_m64(2 * i), -sin_m64(2 * i)));
                if (e) tt = make_double2(tt.y, -tt.x);
                const int klo = k1 + 32 * (16 * e + i), khi = klo + 1024;
                buf[klo + klo / KB] = cadd(a0, tt);
                buf[khi + khi / KB] = csub(a0, tt);
            }
            team_sync(bid); // Y complete

            // ---- post-processing on blocks k = KB l + u (as in w_transform)
            double2 cs[KB], ev[KB];
            double2 run = zero;
    #pragma unroll
            for (int uu = 0; uu < KB; uu++) {
                const int     k = KB * l + uu;
                const double2 yk = buf[k + k / KB];
                if (k == 0) {
                    cs[uu] = yk;
                    ev[uu] = zero;
                } else {
                    const int     km = M - k;
                    const double2 ym = buf[km + km / KB];
                    cs[uu] = cadd(yk, ym);
                    ev[uu] = make_double2(ym.y - yk.y, yk.x - ym.x);
                }
                run = cadd(run, cs[uu]);
                cs[uu] = run;
            }
            const double2 incl = line_scan<32, 1, false>(run, w);
            if (h == 0 && w == 31) carry[tq] = incl;
            team_sync(bid); // every read of Y is done; the first warp's total is visible
            double2 pre = csub(incl, run);
            if (h) pre = cadd(pre, carry[tq]);
    #pragma unroll
            for (int uu = 0; uu < KB; uu++) {
                const int k = KB * l + uu, po = 2 * k, pe = 2 * k - 1;
                buf[(K2 + 1) * (po / K2) + po % K2] = cscale(cadd(pre, cs[uu]), coef);
                if (k > 0) buf[(K2 + 1) * (pe / K2) + pe % K2] = cscale(ev[uu], coef);
            }
            team_sync(bid); // outputs complete
        }
        double2 *dst = dst_of(line_of(t));
#pragma unroll
        for (int q = 0; q < M / TL; q++) {
            const int p = l + TL * q;
            if (p < N) {
                const double2 o = buf[(K2 + 1) * (p / K2) + p % K2];
                dst[p] = UPD ? csub(dst[p], o) : o;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // reads before the refill
        team_sync(bid);
        if (l == 0 && t + NS < tickets) {
            fetch(t + NS);
            __threadfence_block(); // the copy's arrival is registered before its ticket is announced
            gen[b] = want + 1;
        }
    }
    // after an expired wait, copies issued to the ring get a bounded chance to land before the
    // CTA's shared memory is released
    if (failed >= 0 && l == 0)
        for (int t = failed; t < tickets && t < failed + NS; t++) {
            const int b = t % NS;
            if (gen[b] >= t / NS + 1) mbar_wait_parity(&bar[b], (uint32_t)((t / NS) & 1));
        }
}

// ---- columns: line x of plane p is element j at base + p plane + x + (j - 1) ld.  A 4-D tensor
// map (re/im, x, j, plane) brings C = LPW neighbouring columns, all rows, into a [j][c] tile; the
// warp's lanes interleave over the C lines (lane = c + LPW l) so that reading the tile is free of
// bank conflicts, and the outputs go back through the same tile with a tensor store.
template <int M> struct WColGeom {
    using G = WGeom<M>;
    static constexpr int LPW = G::LPW, N = M - 1;
    static constexpr int BR = N < 256 ? N : 256;              // rows per TMA box
    static constexpr int NBOX = (N + BR - 1) / BR;
    // tensor copies need 128-byte aligned shared-memory addresses: tiles and warp areas are
    // whole multiples of 8 elements (boxes inside a tile follow each other at LPW * 256
    // elements, also a multiple of 8, whenever there is more than one)
    static constexpr int TILE = (LPW * BR * NBOX + 7) / 8 * 8;
    // line exchange areas offset so that the LPW lines of an 8-lane phase fall on distinct banks
    static constexpr int BUFC = (G::BUF + 7) / 8 * 8 + (LPW > 1 ? 8 / LPW : 0);
    static constexpr int WPC = WCfg<M>::CWPC, NT = WCfg<M>::CNT;
    static constexpr int WARP_ELEMS = (NT * TILE + LPW * BUFC + 7) / 8 * 8; // NT tiles, one exchange area
    static constexpr int SMEM = 256 + 16 * WARP_ELEMS * WPC;                // + barriers, + base alignment
    static_assert(NBOX == 1 || (LPW * BR) % 8 == 0, "box offsets must stay 128-byte aligned");
    static_assert(NT * WPC * 8 <= 128, "the barriers fit in front of the tiles");
};

template <int M, bool LP = false>
__global__ void __launch_bounds__(32 * WCfg<M>::CWPC, 3)
    k_dst1_wc(const __grid_constant__ CUtensorMap in_map, const __grid_constant__ CUtensorMap out_map, long ncols,
              long nplanes, const double2 *__restrict__ tw, const double *__restrict__ sn, int *err) {
    using G = WGeom<M>;
    using CG = WColGeom<M>;
    constexpr int      TL = G::TL, LPW = G::LPW, KB = G::KB, N = M - 1, K2 = 2 * KB;
    constexpr int      BR = CG::BR, NBOX = CG::NBOX, NT = CG::NT;
    constexpr uint32_t kBoxBytes = LPW * BR * 16;
    extern __shared__ __align__(128) unsigned char dsm_raw[];
    // 128-byte aligned start of the tiles (the allocation carries 128 bytes of slack for this)
    unsigned char *dsm = dsm_raw + ((128u - (smem_u32(dsm_raw) & 127u)) & 127u);
    const int      lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int      c = lane % LPW, l = lane / LPW; // interleaved: lane = c + LPW l
    uint64_t      *bar = reinterpret_cast<uint64_t *>(dsm) + NT * wq;
    double2       *wbase = reinterpret_cast<double2 *>(dsm + 128) + wq * CG::WARP_ELEMS;
    if ((smem_u32(wbase) & 127u) != 0) { // cannot happen with the layout above; never issue a misaligned copy
        if (lane == 0) atomicExch(err, 2);
        return;
    }
    double2   *xbuf = wbase + NT * CG::TILE + c * CG::BUFC; // the line's exchange area
    const long cgroups = (ncols + LPW - 1) / LPW;
    const long groups = cgroups * nplanes;
    const long stride = (long)gridDim.x * CG::WPC;
    const long g0 = (long)blockIdx.x * CG::WPC + wq;
    if (g0 >= groups) return; // whole warp
    // first column x0 and plane p of group g (32-bit division whenever the groups allow it)
    auto coords = [&](long g, int &x0, int &p) {
        if (groups < (1L << 31)) {
            const unsigned gq = (unsigned)g, cg = (unsigned)cgroups;
            x0 = (int)(gq % cg) * LPW;
            p = (int)(gq / cg);
        } else {
            x0 = (int)((g % cgroups) * LPW);
            p = (int)(g / cgroups);
        }
    };

    auto fetch = [&](long grp, int s) {
        int x0, p;
        coords(grp, x0, p);
        mbar_expect_tx(&bar[s], NBOX * kBoxBytes);
        for (int b = 0; b < NBOX; b++)
            tma_tile_load(wbase + s * CG::TILE + b * LPW * BR, &in_map, x0, b * BR, p, &bar[s]);
    };
    if (lane == 0) {
        for (int u = 0; u < NT; u++) mbar_init(&bar[u], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (lane == 0)
        for (int u = 0; u < NT && g0 + u * stride < groups; u++) fetch(g0 + u * stride, u);
    WConst<M> K;
    K.load(l, tw, sn);

    int  it = 0;
    long failed = -1;
    for (long grp = g0; grp < groups; grp += stride, it++) {
        const int s = it % NT;
        double2  *tile = wbase + s * CG::TILE;
        int        gx0, gpl;
        coords(grp, gx0, gpl);
        const bool live = gx0 + c < ncols;
        if (!mbar_wait_parity(&bar[s], (it / NT) & 1)) {
            if (lane == 0) atomicExch(err, 1);
            failed = grp;
            break;
        }
        if constexpr (LP) w_transform_lp<M, true>([&](int j) { return tile[(j - 1) * LPW + c]; }, xbuf, l, live, K);
        else w_transform<M, true>([&](int j) { return tile[(j - 1) * LPW + c]; }, xbuf, l, live, K);
        // outputs into the tile ([j][c], rows past N untouched), then one tensor store per box
#pragma unroll
        for (int q = 0; q < M / TL; q++) {
            const int p = l + TL * q;
            if (p < N) tile[p * LPW + c] = xbuf[(K2 + 1) * (p / K2) + p % K2];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // tile writes before the store reads
        __syncwarp();
        if (lane == 0) {
            for (int b = 0; b < NBOX; b++) tma_tile_store(&out_map, gx0, b * BR, gpl, tile + b * LPW * BR);
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            // the tile is read by the store before the next load overwrites it
            if (grp + NT * stride < groups) {
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                fetch(grp + NT * stride, s);
            }
        }
        __syncwarp();
    }
    if (lane == 0) {
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); // stores complete before exit
        if (failed >= 0) // copies still in flight get a bounded chance to land
            for (int j = 0; j < NT && failed + j * stride < groups; j++)
                mbar_wait_parity(&bar[(it + j) % NT], ((it + j) / NT) & 1);
    }
}

// ---- columns, CTA tiles: TC = 8 neighbouring columns of all rows arrive as 128-byte-wide boxes of
// a 3-D map (the doubles of a row, row, plane) with 128-byte swizzle, so that each row of a tile
// is one 128-byte piece of global memory (instead of the LPW * 16 bytes of the per-warp tiles
// above) and reading a column of the tile is free of bank conflicts: element (row r, column cc)
// of a box sits at byte r * 128 + 16 * (cc ^ (r % 8)).  The CTA's WPC = TC / LPW warps each
// transform LPW of the tile's columns (lanes line-major: lane = c * TL + l), write the outputs
// back into the tile, and one thread stores the tile with tensor stores and refills the buffer
// with the CTA's tile NT tickets ahead once the store has read it.
template <int M> struct WTile {
    using G = WGeom<M>;
    static constexpr int TL = G::TL, LPW = G::LPW, N = M - 1;
    static constexpr int TC = 8;                  // columns per tile: one 128-byte swizzle span
    static constexpr int WPC = TC / LPW;          // warps per CTA
    static constexpr int BR = N < 256 ? N : 256;  // rows per box
    static constexpr int NBOX = (N + BR - 1) / BR;
    static constexpr int BOX_BYTES = (BR * 128 + 1023) / 1024 * 1024; // boxes stay 1024-byte aligned
    static constexpr int TILE_BYTES = NBOX * BOX_BYTES;
    static constexpr int NT = 2;                  // tiles per CTA (one loads while one is used)
    static constexpr int XBUF = (G::BUF + 7) / 8 * 8; // exchange area per line (elements)
    static constexpr int SMEM = 1024 + NT * TILE_BYTES + 16 * TC * XBUF; // + alignment slack
    static_assert(WPC * LPW == TC, "the warps cover the tile's columns");
};

template <int M, bool LP = false>
__global__ void __launch_bounds__(32 * WTile<M>::WPC)
    k_dst1_wt(const __grid_constant__ CUtensorMap in_map, const __grid_constant__ CUtensorMap out_map, long ncols,
              long nplanes, const double2 *__restrict__ tw, const double *__restrict__ sn, int *err) {
    using G = WGeom<M>;
    using TG = WTile<M>;
    constexpr int TL = G::TL, LPW = G::LPW, KB = G::KB, N = M - 1, K2 = 2 * KB;
    constexpr int TC = TG::TC, BR = TG::BR, NBOX = TG::NBOX, NT = TG::NT;
    __shared__ __align__(8) uint64_t full[NT];
    extern __shared__ __align__(1024) unsigned char wt_raw[];
    // 1024-byte aligned tiles (the 128-byte swizzle pattern repeats every 1024 bytes)
    unsigned char *tiles = wt_raw + ((1024u - (smem_u32(wt_raw) & 1023u)) & 1023u);
    const int      lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    const int      c = lane / TL, l = lane % TL;
    const int      col = wq * LPW + c; // this line's column within the tile
    double2       *xbuf = reinterpret_cast<double2 *>(tiles + NT * TG::TILE_BYTES) + (long)col * TG::XBUF;
    if ((smem_u32(tiles) & 1023u) != 0) { // cannot happen with the slack above; never issue a misaligned copy
        if (threadIdx.x == 0) atomicExch(err, 2);
        return;
    }
    const long cgroups = (ncols + TC - 1) / TC;
    const long groups = cgroups * nplanes;
    if ((long)blockIdx.x >= groups) return; // whole CTA
    const int tickets = (int)((groups - blockIdx.x + gridDim.x - 1) / gridDim.x);
    auto coords = [&](int t, int &x0, int &p) {
        const long g = (long)blockIdx.x + (long)t * gridDim.x;
        x0 = (int)(g % cgroups) * TC;
        p = (int)(g / cgroups);
    };
    auto fetch = [&](int t) { // thread 0: ticket t into buffer t % NT
        int x0, p;
        coords(t, x0, p);
        unsigned char *dst = tiles + (t % NT) * TG::TILE_BYTES;
        mbar_expect_tx(&full[t % NT], (uint32_t)(NBOX * BR * 128));
        for (int b = 0; b < NBOX; b++) tma_load_3d(dst + b * TG::BOX_BYTES, &in_map, 2 * x0, b * BR, p, &full[t % NT]);
    };
    if (threadIdx.x == 0) {
        for (int u = 0; u < NT; u++) mbar_init(&full[u], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int u = 0; u < NT && u < tickets; u++) fetch(u);
    }
    __syncthreads();
    WConst<M> K;
    K.load(l, tw, sn);

    int failed = -1;
    for (int t = 0; t < tickets; t++) {
        const int s = t % NT;
        // every thread waits (bounded); the CTA leaves together if any wait expired
        const bool ok = mbar_wait_parity(&full[s], (uint32_t)((t / NT) & 1));
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) atomicExch(err, 1);
            failed = t;
            break;
        }
        unsigned char *tile = tiles + s * TG::TILE_BYTES;
        auto at = [&](int row) -> double2 * { // element (row, col) of the tile
            const int b = row / BR, r = row - b * BR;
            return reinterpret_cast<double2 *>(tile + b * TG::BOX_BYTES + r * 128 + ((col ^ (r & 7)) << 4));
        };
        int x0, p;
        coords(t, x0, p);
        const bool live = x0 + col < ncols;
        if constexpr (LP) w_transform_lp<M, false>([&](int j) { return *at(j - 1); }, xbuf, l, live, K);
        else w_transform<M, false>([&](int j) { return *at(j - 1); }, xbuf, l, live, K);
#pragma unroll
        for (int q = 0; q < M / TL; q++) {
            const int pp = l + TL * q;
            if (pp < N) *at(pp) = xbuf[(K2 + 1) * (pp / K2) + pp % K2];
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); // tile writes before the store reads
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int b = 0; b < NBOX; b++) tma_store_3d(&out_map, 2 * x0, b * BR, p, tile + b * TG::BOX_BYTES);
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            if (t + NT < tickets) {
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); // the store has read the tile
                fetch(t + NT);
            }
        }
    }
    if (threadIdx.x == 0) {
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); // stores complete before exit
        if (failed >= 0) // loads still in flight get a bounded chance to land
            for (int u = failed; u < tickets && u < failed + NT; u++) mbar_wait_parity(&full[u % NT], (uint32_t)((u / NT) & 1));
    }
}

// ---------------------------------------------- direct DST (any n, dense sine matrix) ----
// out_k = sqrt(2/(n+1)) sum_m in_m sin(pi (k+1)(m+1)/(n+1)); `mat` holds the n*n sines.
constexpr int kDenseThreads = 128;
template <bool STRIDED>
__global__ void __launch_bounds__(kDenseThreads)
    k_dst1_dense(const double2 *__restrict__ in, double2 *__restrict__ out, int n, long nlines, long in_ld,
                 long out_ld, long plane_stride, const double *__restrict__ mat) {
    extern __shared__ __align__(128) unsigned char smem_dense[];
    double2   *x = reinterpret_cast<double2 *>(smem_dense);
    const long line = blockIdx.x;
    const long pbase = STRIDED ? (long)blockIdx.y * plane_stride : 0;
    for (int m = threadIdx.x; m < n; m += blockDim.x)
        x[m] = STRIDED ? in[pbase + line + (long)m * in_ld] : in[line * in_ld + m];
    __syncthreads();
    const double coef = sqrt(2.0 / (n + 1));
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const double *row = mat + (long)k * n;
        double        sr = 0.0, si = 0.0;
        for (int m = 0; m < n; m++) {
            const double s = __ldg(row + m);
            sr = fma(s, x[m].x, sr);
            si = fma(s, x[m].y, si);
        }
        const double2 r = make_double2(coef * sr, coef * si);
        if (STRIDED) out[pbase + line + (long)k * out_ld] = r;
        else out[line * out_ld + k] = r;
    }
}

// ------------------------------------------------------------------ tables --------
__global__ void k_make_tables(int m, double2 *tw, double *sn) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)t / (double)m, &s, &c); // exp(-2 pi i t/m) = c - i s
        tw[t] = make_double2(c, -s);
        sn[t] = sinpi((double)t / (double)m);
    }
}

__global__ void k_make_dense(int n, double *mat) {
    const long tot = (long)n * n;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
        const long k = q / n, m = q % n;
        // (k+1)(m+1) reduced mod 2(n+1) keeps the argument of sinpi in [0, 2)
        const long   num = ((k + 1) * (m + 1)) % (2L * (n + 1));
        mat[q] = sinpi((double)num / (double)(n + 1));
    }
}

int tables_for(Ctx *c, int m, const double2 **tw, const double **sn) {
    std::lock_guard<std::mutex> g(c->mu);
    auto it = c->tw.find(m);
    if (it == c->tw.end()) {
        double2 *t2 = nullptr;
        double  *s1 = nullptr;
        HH_CUDA(cudaMalloc(&t2, sizeof(double2) * (size_t)m));
        HH_CUDA(cudaMalloc(&s1, sizeof(double) * (size_t)m));
        k_make_tables<<<(m + 255) / 256, 256, 0, c->stream>>>(m, t2, s1);
        HH_CUDA(cudaGetLastError());
        c->launches++;
        c->tw[m] = t2;
        c->sn[m] = s1;
        it = c->tw.find(m);
    }
    *tw = it->second;
    *sn = c->sn[m];
    return HH_OK;
}

int prepare_dst(Ctx *c, int n) {
    const int m = n + 1;
    if (m >= 64 && m <= 8192 && (m & (m - 1)) == 0) {
        const double2 *tw;
        const double  *sn;
        return tables_for(c, m, &tw, &sn);
    }
    if (n >= 1 && n <= 4096) {
        const double *mat;
        return dense_for(c, n, &mat);
    }
    return HH_OK; // lengths the transforms refuse fail at solve time
}

int dense_for(Ctx *c, int n, const double **mat) {
    std::lock_guard<std::mutex> g(c->mu);
    auto it = c->dense.find(n);
    if (it == c->dense.end()) {
        double *d = nullptr;
        HH_CUDA(cudaMalloc(&d, sizeof(double) * (size_t)n * (size_t)n));
        k_make_dense<<<256, 256, 0, c->stream>>>(n, d);
        HH_CUDA(cudaGetLastError());
        c->launches++;
        c->dense[n] = d;
        it = c->dense.find(n);
    }
    *mat = it->second;
    return HH_OK;
}

// -------------------------------------------------------------------- launch ------
struct DstArgs {
    const double2 *in;
    double2       *out;
    long           nlines, planes, in_ld, out_ld, in_plane, out_plane;
    int            rows_kernel = 0; // contiguous rows: 0 default, 1 CTA ring, 2 per-warp (2048: the Stockham kernel)
};

template <int M, bool IS, bool OS> static int launch_fft(Ctx *c, const DstArgs &a) {
    using G = DstGeom<M>;
    const double2 *tw;
    const double  *sn;
    HH_TRY(tables_for(c, M, &tw, &sn));
    HH_CUDA(cudaFuncSetAttribute(k_dst1<M, IS, OS>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
    dim3 grid((unsigned)((a.nlines + G::S - 1) / G::S), (unsigned)a.planes);
    k_dst1<M, IS, OS><<<grid, G::NT, G::SMEM, c->stream>>>(a.in, a.out, a.nlines, a.in_ld, a.out_ld, a.in_plane,
                                                            a.out_plane, tw, sn, c->err_word);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

template <int M, bool LP, bool UPD = false> static int launch_wr(Ctx *c, const DstArgs &a) {
    using G = WGeom<M>;
    using RG = WRing<M>;
    const double2 *tw;
    const double  *sn;
    HH_TRY(tables_for(c, M, &tw, &sn));
    HH_CUDA(cudaFuncSetAttribute(k_dst1_wr<M, LP, UPD>, cudaFuncAttributeMaxDynamicSharedMemorySize, RG::SMEM));
    int dev = 0, sms = 148, per_sm = 0;
    HH_CUDA(cudaGetDevice(&dev));
    HH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dst1_wr<M, LP, UPD>, 32 * RG::WPC, RG::SMEM));
    const long groups = (a.nlines * a.planes + G::LPW - 1) / G::LPW;
    const long ctas = std::min<long>((groups + RG::WPC - 1) / RG::WPC, (long)std::max(1, per_sm) * sms);
    k_dst1_wr<M, LP, UPD><<<(unsigned)ctas, 32 * RG::WPC, RG::SMEM, c->stream>>>(
        a.in, a.out, a.nlines, a.planes, a.in_ld, a.out_ld, a.in_plane, a.out_plane, tw, sn, c->err_word);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

template <int M, bool LP, bool UPD = false> static int launch_wp(Ctx *c, const DstArgs &a) {
    using G = WGeom<M>;
    const double2 *tw;
    const double  *sn;
    HH_TRY(tables_for(c, M, &tw, &sn));
    HH_CUDA(cudaFuncSetAttribute(k_dst1_w<M, LP, UPD>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
    int dev = 0, sms = 148, per_sm = 0;
    HH_CUDA(cudaGetDevice(&dev));
    HH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dst1_w<M, LP, UPD>, 32 * G::WPC, G::SMEM));
    const long groups = (a.nlines * a.planes + G::LPW - 1) / G::LPW;
    const long ctas = std::min<long>((groups + G::WPC - 1) / G::WPC, (long)std::max(1, per_sm) * sms);
    k_dst1_w<M, LP, UPD><<<(unsigned)ctas, 32 * G::WPC, G::SMEM, c->stream>>>(a.in, a.out, a.nlines, a.planes, a.in_ld, a.out_ld,
                                                                     a.in_plane, a.out_plane, tw, sn, c->err_word,
                                                                     c->inject_word);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

template <int M, bool LP, bool UPD = false> static int launch_w2(Ctx *c, const DstArgs &a) {
    using G = W2Geom<M>;
    const double2 *tw;
    const double  *sn;
    HH_TRY(tables_for(c, M, &tw, &sn));
    HH_CUDA(cudaFuncSetAttribute(k_dst1_w2<M, LP, UPD>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM));
    int dev = 0, sms = 148, per_sm = 0;
    HH_CUDA(cudaGetDevice(&dev));
    HH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_dst1_w2<M, LP, UPD>, 64 * G::TPC, G::SMEM));
    const long lines = a.nlines * a.planes;
    const long ctas = std::min<long>((lines + G::TPC - 1) / G::TPC, (long)std::max(1, per_sm) * sms);
    k_dst1_w2<M, LP, UPD><<<(unsigned)ctas, 64 * G::TPC, G::SMEM, c->stream>>>(a.in, a.out, a.nlines, a.planes, a.in_ld,
                                                                        a.out_ld, a.in_plane, a.out_plane, tw, sn,
                                                                        c->err_word);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

// rows kernel: a.rows_kernel 1 = the CTA ring, 2 = per-warp buffers, 0 = the length's default
template <int M, bool LP, bool UPD = false> static int launch_w(Ctx *c, const DstArgs &a) {
    const bool ring = a.rows_kernel == 0 ? (bool)WCfg<M>::RING : a.rows_kernel == 1;
    return ring ? launch_wr<M, LP, UPD>(c, a) : launch_wp<M, LP, UPD>(c, a);
}

// LP: single-precision arithmetic where the persistent-warp kernels serve (n + 1 = 64 .. 2048);
// the other kernels compute in FP64 either way.
// UPD: out <- out - result, only where the persistent-warp kernels serve (rows_update_supported)
template <bool IS, bool OS, bool LP = false, bool UPD = false> static int launch_dispatch(Ctx *c, int n, const DstArgs &a) {
    if (n < 1) { set_error("DST length must be >= 1 (got %d)", n); return HH_ERR_INVALID; }
    if (a.nlines <= 0 || a.planes <= 0) return HH_OK;
    if (a.planes > 65535) { set_error("DST: too many planes (%ld)", a.planes); return HH_ERR_INVALID; }
    if (!IS && (((uintptr_t)a.in) & 15)) {
        set_error("DST rows must be 16-byte aligned");
        return HH_ERR_INVALID;
    }
    if (!IS && !OS) {
        switch (n + 1) { // contiguous rows: persistent-warp kernels
        case 64: return launch_w<64, LP, UPD>(c, a);
        case 128: return launch_w<128, LP, UPD>(c, a);
        case 256: return launch_w<256, LP, UPD>(c, a);
        case 512: return launch_w<512, LP, UPD>(c, a);
        case 1024: return launch_w<1024, LP, UPD>(c, a);
        case 2048: // two warps per line; rows_kernel 2 keeps the (FP64) Stockham kernel below
            if (a.rows_kernel != 2) return launch_w2<2048, LP, UPD>(c, a);
            break;
        default: break;
        }
    }
    if constexpr (UPD) {
        set_error("DST length %d: no subtracting form for these kernels", n);
        return HH_ERR_UNSUPPORTED;
    }
    switch (n + 1) {
    case 64: return launch_fft<64, IS, OS>(c, a);
    case 128: return launch_fft<128, IS, OS>(c, a);
    case 256: return launch_fft<256, IS, OS>(c, a);
    case 512: return launch_fft<512, IS, OS>(c, a);
    case 1024: return launch_fft<1024, IS, OS>(c, a);
    case 2048: return launch_fft<2048, IS, OS>(c, a);
    case 4096: return launch_fft<4096, IS, OS>(c, a);
    case 8192: return launch_fft<8192, IS, OS>(c, a);
    default: break;
    }
    if (n > 4096) {
        set_error("DST length %d: n+1 must be a power of two (64..8192) or n <= 4096", n);
        return HH_ERR_UNSUPPORTED;
    }
    if (IS != OS) {
        set_error("DST length %d: transposing modes need n+1 a power of two", n);
        return HH_ERR_UNSUPPORTED;
    }
    const double *mat;
    HH_TRY(dense_for(c, n, &mat));
    const size_t shm = sizeof(double2) * (size_t)n;
    if (shm > 48 * 1024)
        HH_CUDA(cudaFuncSetAttribute(k_dst1_dense<IS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    dim3 grid((unsigned)a.nlines, (unsigned)a.planes);
    k_dst1_dense<IS><<<grid, kDenseThreads, shm, c->stream>>>(a.in, a.out, n, a.nlines, a.in_ld, a.out_ld,
                                                              a.in_plane, mat);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

bool rows_update_supported(int n, int rows_kernel) {
    const int m = n + 1;
    return (m >= 64 && m <= 1024 && (m & (m - 1)) == 0) || (m == 2048 && rows_kernel != 2);
}

int launch_dst_rows_update(Ctx *c, int n, long rows, const double2 *in, long in_ld, double2 *out, long out_ld,
                           int rows_kernel) {
    DstArgs a{in, out, rows, 1, in_ld, out_ld, 0, 0, rows_kernel};
    return launch_dispatch<false, false, true, true>(c, n, a);
}

int launch_dst_rows(Ctx *c, int n, long rows, const double2 *in, long in_ld, double2 *out, long out_ld, bool lp,
                    int rows_kernel) {
    DstArgs a{in, out, rows, 1, in_ld, out_ld, 0, 0, rows_kernel};
    return lp ? launch_dispatch<false, false, true>(c, n, a) : launch_dispatch<false, false>(c, n, a);
}

// 4-D tensor map over (re/im, column x, row j, plane) of complex doubles, boxes of `box_cols`
// columns by `box_rows` rows.
static int encode_col_map(CUtensorMap *map, const double2 *base, long ncols, long rows, long planes, long ld,
                          long plane_stride, int box_cols, int box_rows) {
    const unsigned long long dims[4] = {2, (unsigned long long)ncols, (unsigned long long)rows,
                                        (unsigned long long)planes};
    const unsigned long long strides[3] = {16, (unsigned long long)ld * 16, (unsigned long long)plane_stride * 16};
    const unsigned           box[4] = {2, (unsigned)box_cols, (unsigned)box_rows, 1};
    return encode_tensor_map(map, base, 4, dims, strides, box);
}

int encode_tensor_map(CUtensorMap *map, const void *base, int rank, const unsigned long long *dims,
                      const unsigned long long *strides, const unsigned *box, bool swizzle128) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void                           *fn = nullptr;
        HH_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (!fn || q != cudaDriverEntryPointSuccess) {
            set_error("cuTensorMapEncodeTiled is not available");
            return HH_ERR_CUDA;
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    cuuint64_t d[5], s[4];
    cuuint32_t b[5], e[5] = {1, 1, 1, 1, 1};
    for (int i = 0; i < rank; i++) {
        d[i] = dims[i];
        b[i] = box[i];
        if (i + 1 < rank) s[i] = strides[i];
    }
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, const_cast<void *>(base), d, s, b, e,
                              CU_TENSOR_MAP_INTERLEAVE_NONE,
                              swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return HH_ERR_CUDA;
    }
    return HH_OK;
}

template <int M>
static int launch_wc(Ctx *c, long ncols, long planes, const double2 *in, long ld, long plane_stride, double2 *out,
                     bool lp) {
    using G = WGeom<M>;
    using CG = WColGeom<M>;
    const double2 *tw;
    const double  *sn;
    HH_TRY(tables_for(c, M, &tw, &sn));
    CUtensorMap in_map, out_map;
    HH_TRY(encode_col_map(&in_map, in, ncols, M - 1, planes, ld, plane_stride, G::LPW, CG::BR));
    HH_TRY(encode_col_map(&out_map, out, ncols, M - 1, planes, ld, plane_stride, G::LPW, CG::BR));
    auto kern = lp ? k_dst1_wc<M, true> : k_dst1_wc<M, false>;
    HH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CG::SMEM));
    int dev = 0, sms = 148, per_sm = 0;
    HH_CUDA(cudaGetDevice(&dev));
    HH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * CG::WPC, CG::SMEM));
    const long groups = (ncols + G::LPW - 1) / G::LPW * planes;
    const long ctas = std::min<long>((groups + CG::WPC - 1) / CG::WPC, (long)std::max(1, per_sm) * sms);
    kern<<<(unsigned)ctas, 32 * CG::WPC, CG::SMEM, c->stream>>>(in_map, out_map, ncols, planes, tw, sn, c->err_word);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

// (double, row, plane) map of column tiles: boxes of 16 doubles (8 complex columns) by br rows,
// 128-byte swizzle
static int encode_tile_map(CUtensorMap *map, const double2 *base, long ncols, long rows, long planes, long ld,
                           long plane_stride, int box_rows) {
    const unsigned long long dims[3] = {2ULL * (unsigned long long)ncols, (unsigned long long)rows,
                                        (unsigned long long)planes};
    const unsigned long long strides[2] = {(unsigned long long)ld * 16, (unsigned long long)plane_stride * 16};
    const unsigned           box[3] = {16, (unsigned)box_rows, 1};
    return encode_tensor_map(map, base, 3, dims, strides, box, true);
}

template <int M>
static int launch_wt(Ctx *c, long ncols, long planes, const double2 *in, long ld, long plane_stride, double2 *out,
                     bool lp) {
    using TG = WTile<M>;
    const double2 *tw;
    const double  *sn;
    HH_TRY(tables_for(c, M, &tw, &sn));
    CUtensorMap in_map, out_map;
    HH_TRY(encode_tile_map(&in_map, in, ncols, M - 1, planes, ld, plane_stride, TG::BR));
    HH_TRY(encode_tile_map(&out_map, out, ncols, M - 1, planes, ld, plane_stride, TG::BR));
    auto kern = lp ? k_dst1_wt<M, true> : k_dst1_wt<M, false>;
    HH_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, TG::SMEM));
    int dev = 0, sms = 148, per_sm = 0;
    HH_CUDA(cudaGetDevice(&dev));
    HH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    HH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * TG::WPC, TG::SMEM));
    const long groups = (ncols + TG::TC - 1) / TG::TC * planes;
    const long ctas = std::min<long>(groups, (long)std::max(1, per_sm) * sms);
    kern<<<(unsigned)ctas, 32 * TG::WPC, TG::SMEM, c->stream>>>(in_map, out_map, ncols, planes, tw, sn, c->err_word);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

int launch_dst_cols(Ctx *c, int n, long ncols, long planes, const double2 *in, long ld, long plane_stride,
                    double2 *out, bool lp, int kern) {
    // CTA tiles of 8 swizzled columns: the tensor map covers 2 * ncols doubles per row (an
    // 8-column box needs ncols >= 8), rows ld * 16 and planes plane_stride * 16 bytes apart
    if (kern == 0 && planes > 0 && ncols >= 8 && ld * 16 < (1L << 40) && plane_stride * 16 < (1L << 40) &&
        planes < (1L << 31) && ((uintptr_t)in & 15) == 0 && ((uintptr_t)out & 15) == 0) {
        switch (n + 1) {
        case 64: return launch_wt<64>(c, ncols, planes, in, ld, plane_stride, out, lp);
        case 128: return launch_wt<128>(c, ncols, planes, in, ld, plane_stride, out, lp);
        case 256: return launch_wt<256>(c, ncols, planes, in, ld, plane_stride, out, lp);
        case 512: return launch_wt<512>(c, ncols, planes, in, ld, plane_stride, out, lp);
        default: break;
        }
    }
    // tensor maps need 16-byte aligned bases (always true for double2) and byte strides below 2^40
    // (the tensor-map box never exceeds the tensor: at least LPW columns)
    if (planes > 0 && ld * 16 < (1L << 40) && plane_stride * 16 < (1L << 40) && planes < (1L << 31)) {
        switch (n + 1) {
        case 64: if (ncols >= WGeom<64>::LPW) return launch_wc<64>(c, ncols, planes, in, ld, plane_stride, out, lp); break;
        case 128: if (ncols >= WGeom<128>::LPW) return launch_wc<128>(c, ncols, planes, in, ld, plane_stride, out, lp); break;
        case 256: if (ncols >= WGeom<256>::LPW) return launch_wc<256>(c, ncols, planes, in, ld, plane_stride, out, lp); break;
        case 512: if (ncols >= WGeom<512>::LPW) return launch_wc<512>(c, ncols, planes, in, ld, plane_stride, out, lp); break;
        case 1024: if (ncols >= WGeom<1024>::LPW) return launch_wc<1024>(c, ncols, planes, in, ld, plane_stride, out, lp); break;
        default: break;
        }
    }
    DstArgs a{in, out, ncols, planes, ld, ld, plane_stride, plane_stride};
    return launch_dispatch<true, true>(c, n, a);
}

} // namespace hh
