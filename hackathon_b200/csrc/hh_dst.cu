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

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// 1D bulk copy global -> shared completing on `bar` (addresses 16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void tma_bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// bounded wait on phase 0; returns false if the copy did not land within the budget
__device__ __forceinline__ bool mbar_wait0(uint64_t *bar) {
    const uint32_t a = smem_u32(bar);
    for (long it = 0; it < (1L << 26); it++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a)
            : "memory");
        if (done) return true;
    }
    return false;
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

// ------------------------------------------ one warp per line: M = 1024 rows ------
// The same transform for contiguous rows of length N = 1023 with one warp per line and M = 32 x 32:
//   lane b loads x_j and the mirror x_{M-j} for j = b + 32 q straight from global memory
//   (coalesced), forms y_j in registers, runs a 32-point DFT over q, twiddles, and exchanges
//   through one padded transpose; the second 32-point DFT leaves Y_{b + 32 k2} in lane b.
//   Post-processing runs on blocks (lane t owns k in [16t, 16t + 16)), so the prefix sum of the
//   odd outputs is a sequential sum plus one warp scan; the outputs go back through shared
//   memory so that the global stores are coalesced.
// Shared-memory traffic per point: transpose (write + read), Y (write + read), S (write + read);
// the staged design above makes about twice as many passes.

// sin(pi m / 32), m = 0..16
__device__ __forceinline__ constexpr double sinpi32(int m) {
    constexpr double s[17] = {0.0,
                              0.098017140329560601994,
                              0.19509032201612826785,
                              0.29028467725446236764,
                              0.38268343236508977173,
                              0.47139673682599764856,
                              0.55557023301960222474,
                              0.63439328416364549822,
                              0.7071067811865475244,
                              0.77301045336273696081,
                              0.83146961230254523708,
                              0.88192126434835502971,
                              0.92387953251128675613,
                              0.95694033573220886494,
                              0.98078528040323044913,
                              0.99518472667219688624,
                              1.0};
    return s[m];
}
// sin(pi q / 32) and cos(pi q / 32) for q = 0..31
__device__ __forceinline__ constexpr double sin_q32(int q) { return q <= 16 ? sinpi32(q) : sinpi32(32 - q); }
__device__ __forceinline__ constexpr double cos_q32(int q) { return q <= 16 ? sinpi32(16 - q) : -sinpi32(q - 16); }

// v * exp(-2 pi i t / 32), t = 0..15: cos(2 pi t/32) = sin(pi (8 - t)/16) = sinpi32(16 - 2t)
template <int t> __device__ __forceinline__ double2 tw32_mul(double2 v) {
    if constexpr (t == 0) return v;
    else if constexpr (t == 8) return make_double2(v.y, -v.x);
    else if constexpr (t == 4) {
        constexpr double r = sinpi32(8);
        return make_double2((v.x + v.y) * r, (v.y - v.x) * r);
    } else if constexpr (t == 12) {
        constexpr double r = sinpi32(8);
        return make_double2((v.y - v.x) * r, -(v.x + v.y) * r);
    } else {
        constexpr double c = t < 8 ? sinpi32(16 - 2 * t) : -sinpi32(2 * t - 16), s = sinpi32(t < 8 ? 2 * t : 32 - 2 * t);
        return make_double2(fma(v.x, c, v.y * s), fma(v.y, c, -(v.x * s)));
    }
}
template <int SPAN, int J> struct Dif32Butterflies {
    __device__ __forceinline__ static void run(double2 (&v)[32], int start) {
        if constexpr (J < SPAN) {
            const double2 a = v[start + J], b = v[start + J + SPAN];
            v[start + J] = cadd(a, b);
            v[start + J + SPAN] = tw32_mul<J * (16 / SPAN)>(csub(a, b));
            Dif32Butterflies<SPAN, J + 1>::run(v, start);
        }
    }
};
template <int SPAN, int START> struct Dif32Stage {
    __device__ __forceinline__ static void run(double2 (&v)[32]) {
        if constexpr (START < 32) {
            Dif32Butterflies<SPAN, 0>::run(v, START);
            Dif32Stage<SPAN, START + 2 * SPAN>::run(v);
        }
    }
};
template <int SPAN> struct Dif32All {
    __device__ __forceinline__ static void run(double2 (&v)[32]) {
        if constexpr (SPAN >= 1) {
            Dif32Stage<SPAN, 0>::run(v);
            Dif32All<SPAN / 2>::run(v);
        }
    }
};
// forward 32-point DFT in registers; X[k] = v[bitrev5(k)]
__device__ __forceinline__ void dft32(double2 (&v)[32]) { Dif32All<16>::run(v); }

constexpr int kDstWarps = 2;                  // warps per CTA
constexpr int kDstWarpBuf = 1088;             // double2 per buffer: max(32 x 33, 1024 + 1024/16)
__host__ __device__ constexpr int hibit(int k) { return k <= 1 ? 0 : 1 + hibit(k >> 1); }
__host__ __device__ constexpr int t33(int i, int j) { return 33 * i + j; }          // transpose layout
__host__ __device__ constexpr int p16(int k) { return k + (k >> 4); }               // Y layout
__host__ __device__ constexpr int o33(int p) { return 33 * (p >> 5) + (p & 31); }   // output layout

// bounded wait on an mbarrier phase; false if it did not complete within the budget
__device__ __forceinline__ bool mbar_wait_parity(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long it = 0; it < (1L << 26); it++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Persistent warps: warp w of the grid transforms lines w, w + W, w + 2W, ... (W warps in all),
// each line (plane = g / nlines, line = g % nlines) at in + plane*in_plane + line*in_ld with x_1..x_N
// at offsets 0..N-1, and likewise for the output.  Each warp owns two line buffers: while it
// transforms one line, the TMA brings in its next.  in and out may be the same buffer.
__global__ void __launch_bounds__(32 * kDstWarps, 3)
    k_dst1_w1024(const double2 *in, double2 *out, long nlines, long nplanes, long in_ld, long out_ld, long in_plane,
                 long out_plane, const double2 *__restrict__ tw, const double *__restrict__ sn, int *err) {
    constexpr int      M = 1024, N = M - 1;
    constexpr uint32_t kBytes = N * 16;
    extern __shared__ __align__(128) unsigned char dsm[];
    const int  lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
    uint64_t  *bar = reinterpret_cast<uint64_t *>(dsm) + 2 * wq;
    double2   *bufs = reinterpret_cast<double2 *>(dsm + 16 * kDstWarps) + 2 * wq * kDstWarpBuf;
    const long total = nlines * nplanes;
    const long stride = (long)gridDim.x * kDstWarps;
    const long g0 = (long)blockIdx.x * kDstWarps + wq;
    if (g0 >= total) return; // whole warp
    const double2 zero = make_double2(0.0, 0.0);

    auto src_of = [&](long g) { return in + (g / nlines) * in_plane + (g % nlines) * in_ld; };
    auto dst_of = [&](long g) { return out + (g / nlines) * out_plane + (g % nlines) * out_ld; };
    if (lane == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (lane == 0) {
        mbar_expect_tx(&bar[0], kBytes);
        tma_bulk_load(bufs, src_of(g0), kBytes, &bar[0]);
        if (g0 + stride < total) {
            mbar_expect_tx(&bar[1], kBytes);
            tma_bulk_load(bufs + kDstWarpBuf, src_of(g0 + stride), kBytes, &bar[1]);
        }
    }

    // per-lane constants: sin, cos(pi lane / M) and the twiddles W_M^{lane a}, W_M^{8 lane b}
    const double sb = __ldg(sn + lane), cb = __ldg(sn + M / 2 - lane);
    double2      twa[8], twb[4];
#pragma unroll
    for (int a = 0; a < 8; a++) twa[a] = __ldg(tw + ((lane * a) & (M - 1)));
#pragma unroll
    for (int b = 0; b < 4; b++) twb[b] = __ldg(tw + ((8 * lane * b) & (M - 1)));
    const double coef = sqrt(2.0 / M);

    int  i = 0;
    long failed = -1;
    for (long g = g0; g < total; g += stride, i++) {
        double2 *buf = bufs + (i & 1) * kDstWarpBuf;
        if (!mbar_wait_parity(&bar[i & 1], (i >> 1) & 1)) {
            if (lane == 0) atomicExch(err, 1);
            failed = g;
            break;
        }

        // The per-lane sines and twiddles are re-formed for every line: an empty asm hides their
        // inputs from loop-invariant hoisting, which would otherwise pin ~90 registers.
        double sbl = sb, cbl = cb;
        asm volatile("" : "+d"(sbl), "+d"(cbl));
#pragma unroll
        for (int a = 0; a < 8; a++) asm volatile("" : "+d"(twa[a].x), "+d"(twa[a].y));
#pragma unroll
        for (int b = 0; b < 4; b++) asm volatile("" : "+d"(twb[b].x), "+d"(twb[b].y));

        // ---- y_j = sin(pi j/M)(x_j + x_{M-j}) + (x_j - x_{M-j})/2,  j = lane + 32 q
        double2 v[32];
#pragma unroll
        for (int q = 0; q < 32; q++) {
            const int j = lane + 32 * q;
            double2   a = zero, m = zero;
            if (q > 0 || lane > 0) {
                a = buf[j - 1];
                m = buf[M - j - 1];
            }
            const double s = fma(sbl, cos_q32(q), cbl * sin_q32(q)); // sin(pi (lane + 32 q) / M)
            v[q] = make_double2(fma(s, a.x + m.x, 0.5 * (a.x - m.x)), fma(s, a.y + m.y, 0.5 * (a.y - m.y)));
        }
        __syncwarp(); // the raw line is consumed; the buffer becomes the exchange area

        // ---- 32-point DFTs over q, twiddle W_M^{lane k1}, transpose
        dft32(v);
#pragma unroll
        for (int k1 = 0; k1 < 32; k1++)
            buf[t33(k1, lane)] = k1 ? cmul(v[bitrev_c<32>(k1)], cmul(twa[k1 & 7], twb[k1 >> 3])) : v[0];
        __syncwarp();
#pragma unroll
        for (int j1 = 0; j1 < 32; j1++) v[j1] = buf[t33(lane, j1)];
        __syncwarp();

        // ---- 32-point DFTs over j1: Y_{lane + 32 k2} = v[bitrev(k2)]
        dft32(v);
#pragma unroll
        for (int k2 = 0; k2 < 32; k2++) buf[p16(lane + 32 * k2)] = v[bitrev_c<32>(k2)];
        __syncwarp();

        // ---- post-processing on blocks k = 16 lane + u
        double2 cs[16], ev[16];
        double2 run = zero;
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int     k = 16 * lane + u;
            const double2 yk = buf[p16(k)];
            if (k == 0) {
                cs[u] = make_double2(0.5 * yk.x, 0.5 * yk.y);
                ev[u] = zero;
            } else {
                const double2 ym = buf[p16(M - k)];
                cs[u] = make_double2(0.5 * (yk.x + ym.x), 0.5 * (yk.y + ym.y));
                ev[u] = make_double2(0.5 * (ym.y - yk.y), -0.5 * (ym.x - yk.x)); // (Y_{M-k} - Y_k)/(2i)
            }
            run = cadd(run, cs[u]);
            cs[u] = run;
        }
        double2 incl = run;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double ox = __shfl_up_sync(0xffffffffu, incl.x, off), oy = __shfl_up_sync(0xffffffffu, incl.y, off);
            if (lane >= off) { incl.x += ox; incl.y += oy; }
        }
        const double2 pre = csub(incl, run);
        __syncwarp(); // every read of Y is done
#pragma unroll
        for (int u = 0; u < 16; u++) {
            const int k = 16 * lane + u;
            buf[o33(2 * k)] = cscale(cadd(pre, cs[u]), coef);     // S_{2k+1} at offset 2k
            if (k > 0) buf[o33(2 * k - 1)] = cscale(ev[u], coef); // S_{2k}   at offset 2k-1
        }
        __syncwarp();
        double2 *dst = dst_of(g);
#pragma unroll
        for (int q = 0; q < 32; q++) {
            const int p = lane + 32 * q;
            if (p < N) dst[p] = buf[o33(p)];
        }
        __syncwarp();
        // the buffer is free again: bring in the line after next (generic-proxy reads of the
        // buffer are ordered before the asynchronous copy that overwrites it)
        if (lane == 0 && g + 2 * stride < total) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bar[i & 1], kBytes);
            tma_bulk_load(buf, src_of(g + 2 * stride), kBytes, &bar[i & 1]);
        }
    }
    // after an expired wait, give the copies still in flight (this buffer's and the next one's)
    // a bounded chance to land before the CTA's shared memory is released
    if (failed >= 0 && lane == 0) {
        mbar_wait_parity(&bar[i & 1], (i >> 1) & 1);
        if (failed + stride < total) mbar_wait_parity(&bar[(i + 1) & 1], ((i + 1) >> 1) & 1);
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

static int launch_w1024(Ctx *c, const DstArgs &a) {
    const double2 *tw;
    const double  *sn;
    HH_TRY(tables_for(c, 1024, &tw, &sn));
    const int shm = 16 * kDstWarps + (int)(sizeof(double2) * kDstWarpBuf * 2 * kDstWarps);
    HH_CUDA(cudaFuncSetAttribute(k_dst1_w1024, cudaFuncAttributeMaxDynamicSharedMemorySize, shm));
    int dev = 0, sms = 148;
    HH_CUDA(cudaGetDevice(&dev));
    HH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long lines = a.nlines * a.planes;
    const long ctas = std::min<long>((lines + kDstWarps - 1) / kDstWarps, 3L * sms);
    k_dst1_w1024<<<(unsigned)ctas, 32 * kDstWarps, shm, c->stream>>>(a.in, a.out, a.nlines, a.planes, a.in_ld, a.out_ld,
                                                                     a.in_plane, a.out_plane, tw, sn, c->err_word);
    HH_CUDA(cudaGetLastError());
    c->launches++;
    return HH_OK;
}

template <bool IS, bool OS> static int launch_dispatch(Ctx *c, int n, const DstArgs &a) {
    if (n < 1) { set_error("DST length must be >= 1 (got %d)", n); return HH_ERR_INVALID; }
    if (a.nlines <= 0 || a.planes <= 0) return HH_OK;
    if (a.planes > 65535) { set_error("DST: too many planes (%ld)", a.planes); return HH_ERR_INVALID; }
    if (!IS && (((uintptr_t)a.in) & 15)) {
        set_error("DST rows must be 16-byte aligned");
        return HH_ERR_INVALID;
    }
    if (n == 1023 && !IS && !OS) return launch_w1024(c, a);
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

int launch_dst_rows(Ctx *c, int n, long rows, const double2 *in, long in_ld, double2 *out, long out_ld) {
    DstArgs a{in, out, rows, 1, in_ld, out_ld, 0, 0};
    return launch_dispatch<false, false>(c, n, a);
}

int launch_dst_cols(Ctx *c, int n, long ncols, long planes, const double2 *in, long ld, long plane_stride,
                    double2 *out) {
    DstArgs a{in, out, ncols, planes, ld, ld, plane_stride, plane_stride};
    return launch_dispatch<true, true>(c, n, a);
}

} // namespace hh
