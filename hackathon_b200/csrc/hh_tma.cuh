// TMA and mbarrier helpers shared by the transform and line-solve kernels (sm_100a).
//
// Every wait is bounded: mbar_wait_parity polls at most 2^26 times and reports failure, so a
// copy that never lands cannot hang a kernel.  Every copy lands in the issuing CTA's own
// shared memory only.
#ifndef HH_TMA_CUH
#define HH_TMA_CUH

#include <cuda.h>
#include <cudaTypedefs.h>

#include "hh_internal.cuh"

namespace hh {

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

// the same wait with a caller-chosen poll budget (failure injection uses a short one)
__device__ __forceinline__ bool mbar_wait_parity_n(uint64_t *bar, uint32_t parity, long polls) {
    const uint32_t a = smem_u32(bar);
    for (long it = 0; it < polls; it++) {
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
// counts `bytes` of the current phase's expected transaction bytes as arrived (the failure
// injection's drain settles the bytes it added this way)
__device__ __forceinline__ void mbar_complete_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.complete_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Tensor copies (cp.async.bulk.tensor) need 128-byte aligned shared-memory addresses and a
// tensor map whose innermost coordinate here is always 0 (the re/im pair of a complex double).
__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, int c1, int c2, int c3, int c4,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store_5d(const CUtensorMap *map, int c1, int c2, int c3, int c4, const void *src) {
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4, %5}], [%6];" ::"l"(map),
                 "r"(0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(src))
                 : "memory");
}
// 4-D tensor copies over (re/im, x, j, plane) maps: one box at column x, row j, plane p
__device__ __forceinline__ void tma_tile_load(void *dst, const CUtensorMap *map, int x, int j, int p, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(0), "r"(x), "r"(j), "r"(p), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_tile_store(const CUtensorMap *map, int x, int j, int p, const void *src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];" ::"l"(map),
                 "r"(0), "r"(x), "r"(j), "r"(p), "r"(smem_u32(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 3-D tensor copies over (double, row, plane) maps: one box at double offset x (a multiple of 2,
// so that x * 8 bytes stays on a 16-byte boundary), row j, plane p
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int j, int p, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(j), "r"(p), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, int x, int j, int p, const void *src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(map),
                 "r"(x), "r"(j), "r"(p), "r"(smem_u32(src))
                 : "memory");
}

// A tiled tensor map of FLOAT64 values: dims[0] innermost (for complex data 2 = (re, im), or the
// doubles of a whole row), strides in bytes for dims[1..rank-1] (multiples of 16), box extents
// per dimension (<= 256).  swizzle128: 128-byte swizzle (box dims[0] * 8 must be 128 bytes; the
// 16-byte chunk c of the box's 128-byte row r lands at chunk c ^ (r % 8) of a 1024-byte aligned
// destination).
int encode_tensor_map(CUtensorMap *map, const void *base, int rank, const unsigned long long *dims,
                      const unsigned long long *strides, const unsigned *box, bool swizzle128 = false);

} // namespace hh

#endif
