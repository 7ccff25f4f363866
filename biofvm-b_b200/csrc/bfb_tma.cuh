// bfb_tma.cuh -- device helpers for the TMA kernels: mbarriers with bounded
// waits, 2-D/3-D tensor copies and 1-D bulk copies between this GPU's global
// memory and the issuing CTA's shared memory (no multicast).
#pragma once
#include <cuda.h>

#include "bfb_line.cuh"

namespace bfb {

constexpr int kWaitLimit = 1 << 22;  // try_wait polls before a wait is declared lost

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned phase) {
    for (int i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}
__device__ __forceinline__ void tma_load(unsigned dst, const CUtensorMap *map, int c0, int c1, int c2, int rank,
                                         unsigned bar) {
    const unsigned long long m = reinterpret_cast<unsigned long long>(map);
    if (rank == 2)
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
                "r"(dst),
            "l"(m), "r"(c0), "r"(c1), "r"(bar)
            : "memory");
    else
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
            "[%5];\n" ::"r"(dst),
            "l"(m), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
            : "memory");
}
__device__ __forceinline__ void tma_store(const CUtensorMap *map, int c0, int c1, int c2, int rank, unsigned src) {
    const unsigned long long m = reinterpret_cast<unsigned long long>(map);
    if (rank == 2)
        asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(m), "r"(c0),
                     "r"(c1), "r"(src)
                     : "memory");
    else
        asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(m),
                     "r"(c0), "r"(c1), "r"(c2), "r"(src)
                     : "memory");
}
__device__ __forceinline__ void bulk_load(unsigned dst, const void *src, unsigned bytes, unsigned bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ void bulk_store(void *dst, unsigned src, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst), "r"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// Lines of the narrow FP64 strided tile: 22 x 8 B rows are whole 16-byte
// vectors, and at 256 rows five such tiles fit an SM where three of 32 do.
constexpr int kNarrowLinesF64 = 22;

// Rows per TMA box (one row group) of a strided tile of `lines` lines of n
// rows in `chunks` groups: ceil(n / chunks), rounded up so that every group's
// shared-memory start (a multiple of crow*lines*elem bytes past the 128-byte
// aligned tile) is 128-byte aligned, as tensor copies require.
__host__ __device__ inline int strided_box_rows(int n, int chunks, int lines, int elem) {
    int m = 128;  // 128 / gcd(128, lines*elem)
    for (int v = lines * elem; v % 2 == 0 && m > 1; v /= 2) m /= 2;
    const int crow = (n + chunks - 1) / chunks;
    return (crow + m - 1) / m * m;
}

// Bytes of one warp's region in a strided TMA CTA: kChunks mbarriers padded to
// 128 B, then the tile of nch*crow rows x `lines` lines (the last box may
// reach past row n; TMA zero-fills those rows and the store clips them).
__host__ __device__ inline size_t strided_tma_warp_bytes(int n, int crow, int elem, int lines) {
    const int nch = (n + crow - 1) / crow;
    return 128 + (size_t)nch * crow * lines * elem;
}

}  // namespace bfb
