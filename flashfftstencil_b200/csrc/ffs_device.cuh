// Device-side helpers shared by the sm_100a kernels: FP64 DMMA, mbarrier,
// TMA (cp.async.bulk.tensor / cp.async.bulk) and bounded waits.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ffs_kernels.h"

namespace ffst {

// i mod n for a tile coordinate, which lies within a few periods of [0, n): a few
// conditional steps instead of a 64-bit division (emulated, and it was the bulk of
// the periodic plain-load fills).
__device__ __forceinline__ int64_t wrap_near(int64_t i, int64_t n)
{
    while (i < 0)
        i += n;
    while (i >= n)
        i -= n;
    return i;
}

// Spin limit for every mbarrier wait: ~2^26 polls is several seconds, far above
// any legitimate wait; on expiry the kernel records FFS device error and returns.
constexpr uint32_t kSpinLimit = 1u << 26;

__device__ __forceinline__ void record_error(int *status, int code)
{
    if (status)
        atomicCAS(status, 0, code);
}

// D(8x8, f64) += A(8x4, row) * B(4x8, col).  Fragment layout (PTX ISA,
// mma.m8n8k4 .f64): A: lane holds A[lane>>2][lane&3]; B: B[lane&3][lane>>2];
// C/D: D[lane>>2][2*(lane&3) + {0,1}].
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: returns false (and leaves the barrier alone) after kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

// 2D tiled TMA load global -> shared (no multicast), completion on `bar`.
__device__ __forceinline__ void tma_load_2d(void *smem_dst, const void *tmap, uint64_t *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];\n" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// 3D tiled TMA load (x fastest).
__device__ __forceinline__ void tma_load_3d(void *smem_dst, const void *tmap, uint64_t *bar, int x, int y,
                                            int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];\n" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Untiled bulk copy global -> shared; both addresses 16-B aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_load(void *smem_dst, const void *gsrc, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(smem_dst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

struct cplx {
    double re, im;
};

__device__ __forceinline__ void cmul(double &re, double &im, double wr, double wi)
{
    double r = re * wr - im * wi;
    double i = re * wi + im * wr;
    re = r;
    im = i;
}

} // namespace ffst
