// 2D FP64-DMMA fused tile: per-item device functions shared by the persistent
// 2D kernel (ffs_dmma2d.cu) and the batched multi-problem kernel (ffs_batch.cu).
#pragma once
#include "ffs_device.cuh"
#include "ffs_kernels.h"
#include "ffs_radix64.cuh"

namespace ffst {
namespace dmma2d {

using namespace r64;
constexpr int NT = 512;
constexpr int NWARP = NT / 32;
constexpr size_t STAGE_BYTES = 2ull * N * N * sizeof(double); // two dense TMA boxes
constexpr size_t WORK_BYTES = (size_t)N * N * sizeof(double2);
constexpr size_t SPEC_BYTES = (size_t)N * N * sizeof(double2);
constexpr size_t SMEM_BYTES = STAGE_BYTES + WORK_BYTES + SPEC_BYTES + 16;

struct Item {
    int64_t ty, txa;
    int64_t ly0, lxa, lxb;
    bool has_b;
};

__device__ __forceinline__ Item item_of(const TileWork &p, int64_t w)
{
    Item it;
    const int64_t pr = w % p.npx;
    it.ty = p.t0[1] + w / p.npx;
    it.txa = p.t0[0] + 2 * pr;
    it.has_b = (2 * pr + 1) < p.nt[0];
    it.ly0 = it.ty * p.useful - p.halo;
    it.lxa = it.txa * p.useful - p.halo;
    it.lxb = it.lxa + p.useful;
    return it;
}

__device__ __forceinline__ bool tma_ok(const TileWork &p, const Item &it)
{
    if (!p.use_tma)
        return false;
    if (!p.periodic)
        return true; // out-of-range reads are zeros, only used by discarded cells
    const bool yin = it.ly0 >= 0 && it.ly0 + N <= p.ny;
    const bool ain = it.lxa >= 0 && it.lxa + N <= p.nx;
    const bool bin = !it.has_b || (it.lxb >= 0 && it.lxb + N <= p.nx);
    return yin && ain && bin;
}

// Fill the complex work tile of item `it` with plain (L1-bypassing) loads; wraps
// periodically or reads zeros outside the grid.  Each of the NT threads issues all of
// its loads before its first store, so the memory latency is paid once per item.
__device__ __forceinline__ void fill_plain(double2 *work, const TileWork &p, const Item &it, int tid)
{
    constexpr int PER = N * N / NT;
    double re[PER], im[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        const int y = i >> 6, x = i & 63;
        int64_t gy = it.ly0 + y;
        const int64_t ga = it.lxa + x, gb = it.lxb + x;
        re[k] = 0.0;
        im[k] = 0.0;
        if (p.periodic) {
            gy = wrap_near(gy, p.ny);
            re[k] = __ldcg(p.in + gy * p.nx + wrap_near(ga, p.nx));
            if (it.has_b)
                im[k] = __ldcg(p.in + gy * p.nx + wrap_near(gb, p.nx));
        } else if (gy >= 0 && gy < p.ny) {
            if (ga >= 0 && ga < p.nx)
                re[k] = __ldcg(p.in + gy * p.nx + ga);
            if (it.has_b && gb >= 0 && gb < p.nx)
                im[k] = __ldcg(p.in + gy * p.nx + gb);
        }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        work[widx(i >> 6, i & 63)] = make_double2(re[k], im[k]);
    }
}

struct NoAction {
    __device__ __forceinline__ void operator()() const {}
};

struct BlockBarrier {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// Rows forward, columns (DFT, spectrum, inverse), rows inverse with cropped stores.
// `nwarp` warps (the whole CTA); ends before the caller's final barrier.
// The forward row pass reads `load(y, x)` (the work tile itself, or the TMA
// staging planes); `after_rows()` runs once every row has been read.
template <typename Bar = BlockBarrier, typename Load = WorkLoader, typename AfterRows = NoAction>
__device__ __forceinline__ void compute_item(double2 *work, const double2 *spec, const LaneConst &c, const TileWork &p,
                                             const Item &it, int warp, int nwarp, int g, int t, Bar bar = Bar(),
                                             Load load = Load{nullptr}, AfterRows after_rows = AfterRows())
{
#pragma unroll 1
    for (int y = warp; y < N; y += 2 * nwarp) { // two independent rows in flight
        row_forward(work, y, c, g, t, NoHook(), load);
        row_forward(work, y + nwarp, c, g, t, NoHook(), load);
    }
    bar();
    after_rows();
#pragma unroll 1
    for (int x = warp; x < N; x += 2 * nwarp) // two independent columns in flight
        column_pass2(work, spec, x, x + nwarp, c, g, t);
    bar();
#pragma unroll 1
    for (int y = warp; y < N; y += nwarp) {
        const int64_t gy = it.ly0 + y;
        if (y < p.halo || y >= p.halo + p.useful || gy < p.vlo[1] || gy >= p.vhi[1])
            continue;
        double ore[2], oim[2];
        row_inverse(work, y, c, g, t, ore, oim);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int x = g + 8 * (2 * t + e);
            if (x < p.halo || x >= p.halo + p.useful)
                continue;
            const int64_t ga = it.lxa + x, gb = it.lxb + x;
            if (ga >= p.vlo[0] && ga < p.vhi[0])
                p.out[gy * p.nx + ga] = ore[e];
            if (it.has_b && gb >= p.vlo[0] && gb < p.vhi[0])
                p.out[gy * p.nx + gb] = oim[e];
        }
    }
}

} // namespace dmma2d
} // namespace ffst
