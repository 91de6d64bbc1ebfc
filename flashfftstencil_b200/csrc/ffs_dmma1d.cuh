// 1D FP64-DMMA fused tile (4096-point four-step): per-item device functions
// shared by the persistent 1D kernel (ffs_dmma1d.cu) and the batched kernel.
#pragma once
#include "ffs_device.cuh"
#include "ffs_kernels.h"
#include "ffs_radix64.cuh"

namespace ffst {
namespace dmma1d {

using namespace r64;
constexpr int TILE = N * N; // 4096
constexpr int NT = 512;
constexpr int NWARP = NT / 32;
constexpr int T1N = 448; // w4096^m, m <= 63*7
constexpr int T2N = 512; // w512^m
constexpr size_t STAGE_BYTES = 2ull * TILE * sizeof(double);
constexpr size_t WORK_BYTES = (size_t)TILE * sizeof(double2);
constexpr size_t SPEC_BYTES = (size_t)TILE * sizeof(double2);
constexpr size_t TW_BYTES = (size_t)(T1N + T2N) * sizeof(double2);
constexpr size_t SMEM_BYTES = STAGE_BYTES + WORK_BYTES + SPEC_BYTES + TW_BYTES + 32;

// Natural-order (a, b) slot used for the cropped write-back; conflict-free for
// the per-lane writes (a = g + 16t + 8e, fixed b) and for row-contiguous reads.
__device__ __forceinline__ int nat_idx(int a, int b) { return a * N + (b ^ ((a & 1) | ((a >> 3) & 6))); }

struct Item {
    int64_t lxa, lxb;
    bool has_b;
};

__device__ __forceinline__ Item item_of(const TileWork &p, int64_t w)
{
    Item it;
    const int64_t txa = p.t0[0] + 2 * w;
    it.has_b = (2 * w + 1) < p.nt[0];
    it.lxa = txa * p.useful - p.halo;
    it.lxb = it.lxa + p.useful;
    return it;
}

// Bulk copies stage the pair: whole tiles, or with a fixed boundary the part of a tile
// inside the grid (the rest reads zero, which only discarded cells see).  A periodic
// tile that crosses an end wraps and takes plain loads instead.
__device__ __forceinline__ bool bulk_ok(const TileWork &p, const Item &it)
{
    if (!p.use_tma)
        return false;
    if (!p.periodic)
        return true;
    const bool ain = it.lxa >= 0 && it.lxa + TILE <= p.nx;
    const bool bin = !it.has_b || (it.lxb >= 0 && it.lxb + TILE <= p.nx);
    return ain && bin;
}

// Part of the tile starting at lx that the bulk copy stages, in tile coordinates:
// [lo, hi) has an even length (16-byte copies; lx and lo are even), and `tail` marks
// one more in-grid element at hi, loaded plainly.
struct Seg {
    int lo, hi;
    bool tail;
};

__device__ __forceinline__ Seg seg_of(const TileWork &p, int64_t lx)
{
    const int64_t a = lx > 0 ? lx : 0, b = lx + TILE < p.nx ? lx + TILE : p.nx;
    const int64_t n = b > a ? b - a : 0;
    Seg s;
    s.lo = (int)(a - lx);
    s.hi = s.lo + (int)(n & ~1ll);
    s.tail = (n & 1) != 0;
    return s;
}

__device__ __forceinline__ double staged(const double *stage, const TileWork &p, int64_t lx, const Seg &s, int i)
{
    if (i >= s.lo && i < s.hi)
        return stage[i];
    return (s.tail && i == s.hi) ? __ldcg(p.in + lx + i) : 0.0;
}

// w4096^(b*k1) with k1 = g + 8*c2: T1[b*g] * T2[b*c2]
__device__ __forceinline__ void tw4096(const double2 *t1, const double2 *t2, int b, int g, int c2, double &wr,
                                       double &wi)
{
    const double2 x = t1[b * g];
    const double2 y = t2[(b * c2) & (T2N - 1)];
    wr = x.x * y.x - x.y * y.y;
    wi = x.x * y.y + x.y * y.x;
}

struct FwdTwiddle {
    const double2 *t1, *t2;
    int g, t;
    __device__ __forceinline__ void operator()(int b, double re[2], double im[2]) const
    {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            double wr, wi;
            tw4096(t1, t2, b, g, 2 * t + e, wr, wi);
            cmul(re[e], im[e], wr, wi);
        }
    }
};

// Plain (L1-bypassing) loads of item `it`, transposed into the work tile.  Each of the
// NT threads issues all of its loads before its first store.
__device__ __forceinline__ void fill_plain(double2 *work, const TileWork &p, const Item &it, int tid)
{
    constexpr int PER = TILE / NT;
    double re[PER], im[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        const int64_t ga = it.lxa + i, gb = it.lxb + i;
        re[k] = 0.0;
        im[k] = 0.0;
        if (p.periodic) {
            re[k] = __ldcg(p.in + wrap_near(ga, p.nx));
            if (it.has_b)
                im[k] = __ldcg(p.in + wrap_near(gb, p.nx));
        } else {
            if (ga >= 0 && ga < p.nx)
                re[k] = __ldcg(p.in + ga);
            if (it.has_b && gb >= 0 && gb < p.nx)
                im[k] = __ldcg(p.in + gb);
        }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        work[widx(i & 63, i >> 6)] = make_double2(re[k], im[k]);
    }
}

// Four-step DFT-4096, spectrum, inverse and the cropped store of item `it`.
__device__ __forceinline__ void compute_item(double2 *work, const double2 *spec, const double2 *t1,
                                             const double2 *t2, const LaneConst &c, const TileWork &p,
                                             const Item &it, int tid, int nthreads, int warp, int nwarp, int g,
                                             int t)
{
        const FwdTwiddle fwd{t1, t2, g, t};
#pragma unroll 1
        for (int b = warp; b < N; b += 2 * nwarp) { // two independent rows in flight
            row_forward(work, b, c, g, t, fwd);
            row_forward(work, b + nwarp, c, g, t, fwd);
        }
        __syncthreads();
#pragma unroll 1
        for (int x = warp; x < N; x += 2 * nwarp) // two independent columns in flight
            column_pass2(work, spec, x, x + nwarp, c, g, t);
        __syncthreads();
        // conj twiddle and inverse DFT-64 over k1 -> a; every row is loaded before
        // the natural-order result overwrites the same buffer
        constexpr int MAXR = N / 16; // rows per warp with at least 16 warps
        double bre[MAXR][2], bim[MAXR][2];
#pragma unroll
        for (int k = 0; k < MAXR; ++k) {
            const int b = warp + nwarp * k;
            if (b >= N)
                break;
            row_inverse_load(work, b, g, t, bre[k], bim[k]);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                double wr, wi;
                tw4096(t1, t2, b, g, t + 4 * j, wr, wi);
                cmul(bre[k][j], bim[k][j], wr, -wi);
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < MAXR; ++k) {
            const int b = warp + nwarp * k;
            if (b >= N)
                break;
            double ore[2], oim[2];
            row_inverse_compute(c, bre[k], bim[k], ore, oim);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int a = g + 8 * (2 * t + e);
                work[nat_idx(a, b)] = make_double2(ore[e], oim[e]);
            }
        }
        __syncthreads();
        for (int i = tid; i < TILE; i += nthreads) {
            if (i < p.halo || i >= p.halo + p.useful)
                continue;
            const double2 v = work[nat_idx(i >> 6, i & 63)];
            const int64_t ga = it.lxa + i, gb = it.lxb + i;
            if (ga >= p.vlo[0] && ga < p.vhi[0])
                p.out[ga] = v.x;
            if (it.has_b && gb >= p.vlo[0] && gb < p.vhi[0])
                p.out[gb] = v.y;
        }
}

} // namespace dmma1d
} // namespace ffst
