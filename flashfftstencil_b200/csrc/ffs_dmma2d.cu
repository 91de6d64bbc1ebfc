// FP64 fused DFT-tile stencil kernel for 2D grids (plain form, DMMA).
//
// One persistent CTA per SM walks tile pairs.  Per pair:
//   1. TMA (cp.async.bulk.tensor.2d, no multicast) stages two 64x64 FP64 halo
//      tiles of the natural row-major grid into shared memory; out-of-range
//      coordinates read zeros.  The next pair is prefetched while this one computes.
//   2. The two real tiles are interleaved into one complex tile (re = left tile,
//      im = right tile) in a swizzled layout that keeps every fragment access
//      below conflict-free for 128-bit shared loads/stores.
//   3. Forward 2D DFT-64x64: each 64-point DFT is two radix-8 stages, each an
//      8x8x8 complex product on mma.sync.m8n8k4.f64, with the 64th-root twiddle
//      applied in registers between them.  The second stage takes its A operand
//      straight from the first stage's accumulators by permuting the contraction
//      order of the DFT-8 matrix (the fragment-reuse idea of the reference,
//      src/2D/rfft_2d/2d_rfft_2.cu:113-116 with src/2D/create_fft_pfa_plan.cu:29).
//   4. Pointwise multiply by spectrum^tau / 64^2 (FP64, prepared on the host).
//   5. Inverse DFT, crop of the halo, direct store of the u x u interior.
// This replaces rfft_2d_8_nwarp (src/2D/rfft_2d/2d_rfft_1_async.cu:17-364): the
// reference uses 8x8 tiles, one step per launch and atomic overlap-add; here a
// tile carries tau fused steps and every output cell is written exactly once.
#include <cstring>

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

__device__ __forceinline__ int64_t wrapi(int64_t i, int64_t n)
{
    i %= n;
    return i < 0 ? i + n : i;
}

__global__ void __launch_bounds__(NT, 1) dmma2d_kernel(const __grid_constant__ CUtensorMap tmap, const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double *stage = reinterpret_cast<double *>(smem);
    double2 *work = reinterpret_cast<double2 *>(smem + STAGE_BYTES);
    double2 *spec = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    for (int i = tid; i < N * N; i += NT)
        spec[i] = p.spec[i];
    LaneConst c;
    {
        const double2 *f8 = p.tables, *w64 = p.tables + 8;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const double2 fa = f8[(g * (t + 4 * j)) & 7];
            const double2 fp = f8[((2 * t + j) * g) & 7];
            const double2 tw = w64[(g * (2 * t + j)) & 63];
            c.fa_re[j] = fa.x; c.fa_im[j] = fa.y; c.fa_nim[j] = -fa.y;
            c.fp_re[j] = fp.x; c.fp_im[j] = fp.y; c.fp_nim[j] = -fp.y;
            c.tw_re[j] = tw.x; c.tw_im[j] = tw.y;
        }
    }
    __syncthreads();

    auto issue = [&](const Item &it) {
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(bar, (uint32_t)STAGE_BYTES);
        tma_load_2d(stage, &tmap, bar, (int)it.lxa, (int)it.ly0);
        tma_load_2d(stage + N * N, &tmap, bar, (int)it.lxb, (int)it.ly0);
    };

    uint32_t phase = 0;
    int64_t w = blockIdx.x;
    if (tid == 0 && w < p.nitems) {
        const Item it = item_of(p, w);
        if (tma_ok(p, it))
            issue(it);
    }
    for (; w < p.nitems; w += gridDim.x) {
        const Item it = item_of(p, w);
        if (tma_ok(p, it)) {
            if (!mbar_wait_bounded(bar, phase)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            phase ^= 1;
            for (int i = tid; i < N * N; i += NT) {
                const int y = i >> 6, x = i & 63;
                work[widx(y, x)] = make_double2(stage[i], stage[N * N + i]);
            }
        } else {
            for (int i = tid; i < N * N; i += NT) {
                const int y = i >> 6, x = i & 63;
                int64_t gy = it.ly0 + y, ga = it.lxa + x, gb = it.lxb + x;
                double re = 0.0, im = 0.0;
                if (p.periodic) {
                    gy = wrapi(gy, p.ny);
                    re = p.in[gy * p.nx + wrapi(ga, p.nx)];
                    if (it.has_b)
                        im = p.in[gy * p.nx + wrapi(gb, p.nx)];
                } else if (gy >= 0 && gy < p.ny) {
                    if (ga >= 0 && ga < p.nx)
                        re = p.in[gy * p.nx + ga];
                    if (it.has_b && gb >= 0 && gb < p.nx)
                        im = p.in[gy * p.nx + gb];
                }
                work[widx(y, x)] = make_double2(re, im);
            }
        }
        __syncthreads();
        if (tid == 0 && w + gridDim.x < p.nitems) {
            const Item nx_it = item_of(p, w + gridDim.x);
            if (tma_ok(p, nx_it))
                issue(nx_it);
        }
        // forward DFT along x, every row
#pragma unroll 1
        for (int k = 0; k < N / NWARP; k += 2) {
            row_forward(work, warp + NWARP * k, c, g, t);
            row_forward(work, warp + NWARP * (k + 1), c, g, t);
        }
        __syncthreads();
#pragma unroll 1
        for (int k = 0; k < N / NWARP; ++k)
            column_pass(work, spec, warp + NWARP * k, c, g, t);
        __syncthreads();
        // inverse DFT along x and cropped store of the interior rows
#pragma unroll 1
        for (int k = 0; k < N / NWARP; ++k) {
            const int y = warp + NWARP * k;
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
        __syncthreads();
    }
}

} // namespace dmma2d

size_t dmma2d_smem_bytes() { return dmma2d::SMEM_BYTES; }
int dmma2d_tile() { return dmma2d::N; }

cudaError_t prepare_dmma2d()
{
    return cudaFuncSetAttribute(dmma2d::dmma2d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dmma2d::SMEM_BYTES);
}

cudaError_t launch_dmma2d(const CUtensorMap *tmap, const TileWork &w, int grid, cudaStream_t s)
{
    CUtensorMap dummy;
    if (!tmap) {
        memset(&dummy, 0, sizeof(dummy));
        tmap = &dummy;
    }
    dmma2d::dmma2d_kernel<<<grid, dmma2d::NT, dmma2d::SMEM_BYTES, s>>>(*tmap, w);
    return cudaGetLastError();
}

} // namespace ffst
