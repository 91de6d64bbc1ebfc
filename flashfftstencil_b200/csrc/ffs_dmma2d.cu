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

#include "ffs_dmma2d.cuh"

namespace ffst {
namespace dmma2d {

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
        const bool staged = tma_ok(p, it);
        const int64_t wn = w + gridDim.x;
        // the next pair's TMA may only overwrite the staging planes once every row was read
        auto prefetch = [&]() {
            if (tid == 0 && wn < p.nitems) {
                const Item nx_it = item_of(p, wn);
                if (tma_ok(p, nx_it))
                    issue(nx_it);
            }
        };
        if (staged) {
            if (!mbar_wait_bounded(bar, phase)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            phase ^= 1;
            compute_item(work, spec, c, p, it, warp, NWARP, g, t, BlockBarrier(), StageLoader{stage}, prefetch);
        } else {
            fill_plain(work, p, it, tid);
            __syncthreads();
            compute_item(work, spec, c, p, it, warp, NWARP, g, t, BlockBarrier(), WorkLoader{nullptr}, prefetch);
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
