// FP64 fused DFT-tile stencil kernel for 3D grids (plain form, DMMA).
//
// Tile 16 x 16 x 16 (index e = 256 z + 16 y + x); two x-adjacent real tiles
// packed as one complex tile (64 KiB).  Each DFT-16 is one register pass of two
// radix-4 real-block DMMA stages per pair of lines (ffs_dmma3d.cuh).  The next
// pair is staged by two 3D TMA loads (128-byte swizzle), which the first pass
// reads directly; periodic edge pairs and unaligned grids use plain loads.
// Replaces rfft_3d_8_nwarp (src/3D/rfft_3d/3d_rfft_N.cu:16-303), which handles one
// 8^3 tile pair per warp, one step per launch, with atomics on the overlap.
#include <cstring>

#include "ffs_dmma3d.cuh"

namespace ffst {
namespace dmma3d {

__global__ void __launch_bounds__(NT, 1) dmma3d_kernel(const __grid_constant__ CUtensorMap tmap, const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double *stage_buf = reinterpret_cast<double *>(smem);
    double2 *work = reinterpret_cast<double2 *>(smem + STAGE_BYTES);
    double2 *spec = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    for (int i = tid; i < VOL; i += NT)
        spec[sw3(i)] = p.spec[i];
    const Consts c = make_consts(p.tables, g, t);
    __syncthreads();

    auto issue = [&](const Item &it) {
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(bar, (uint32_t)STAGE_BYTES);
        tma_load_3d(stage_buf, &tmap, bar, (int)it.lx, (int)it.ly, (int)it.lz);
        tma_load_3d(stage_buf + VOL, &tmap, bar, (int)it.lxb, (int)it.ly, (int)it.lz);
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
        // once the staged input is consumed, thread 0 starts the next pair's TMA loads
        auto next = [&]() {
            if (tid == 0 && w + gridDim.x < p.nitems) {
                const Item nx_it = item_of(p, w + gridDim.x);
                if (tma_ok(p, nx_it))
                    issue(nx_it);
            }
        };
        if (tma_ok(p, it)) {
            if (!mbar_wait_bounded(bar, phase)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            phase ^= 1;
            compute_item<kFromStage>(work, stage_buf, spec, c, p, it, warp, g, t, next);
        } else {
            fill_plain(work, p, it, tid);
            __syncthreads();
            compute_item<kFromWork>(work, stage_buf, spec, c, p, it, warp, g, t, next);
        }
        __syncthreads();
    }
}

} // namespace dmma3d

size_t dmma3d_smem_bytes() { return dmma3d::SMEM_BYTES; }
int dmma3d_tile() { return dmma3d::N; }

cudaError_t prepare_dmma3d()
{
    return cudaFuncSetAttribute(dmma3d::dmma3d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dmma3d::SMEM_BYTES);
}

cudaError_t launch_dmma3d(const CUtensorMap *tmap, const TileWork &w, int grid, cudaStream_t s)
{
    CUtensorMap dummy;
    if (!tmap) {
        memset(&dummy, 0, sizeof(dummy));
        tmap = &dummy;
    }
    dmma3d::dmma3d_kernel<<<grid, dmma3d::NT, dmma3d::SMEM_BYTES, s>>>(*tmap, w);
    return cudaGetLastError();
}

} // namespace ffst
