// FP64 fused DFT-tile stencil kernel for 3D grids (plain form, DMMA).
//
// Tile 16 x 16 x 16 (index i = 256 z + 16 y + x); two x-adjacent real tiles
// packed as one complex tile (64 KiB).  Each DFT-16 is two radix-4 stages
// (j = 4a + b, frequency k1 + 4 k2 stored at position 4 k1 + k2).  A stage on 8
// four-point lines is one real-block product
//     [Re F X; Im F X] (8 x 8) = [[Re F, -Im F], [Im F, Re F]] (8 x 8) . [Xr; Xi] (8 x 8)
// i.e. two mma.sync.m8n8k4.f64 whose B fragments are exactly the (re, im)
// halves of one 16-byte shared-memory load; a lane-xor-16 shuffle regroups the
// real and imaginary outputs into complex values.
//
// Warp w owns z-plane w for the x and y stages and y-plane w for the z stages,
// so a tile pair needs three block barriers:
//   [x fwd, y fwd] | [z fwd, x spectrum^tau, z inv] | [y inv, x inv -> cropped store].
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
    double2 *w16 = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES + TW_BYTES);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    for (int i = tid; i < VOL; i += NT)
        spec[sw3(i)] = p.spec[i];
    if (tid < 16)
        w16[tid] = p.tables[tid];
    Consts c;
    {   // real-block DFT-4 entries: F4[k][a] = w16^(4 k a); row g < 4 -> Re out k1 = g, else Im out k1 = g - 4
        const int k1 = g & 3;
        const double2 f = p.tables[(4 * k1 * t) & 15];
        const bool re_row = g < 4;
        c.f0 = re_row ? f.x : f.y;   // multiplies Xr[a = t]
        c.f1 = re_row ? -f.y : f.x;  // multiplies Xi[a = t]
        c.i0 = re_row ? f.x : -f.y;  // conjugate
        c.i1 = re_row ? f.y : f.x;
    }
    __syncthreads();
    c.w16 = w16;

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
        if (tma_ok(p, it)) {
            if (!mbar_wait_bounded(bar, phase)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            phase ^= 1;
            for (int i = tid; i < VOL; i += NT)
                work[sw3(i)] = make_double2(stage_buf[i], it.has_b ? stage_buf[VOL + i] : 0.0);
        } else {
            fill_plain(work, p, it, tid, NT);
        }
        __syncthreads();
        if (tid == 0 && w + gridDim.x < p.nitems) {
            const Item nx_it = item_of(p, w + gridDim.x);
            if (tma_ok(p, nx_it))
                issue(nx_it);
        }
        compute_item(work, spec, c, p, it, warp, g, t);
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
