// FP64 fused DFT-tile stencil kernel for 1D grids (plain form, DMMA).
//
// Tile n = 4096 = 64 x 64 cells (tile-local index j = 64a + b), two tiles
// adjacent along x packed as one complex tile.  The 4096-point DFT is the
// four-step form: a DFT-64 over a for every b (each DFT-64 two radix-8
// mma.sync.m8n8k4.f64 stages), the 4096th-root twiddle w^(b*k1), then per k1
// a DFT-64 over b, the spectrum^tau multiply and the inverse DFT-64 over b,
// the conjugate twiddle, and the inverse DFT-64 back to a.  The interior
// u = 4096 - 2*halo cells are stored with coalesced writes.
//
// Replaces rfft_pfa_stencil_8_nwarp (src/1D/rfftstencil_pfa/rfft_8_pfa_fastcomplex.cu:17-340),
// which runs one 56-point prime-factor tile (8 x 7) per warp with a random
// 29/31-tap kernel standing in for 14/7/5 fused steps and atomics on overlap.
#include <cstring>

#include "ffs_dmma1d.cuh"

namespace ffst {
namespace dmma1d {

__global__ void __launch_bounds__(NT, 1) dmma1d_kernel(const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double *stage = reinterpret_cast<double *>(smem);
    double2 *work = reinterpret_cast<double2 *>(smem + STAGE_BYTES);
    double2 *spec = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES);
    double2 *t1 = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES);
    double2 *t2 = t1 + T1N;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES + TW_BYTES);
    uint64_t *cbar = bar + 1; // spectrum and twiddle tables

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    auto issue = [&](const Item &it) {
        const Seg sa = seg_of(p, it.lxa);
        const Seg sb = it.has_b ? seg_of(p, it.lxb) : Seg{0, 0, false};
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(bar, (uint32_t)((sa.hi - sa.lo + sb.hi - sb.lo) * sizeof(double)));
        if (sa.hi > sa.lo)
            bulk_load(stage + sa.lo, p.in + it.lxa + sa.lo, (uint32_t)((sa.hi - sa.lo) * sizeof(double)), bar);
        if (sb.hi > sb.lo)
            bulk_load(stage + TILE + sb.lo, p.in + it.lxb + sb.lo, (uint32_t)((sb.hi - sb.lo) * sizeof(double)),
                      bar);
    };
    uint32_t phase = 0;
    int64_t w = blockIdx.x;
    // the first pair and the constants are copied asynchronously: most launches run a
    // single wave, where a synchronous copy of the 79 KB of tables would sit in front
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(cbar, 1);
        fence_barrier_init();
        if (w < p.nitems) { // a CTA without a pair copies nothing (no copy may outlive it)
            const Item it = item_of(p, w);
            if (bulk_ok(p, it))
                issue(it);
            mbar_arrive_expect_tx(cbar, (uint32_t)(SPEC_BYTES + TW_BYTES));
            bulk_load(spec, p.spec, (uint32_t)SPEC_BYTES, cbar);
            bulk_load(t1, p.tables + 8 + 64, (uint32_t)TW_BYTES, cbar);
        }
    }
    const LaneConst c = lane_consts(p.tables, p.tables + 8, g, t);
    __syncthreads();
    bool consts_ready = false;

    for (; w < p.nitems; w += gridDim.x) {
        const Item it = item_of(p, w);
        // stage -> work, transposed: SMEM row b holds the line a = 0..63 of x[64a + b]
        if (bulk_ok(p, it)) {
            if (!mbar_wait_bounded(bar, phase)) {
                record_error(p.status, kDevTimeoutTma);
                if (!consts_ready)
                    mbar_wait_bounded(cbar, 0); // let the constants' copy land before leaving
                return;
            }
            phase ^= 1;
            const Seg sa = seg_of(p, it.lxa);
            const Seg sb = it.has_b ? seg_of(p, it.lxb) : Seg{0, 0, false};
            for (int i = tid; i < TILE; i += NT) {
                const int a = i >> 6, b = i & 63;
                const double re = staged(stage, p, it.lxa, sa, i);
                const double im = it.has_b ? staged(stage + TILE, p, it.lxb, sb, i) : 0.0;
                work[widx(b, a)] = make_double2(re, im);
            }
        } else {
            fill_plain(work, p, it, tid);
        }
        if (!consts_ready) {
            if (!mbar_wait_bounded(cbar, 0)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            consts_ready = true;
        }
        __syncthreads();
        if (tid == 0 && w + gridDim.x < p.nitems) {
            const Item nx_it = item_of(p, w + gridDim.x);
            if (bulk_ok(p, nx_it))
                issue(nx_it);
        }
        compute_item(work, spec, t1, t2, c, p, it, tid, NT, warp, NWARP, g, t);
        __syncthreads();
    }
}

} // namespace dmma1d

size_t dmma1d_smem_bytes() { return dmma1d::SMEM_BYTES; }
int dmma1d_tile() { return dmma1d::TILE; }

cudaError_t prepare_dmma1d()
{
    return cudaFuncSetAttribute(dmma1d::dmma1d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dmma1d::SMEM_BYTES);
}

cudaError_t launch_dmma1d(const TileWork &w, int grid, cudaStream_t s)
{
    dmma1d::dmma1d_kernel<<<grid, dmma1d::NT, dmma1d::SMEM_BYTES, s>>>(w);
    return cudaGetLastError();
}

} // namespace ffst
