// Direct FP64 stepping of fixed-boundary band boxes: device function shared by
// the band kernel (ffs_band.cu) and the batched kernel.
#pragma once
#include "ffs_device.cuh"
#include "ffs_kernels.h"

namespace ffst {
namespace band {

// Direct stepping of band box `box` with `nthreads` threads; `smem` holds
// band_smem_bytes(max_vol, ntaps) bytes.
template <int DIM>
__device__ __forceinline__ void process_box(const BandWork &p, int box, unsigned char *smem, int nthreads)
{
    const BandBox bx = p.boxes[box];
    const int tau = p.tau, r = p.r;
    const int64_t rt = (int64_t)p.r * p.tau;

    int64_t L[3];
    int ext[3];
    int vol = 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d < DIM) {
            L[d] = bx.lo[d] - rt < 0 ? 0 : bx.lo[d] - rt;
            const int64_t hi = bx.lo[d] + bx.ext[d] + rt;
            ext[d] = (int)((hi > p.n[d] ? p.n[d] : hi) - L[d]);
        } else {
            L[d] = 0;
            ext[d] = 1;
        }
        vol *= ext[d];
    }
    if (vol > p.max_vol) { // the host sizes shared memory for the largest box; refuse otherwise
        if (threadIdx.x == 0)
            record_error(p.status, kDevBadConfig);
        return;
    }
    // staged region is dense with the box's own loaded extents as strides
    const int ex = ext[0], exy = ext[0] * ext[1];
    const int64_t plane = (p.max_vol + 1) & ~(int64_t)1; // keeps the int4 taps 16-byte aligned
    double *buf0 = reinterpret_cast<double *>(smem);
    double *buf1 = buf0 + plane;
    double *wts = buf1 + plane;
    int *toff = reinterpret_cast<int *>(wts + ((p.ntaps + 1) & ~1));
    for (int i = threadIdx.x; i < p.ntaps; i += nthreads) {
        const int4 tp = p.taps[i];
        wts[i] = p.weights[tp.w];
        toff[i] = tp.z * exy + tp.y * ex + tp.x;
    }
    for (int i = threadIdx.x; i < vol; i += nthreads) {
        const int z = DIM == 3 ? i / exy : 0;
        const int rem = i - z * exy;
        const int y = DIM >= 2 ? rem / ex : 0;
        const int x = rem - y * ex;
        buf0[i] = __ldcg(p.in + ((L[2] + z) * p.n[1] + (L[1] + y)) * p.n[0] + (L[0] + x));
    }
    __syncthreads();
    // per-dim bounds of cells that are updated: not in the ring, all taps inside the staged region
    int ulo[3], uhi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d < DIM) {
            const int64_t glo = r, ghi = p.n[d] - r; // exclusive
            int lo = r, hi = ext[d] - r;
            lo = (int)max((int64_t)lo, glo - L[d]);
            hi = (int)min((int64_t)hi, ghi - L[d]);
            ulo[d] = lo;
            uhi[d] = hi;
        } else {
            ulo[d] = 0;
            uhi[d] = 1;
        }
    }
    double *src = buf0, *dst = buf1;
    for (int s = 0; s < tau; ++s) {
        for (int i = threadIdx.x; i < vol; i += nthreads) {
            const int z = DIM == 3 ? i / exy : 0;
            const int rem = i - z * exy;
            const int y = DIM >= 2 ? rem / ex : 0;
            const int x = rem - y * ex;
            double v = src[i];
            const bool upd = x >= ulo[0] && x < uhi[0] && y >= ulo[1] && y < uhi[1] && z >= ulo[2] && z < uhi[2];
            if (upd) {
                double acc = 0.0;
                for (int k = 0; k < p.ntaps; ++k)
                    acc += wts[k] * src[i + toff[k]];
                v = acc;
            }
            dst[i] = v; // ring cells keep their value; cells too close to a cut edge are never read
        }
        __syncthreads();
        double *tmp = src;
        src = dst;
        dst = tmp;
    }
    const int bex = bx.ext[0], bexy = bx.ext[0] * bx.ext[1];
    const int bvol = bexy * bx.ext[2];
    for (int i = threadIdx.x; i < bvol; i += nthreads) {
        const int z = DIM == 3 ? i / bexy : 0;
        const int rem = i - z * bexy;
        const int y = DIM >= 2 ? rem / bex : 0;
        const int x = rem - y * bex;
        const int64_t gx = bx.lo[0] + x, gy = bx.lo[1] + y, gz = bx.lo[2] + z;
        const int li = (int)(((gz - L[2]) * ext[1] + (gy - L[1])) * ext[0] + (gx - L[0]));
        p.out[(gz * p.n[1] + gy) * p.n[0] + gx] = src[li];
    }
}

} // namespace band
} // namespace ffst
