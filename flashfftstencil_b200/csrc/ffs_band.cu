// Direct FP64 time stepping for the cells a fused DFT tile cannot produce
// exactly under a fixed boundary.
//
// With the ring/shell of width r held at its initial value, tau fused steps are
// a pure convolution only for cells at least r*tau away from every face.  The
// cells of the band closer than that (ring included) are computed here: each
// CTA owns one box of band cells, stages the box plus an r*tau halo (clipped to
// the domain) in shared memory, applies the stencil tau times with the ring
// held, and writes the box.  The reference has no fixed boundary (its wrap is
// periodic, src/2D/check_correct.hpp:53-61), so this has no counterpart there;
// it follows the oracle's update rule exactly.
#include "ffs_device.cuh"
#include "ffs_kernels.h"

namespace ffst {
namespace band {

constexpr int NT = 256;

template <int DIM>
__global__ void __launch_bounds__(NT) band_kernel(const BandWork p)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const BandBox bx = p.boxes[blockIdx.x];
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
    for (int i = threadIdx.x; i < p.ntaps; i += NT) {
        const int4 tp = p.taps[i];
        wts[i] = p.weights[tp.w];
        toff[i] = tp.z * exy + tp.y * ex + tp.x;
    }
    for (int i = threadIdx.x; i < vol; i += NT) {
        const int z = DIM == 3 ? i / exy : 0;
        const int rem = i - z * exy;
        const int y = DIM >= 2 ? rem / ex : 0;
        const int x = rem - y * ex;
        buf0[i] = p.in[((L[2] + z) * p.n[1] + (L[1] + y)) * p.n[0] + (L[0] + x)];
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
        for (int i = threadIdx.x; i < vol; i += NT) {
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
    for (int i = threadIdx.x; i < bvol; i += NT) {
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

cudaError_t prepare_band(size_t max_smem)
{
    cudaError_t e = cudaFuncSetAttribute(band::band_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)max_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(band::band_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(band::band_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    return e;
}

cudaError_t launch_band(const BandWork &w, size_t smem_bytes, cudaStream_t s)
{
    if (w.nboxes <= 0)
        return cudaSuccess;
    if (w.dim == 1)
        band::band_kernel<1><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else if (w.dim == 2)
        band::band_kernel<2><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else
        band::band_kernel<3><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    return cudaGetLastError();
}

size_t band_smem_bytes(int64_t max_vol, int ntaps)
{
    return 2 * (size_t)((max_vol + 1) & ~(int64_t)1) * sizeof(double) + ((ntaps + 1) & ~1) * sizeof(double) +
           ntaps * sizeof(int);
}

} // namespace ffst
