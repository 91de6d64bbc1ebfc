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

__global__ void __launch_bounds__(NT) band_kernel(const BandWork p)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const BandBox bx = p.boxes[blockIdx.x];
    const int tau = p.tau, r = p.r, rt = p.r * p.tau;

    int64_t L[3], R[3];
    int ext[3];
    int64_t vol = 1;
    for (int d = 0; d < 3; ++d) {
        if (d < p.dim) {
            L[d] = bx.lo[d] - rt < 0 ? 0 : bx.lo[d] - rt;
            const int64_t hi = bx.lo[d] + bx.ext[d] + rt;
            R[d] = hi > p.n[d] ? p.n[d] : hi;
        } else {
            L[d] = 0;
            R[d] = 1;
        }
        ext[d] = (int)(R[d] - L[d]);
        vol *= ext[d];
    }
    if (vol > p.max_vol) { // the host sizes shared memory for the largest box; refuse otherwise
        if (threadIdx.x == 0)
            record_error(p.status, kDevBadConfig);
        return;
    }
    // staged region is dense with the box's own loaded extents as strides
    const int cap_x = ext[0], cap_y = ext[1];
    const int64_t plane = (p.max_vol + 1) & ~(int64_t)1; // keeps the int4 taps 16-byte aligned
    double *buf0 = reinterpret_cast<double *>(smem);
    double *buf1 = buf0 + plane;
    double *wts = buf1 + plane;
    int4 *taps = reinterpret_cast<int4 *>(wts + ((p.ntaps + 1) & ~1));
    for (int i = threadIdx.x; i < p.ntaps; i += NT) {
        taps[i] = p.taps[i];
        wts[i] = p.weights[p.taps[i].w];
    }
    for (int64_t i = threadIdx.x; i < vol; i += NT) {
        const int x = (int)(i % ext[0]);
        const int y = (int)((i / ext[0]) % ext[1]);
        const int z = (int)(i / ((int64_t)ext[0] * ext[1]));
        const int64_t g = ((L[2] + z) * p.n[1] + (L[1] + y)) * p.n[0] + (L[0] + x);
        buf0[((int64_t)z * cap_y + y) * cap_x + x] = p.in[g];
    }
    __syncthreads();
    double *src = buf0, *dst = buf1;
    for (int s = 0; s < tau; ++s) {
        for (int64_t i = threadIdx.x; i < vol; i += NT) {
            const int c[3] = {(int)(i % ext[0]), (int)((i / ext[0]) % ext[1]),
                              (int)(i / ((int64_t)ext[0] * ext[1]))};
            const int64_t li = ((int64_t)c[2] * cap_y + c[1]) * cap_x + c[0];
            bool ring = false, inside = true;
            for (int d = 0; d < p.dim; ++d) {
                const int64_t gc = L[d] + c[d];
                ring |= (gc < r) || (gc >= p.n[d] - r);
                inside &= (c[d] >= r) && (c[d] + r < ext[d]);
            }
            double v = src[li];
            if (!ring && inside) {
                double acc = 0.0;
                for (int k = 0; k < p.ntaps; ++k) {
                    const int4 tp = taps[k];
                    acc += wts[k] * src[li + ((int64_t)tp.z * cap_y + tp.y) * cap_x + tp.x];
                }
                v = acc;
            }
            dst[li] = v; // ring cells keep their value; cells too close to a cut edge are never read
        }
        __syncthreads();
        double *tmp = src;
        src = dst;
        dst = tmp;
    }
    const int64_t bvol = (int64_t)bx.ext[0] * bx.ext[1] * bx.ext[2];
    for (int64_t i = threadIdx.x; i < bvol; i += NT) {
        const int x = (int)(i % bx.ext[0]);
        const int y = (int)((i / bx.ext[0]) % bx.ext[1]);
        const int z = (int)(i / ((int64_t)bx.ext[0] * bx.ext[1]));
        const int64_t gx = bx.lo[0] + x, gy = bx.lo[1] + y, gz = bx.lo[2] + z;
        const int64_t li = ((gz - L[2]) * cap_y + (gy - L[1])) * cap_x + (gx - L[0]);
        p.out[(gz * p.n[1] + gy) * p.n[0] + gx] = src[li];
    }
}

} // namespace band

cudaError_t prepare_band(size_t max_smem)
{
    return cudaFuncSetAttribute(band::band_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
}

cudaError_t launch_band(const BandWork &w, size_t smem_bytes, cudaStream_t s)
{
    if (w.nboxes <= 0)
        return cudaSuccess;
    band::band_kernel<<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    return cudaGetLastError();
}

size_t band_smem_bytes(int64_t max_vol, int ntaps)
{
    return 2 * (size_t)((max_vol + 1) & ~(int64_t)1) * sizeof(double) + ((ntaps + 1) & ~1) * sizeof(double) + ntaps * sizeof(int4);
}

} // namespace ffst
