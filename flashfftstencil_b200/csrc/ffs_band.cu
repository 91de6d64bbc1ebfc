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
#include "ffs_band.cuh"

namespace ffst {
namespace band {

constexpr int NT = 256;

template <int DIM, int NTAPS, bool ROWS = false>
__global__ void __launch_bounds__(NT) band_kernel(const BandWork p)
{
    extern __shared__ __align__(16) unsigned char smem[];
    process_box<DIM, NTAPS, ROWS>(p, blockIdx.x, smem, NT);
}

} // namespace band

cudaError_t prepare_band(size_t max_smem)
{
    cudaError_t e = cudaSuccess;
    auto set = [&](const void *k) {
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
    };
    set((const void *)band::band_kernel<1, 0>);
    set((const void *)band::band_kernel<2, 0>);
    set((const void *)band::band_kernel<2, 5>);
    set((const void *)band::band_kernel<2, 9>);
    set((const void *)band::band_kernel<2, 9, true>);
    set((const void *)band::band_kernel<3, 0>);
    set((const void *)band::band_kernel<3, 7>);
    set((const void *)band::band_kernel<3, 27>);
    return e;
}

cudaError_t launch_band(const BandWork &w, size_t smem_bytes, cudaStream_t s)
{
    if (w.nboxes <= 0)
        return cudaSuccess;
    // stencils of 5 and 9 (2D: Heat-2D; Box2D9P, Star2D9P) and 7 and 27 (3D: Heat-3D, Box3D27P)
    // non-zero taps keep their taps in registers
    if (w.dim == 1)
        band::band_kernel<1, 0><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else if (w.dim == 2 && w.ntaps == 5)
        band::band_kernel<2, 5><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else if (w.dim == 2 && w.ntaps == 9 && w.warp_rows)
        band::band_kernel<2, 9, true><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else if (w.dim == 2 && w.ntaps == 9)
        band::band_kernel<2, 9><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else if (w.dim == 2)
        band::band_kernel<2, 0><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else if (w.ntaps == 7)
        band::band_kernel<3, 7><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else if (w.ntaps == 27)
        band::band_kernel<3, 27><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    else
        band::band_kernel<3, 0><<<w.nboxes, band::NT, smem_bytes, s>>>(w);
    return cudaGetLastError();
}

size_t band_smem_bytes(int64_t max_vol, int ntaps)
{
    return 2 * (size_t)((max_vol + 1) & ~(int64_t)1) * sizeof(double) + ((ntaps + 1) & ~1) * sizeof(double) +
           ntaps * sizeof(int);
}

} // namespace ffst
