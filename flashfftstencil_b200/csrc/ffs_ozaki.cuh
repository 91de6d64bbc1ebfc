// FP64 <-> integer-slice helpers of the Ozaki scheme (shared by the 2D and 3D
// tcgen05 forms).  Published method: Ozaki, Ogita, Oishi & Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication and its applications", Numer. Algorithms 59 (2012), with the
// integer-slice variant of Ootomo, Ozaki & Yokota (2024) on INT8 tensor cores.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ffst {
namespace oz {

__device__ __forceinline__ double pow2(int e) // 2^e for |e| < 1000
{
    return __hiloint2double((e + 1023) << 20, 0);
}

__device__ __forceinline__ int exponent_above(double m) // smallest e with m < 2^e (m > 0)
{
    return ((__double2hiint(m) >> 20) & 0x7ff) - 1022;
}

// signed 7-bit digits of y (|y| <= 64): d_0 = rint(y), y <- (y - d_0) * 128, ...
// (rint through the 1.5 * 2^52 addition, exact for |y| < 2^51)
template <int S>
__device__ __forceinline__ void digits(double y, int (&d)[S])
{
    const double magic = 6755399441055744.0; // 1.5 * 2^52
#pragma unroll
    for (int i = 0; i < S; ++i) {
        const double t = y + magic;
        const double q = t - magic;
        d[i] = __double2loint(t);
        y = (y - q) * 128.0;
    }
}

__device__ __forceinline__ double i32_to_f64(uint32_t v) // exact, via the 2^52 + 2^31 bias
{
    return __hiloint2double(0x43300000, (int)(v ^ 0x80000000u)) - 4503601774854144.0;
}

} // namespace oz
} // namespace ffst
