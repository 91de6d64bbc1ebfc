// FP64 <-> integer-slice helpers of the Ozaki scheme (shared by the 2D and 3D
// tcgen05 forms).  Published method: Ozaki, Ogita, Oishi & Rump, "Error-free
// transformations of matrix multiplication by using fast routines of matrix
// multiplication and its applications", Numer. Algorithms 59 (2012), with the
// integer-slice variant of Ootomo, Ozaki & Yokota (2024) on INT8 tensor cores.
//
// Slices here are balanced base-256 digits: a value scaled to |y| <= 64 is
// y = sum_i d_i 256^(-i) with d_0 in [-64, 64] and d_i in [-128, 127] (i > 0).
// A product of two digits is at most 2^14 in magnitude, so a K = 128 dot product
// of one slice pair stays below 2^21 and a diagonal of up to 8 slice pairs below
// 2^24: every diagonal sums exactly in INT32.
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

__host__ __device__ __forceinline__ uint64_t f64_bits(double x)
{
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    __builtin_memcpy(&u, &x, 8);
    return u;
#endif
}

// The S digits of y (|y| <= 64) as the bytes of one integer:
//   U = round(y * 256^(S-1)) + 0x80...80 (S bytes);
// byte S-1-i of U is d_i + 128.  The rounding is the 1.5 * 2^52 addition while
// |y * 256^(S-1)| <= 2^46 (S <= 6), a 64-bit conversion beyond.
template <int S>
__host__ __device__ __forceinline__ uint64_t digit_bytes(double y)
{
    static_assert(S >= 2 && S <= 8, "2 to 8 digits");
    constexpr uint64_t bias = 0x8080808080808080ull >> (8 * (8 - S));
    const double scale = (double)(1ull << (8 * (S - 1)));
    int64_t X;
    if constexpr (S <= 6) {
        const double t = fma(y, scale, 6755399441055744.0);
        X = (int64_t)(f64_bits(t) & ((1ull << 52) - 1)) - (1ll << 51);
    } else {
#ifdef __CUDA_ARCH__
        X = __double2ll_rn(y * scale);
#else
        X = llrint(y * scale);
#endif
    }
    return (uint64_t)X + bias;
}

// Byte k of four words as one word of int8 digits (byte - 128 = byte ^ 0x80).
__device__ __forceinline__ uint32_t gather_digit(uint32_t a, uint32_t b, uint32_t c, uint32_t d, int k)
{
    const uint32_t sel = (uint32_t)k | ((uint32_t)(4 + k) << 4);
    const uint32_t ab = __byte_perm(a, b, sel);
    const uint32_t cd = __byte_perm(c, d, sel);
    return __byte_perm(ab, cd, 0x5410) ^ 0x80808080u;
}

// w[i][q] = digit i of the four values U[4q .. 4q+3] (from digit_bytes), packed.
template <int S, int NV>
__device__ __forceinline__ void digit_words(const uint64_t (&U)[NV], uint32_t (&w)[S][NV / 4])
{
#pragma unroll
    for (int q = 0; q < NV / 4; ++q)
#pragma unroll
        for (int i = 0; i < S; ++i) {
            const int byte = S - 1 - i;
            const int sh = byte < 4 ? 0 : 32, k = byte & 3;
            w[i][q] = gather_digit((uint32_t)(U[4 * q] >> sh), (uint32_t)(U[4 * q + 1] >> sh),
                                   (uint32_t)(U[4 * q + 2] >> sh), (uint32_t)(U[4 * q + 3] >> sh), k);
        }
}

__device__ __forceinline__ double i32_to_f64(uint32_t v) // exact, via the 2^52 + 2^31 bias
{
    return __hiloint2double(0x43300000, (int)(v ^ 0x80000000u)) - 4503601774854144.0;
}

// V = sum_d 256^(-d) D_d for the S diagonal accumulators of one value (Horner, FMA).
template <int S>
__device__ __forceinline__ double combine(const uint32_t (&acc)[S])
{
    double s = i32_to_f64(acc[S - 1]);
#pragma unroll
    for (int d = S - 2; d >= 0; --d)
        s = fma(s, 0.00390625, i32_to_f64(acc[d]));
    return s;
}

} // namespace oz
} // namespace ffst
