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

// Exact int64 -> double for |x| < 2^51: the bit pattern of 1.5 * 2^52 plus x is
// the double 1.5 * 2^52 + x.
__host__ __device__ __forceinline__ double i64_to_f64(int64_t x)
{
    const int64_t b = x + 0x4338000000000000ll;
#ifdef __CUDA_ARCH__
    const double d = __longlong_as_double(b);
#else
    double d;
    __builtin_memcpy(&d, &b, 8);
#endif
    return d - 6755399441055744.0;
}

// V = sum_d 256^(-d) D_d for the S diagonal accumulators of one value.  Three
// diagonals at a time are summed exactly in int64 (|D_d| < 2^24, so a group is
// below 2^41), each group is converted once and the groups are combined in FP64.
template <int S>
__host__ __device__ __forceinline__ double combine(const uint32_t (&acc)[S])
{
    constexpr int G = (S + 2) / 3;
    double v = 0.0;
#pragma unroll
    for (int g = G - 1; g >= 0; --g) {
        const int d0 = 3 * g, n = (S - d0) < 3 ? (S - d0) : 3;
        int64_t x = (int32_t)acc[d0];
#pragma unroll
        for (int k = 1; k < n; ++k)
            x = x * 256 + (int32_t)acc[d0 + k];
        // this group is worth x * 256^(-(d0 + n - 1)); fold the later groups in below it
        const double gv = i64_to_f64(x) * (n == 3 ? 1.0 / 65536.0 : (n == 2 ? 1.0 / 256.0 : 1.0));
        v = (g == G - 1) ? gv : fma(v, 1.0 / 16777216.0, gv);
    }
    return v;
}

} // namespace oz
} // namespace ffst
