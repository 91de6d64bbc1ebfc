// DFT-32 of one line held in one thread's registers (FP64, compile-time roots).
//
// X[k] = sum_n x[n] w^(n k), w = exp(-2 pi i / 32) forward and its conjugate for
// the inverse (no scaling), natural order in and out.  Cooley-Tukey 4 x 8:
// n = 8 n1 + n2, k = k1 + 4 k2.  A DFT-4 over n1 for each n2 leaves k1 in slot
// 8 k1 + n2; the twiddle w^(n2 k1); a DFT-8 over n2 for each k1 (itself 2 x 4)
// leaves k2 in slot 8 k1 + k2; the final 4 x 8 index transpose is a renaming.
// About 13 FP64 operations per point.  Host-callable, so the factorisation can be
// checked against a direct DFT without a GPU.
#pragma once

namespace ffst {
namespace dft32 {

constexpr int N = 32;

// cos(2 pi m / 32) for m = 0..8 (correctly rounded doubles)
__host__ __device__ constexpr double cos32(int m)
{
    return m == 0   ? 1.0
           : m == 1 ? 0.9807852804032304
           : m == 2 ? 0.9238795325112867
           : m == 3 ? 0.8314696123025452
           : m == 4 ? 0.7071067811865476
           : m == 5 ? 0.5555702330196022
           : m == 6 ? 0.3826834323650898
           : m == 7 ? 0.19509032201612828
                    : 0.0;
}

// cos and sin of 2 pi m / 32 for any m, from the first-octant table by symmetry
__host__ __device__ constexpr double cosf32(int m)
{
    m &= 31;
    return m <= 8 ? cos32(m) : m <= 16 ? -cos32(16 - m) : m <= 24 ? -cos32(m - 16) : cos32(32 - m);
}
__host__ __device__ constexpr double sinf32(int m) { return cosf32(m - 8); }

// (re + i im) *= w^M, w = exp(-2 pi i / 32) (INV: exp(+2 pi i / 32)).
template <int M, bool INV>
__host__ __device__ __forceinline__ void rot(double &re, double &im)
{
    constexpr int m = ((M % 32) + 32) % 32;
    if constexpr (m == 0) {
        return;
    } else if constexpr (m == 16) {
        re = -re;
        im = -im;
    } else if constexpr (m == 8 || m == 24) { // w^8 = -i forward
        constexpr bool minus_i = (m == 8) != INV;
        const double r = re;
        re = minus_i ? im : -im;
        im = minus_i ? -r : r;
    } else {
        // w^m = c - i s forward, c + i s inverse
        constexpr double c = cosf32(m), s = INV ? -sinf32(m) : sinf32(m);
        const double r = re * c + im * s;
        const double i = im * c - re * s;
        re = r;
        im = i;
    }
}

// DFT-4 over slots B, B + S, B + 2S, B + 3S of a length-L line, natural order out.
template <int B, int S, bool INV, int L>
__host__ __device__ __forceinline__ void dft4(double (&xr)[L], double (&xi)[L])
{
    const double t0r = xr[B] + xr[B + 2 * S], t0i = xi[B] + xi[B + 2 * S];
    const double t1r = xr[B] - xr[B + 2 * S], t1i = xi[B] - xi[B + 2 * S];
    const double t2r = xr[B + S] + xr[B + 3 * S], t2i = xi[B + S] + xi[B + 3 * S];
    const double t3r = xr[B + S] - xr[B + 3 * S], t3i = xi[B + S] - xi[B + 3 * S];
    xr[B] = t0r + t2r;
    xi[B] = t0i + t2i;
    xr[B + 2 * S] = t0r - t2r;
    xi[B + 2 * S] = t0i - t2i;
    if (!INV) { // X1 = t1 - i t3, X3 = t1 + i t3
        xr[B + S] = t1r + t3i;
        xi[B + S] = t1i - t3r;
        xr[B + 3 * S] = t1r - t3i;
        xi[B + 3 * S] = t1i + t3r;
    } else {
        xr[B + S] = t1r - t3i;
        xi[B + S] = t1i + t3r;
        xr[B + 3 * S] = t1r + t3i;
        xi[B + 3 * S] = t1i - t3r;
    }
}

// DFT-8 over slots B + j, j = 0..7, natural order out: j = 4 a + b; DFT-2 over a
// (k1 in slot 4 k1 + b of a temporary), twiddle w8^(b k1) = w^(4 b k1), DFT-4 over b
// (k2 in slot 4 k1 + k2), X[k1 + 2 k2] written back to slot B + k1 + 2 k2.
template <int B, bool INV, int L>
__host__ __device__ __forceinline__ void dft8(double (&xr)[L], double (&xi)[L])
{
    double ar[8], ai[8];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        ar[b] = xr[B + b] + xr[B + b + 4];
        ai[b] = xi[B + b] + xi[B + b + 4];
        ar[4 + b] = xr[B + b] - xr[B + b + 4];
        ai[4 + b] = xi[B + b] - xi[B + b + 4];
    }
    rot<4, INV>(ar[5], ai[5]);
    rot<8, INV>(ar[6], ai[6]);
    rot<12, INV>(ar[7], ai[7]);
    dft4<0, 1, INV>(ar, ai);
    dft4<4, 1, INV>(ar, ai);
#pragma unroll
    for (int k1 = 0; k1 < 2; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) {
            xr[B + k1 + 2 * k2] = ar[4 * k1 + k2];
            xi[B + k1 + 2 * k2] = ai[4 * k1 + k2];
        }
}

template <int N2, bool INV>
__host__ __device__ __forceinline__ void twiddle_row(double (&xr)[N], double (&xi)[N])
{
    rot<N2 * 1, INV>(xr[8 + N2], xi[8 + N2]);
    rot<N2 * 2, INV>(xr[16 + N2], xi[16 + N2]);
    rot<N2 * 3, INV>(xr[24 + N2], xi[24 + N2]);
}

template <bool INV>
__host__ __device__ __forceinline__ void dft32(double (&xr)[N], double (&xi)[N])
{
    dft4<0, 8, INV>(xr, xi);
    dft4<1, 8, INV>(xr, xi);
    dft4<2, 8, INV>(xr, xi);
    dft4<3, 8, INV>(xr, xi);
    dft4<4, 8, INV>(xr, xi);
    dft4<5, 8, INV>(xr, xi);
    dft4<6, 8, INV>(xr, xi);
    dft4<7, 8, INV>(xr, xi);
    twiddle_row<1, INV>(xr, xi);
    twiddle_row<2, INV>(xr, xi);
    twiddle_row<3, INV>(xr, xi);
    twiddle_row<4, INV>(xr, xi);
    twiddle_row<5, INV>(xr, xi);
    twiddle_row<6, INV>(xr, xi);
    twiddle_row<7, INV>(xr, xi);
    dft8<0, INV>(xr, xi);
    dft8<8, INV>(xr, xi);
    dft8<16, INV>(xr, xi);
    dft8<24, INV>(xr, xi);
    // slot 8 k1 + k2 holds X[k1 + 4 k2]
    double yr[N], yi[N];
#pragma unroll
    for (int s = 0; s < N; ++s) {
        yr[s] = xr[s];
        yi[s] = xi[s];
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) {
            xr[k1 + 4 * k2] = yr[8 * k1 + k2];
            xi[k1 + 4 * k2] = yi[8 * k1 + k2];
        }
}

} // namespace dft32
} // namespace ffst
