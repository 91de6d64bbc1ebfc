// Radix-8 butterfly DFT-64 of one line by a group of 8 threads, shared by the 1D
// and 2D FP64 butterfly kernels (ffs_fft1d.cu, ffs_fft2d.cu).
#pragma once
#include "ffs_device.cuh"

namespace ffst {
namespace fft64 {

// Complex 64 x 64 work tile: element (y, x) in 16-byte slot y * 64 + (x ^ (y & 7)).
// The row and column accesses of the butterfly kernels have the 8 threads of a group
// (one quarter warp for 16-byte accesses) on 8 distinct slots modulo 8, i.e. on all
// 32 banks once.
__device__ __forceinline__ int widx(int y, int x) { return (y << 6) | (x ^ (y & 7)); }

// In-place DFT-8 of (xr, xi) over the register index, natural order out:
// X[k] = sum_a x[a] w^(a k), w = exp(-+ 2 pi i / 8) (forward / inverse).
// Radix-2 decimation in frequency; the last stage's outputs land at bit-reversed
// positions, renamed at compile time.
template <bool INV>
__device__ __forceinline__ void dft8(double (&xr)[8], double (&xi)[8])
{
    constexpr double R = 0.70710678118654752440;
    double ar[8], ai[8];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        ar[a] = xr[a] + xr[a + 4];
        ai[a] = xi[a] + xi[a + 4];
        ar[a + 4] = xr[a] - xr[a + 4];
        ai[a + 4] = xi[a] - xi[a + 4];
    }
    { // w^1, w^2, w^3 on the difference half
        const double r1 = ar[5], i1 = ai[5], r3 = ar[7], i3 = ai[7], r2 = ar[6], i2 = ai[6];
        if (!INV) {
            ar[5] = (r1 + i1) * R;
            ai[5] = (i1 - r1) * R;
            ar[6] = i2;
            ai[6] = -r2;
            ar[7] = (i3 - r3) * R;
            ai[7] = -(r3 + i3) * R;
        } else {
            ar[5] = (r1 - i1) * R;
            ai[5] = (r1 + i1) * R;
            ar[6] = -i2;
            ai[6] = r2;
            ar[7] = -(r3 + i3) * R;
            ai[7] = (r3 - i3) * R;
        }
    }
    double br[8], bi[8];
#pragma unroll
    for (int h = 0; h < 8; h += 4) {
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            br[h + b] = ar[h + b] + ar[h + b + 2];
            bi[h + b] = ai[h + b] + ai[h + b + 2];
            br[h + b + 2] = ar[h + b] - ar[h + b + 2];
            bi[h + b + 2] = ai[h + b] - ai[h + b + 2];
        }
        const double r = br[h + 3], i = bi[h + 3]; // w4^1 = -+i
        br[h + 3] = INV ? -i : i;
        bi[h + 3] = INV ? r : -r;
    }
    // last stage: position p = 4 e1 + 2 e2 + e3 holds frequency 4 e3 + 2 e2 + e1
#pragma unroll
    for (int p = 0; p < 8; p += 2) {
        const int k0 = ((p & 1) << 2) | (p & 2) | ((p >> 2) & 1);             // bitrev3(p)
        const int k1 = (((p + 1) & 1) << 2) | ((p + 1) & 2) | (((p + 1) >> 2) & 1);
        xr[k0] = br[p] + br[p + 1];
        xi[k0] = bi[p] + bi[p + 1];
        xr[k1] = br[p] - br[p + 1];
        xi[k1] = bi[p] - bi[p + 1];
    }
}

struct Twiddle {
    double re[8], im[8]; // w64^(j k1), k1 = 0..7 (forward; the inverse conjugates)
};

// One DFT-64 of a line by its 8-thread group.  On entry thread j holds the points
// 8a + j in (xr[a], xi[a]); on exit it holds the outputs j + 8 k2 in (xr[k2], xi[k2]).
// `slot(p)` is the work-tile slot of line position p, used for the transpose;
// `gmask` is the group's lane mask.
template <bool INV, class Slot>
__device__ __forceinline__ void dft64_line(double (&xr)[8], double (&xi)[8], const Twiddle &tw, int j,
                                           double2 *work, Slot slot, unsigned gmask)
{
    dft8<INV>(xr, xi);
#pragma unroll
    for (int k = 1; k < 8; ++k) {
        const double wi = INV ? -tw.im[k] : tw.im[k];
        cmul(xr[k], xi[k], tw.re[k], wi);
    }
    // transpose: value (j, k1) goes to position 8 k1 + (j ^ k1), so that every
    // quarter-warp access below touches 8 distinct slots
#pragma unroll
    for (int k = 0; k < 8; ++k)
        work[slot(8 * k + (j ^ k))] = make_double2(xr[k], xi[k]);
    __syncwarp(gmask);
#pragma unroll
    for (int jj = 0; jj < 8; ++jj) {
        const double2 v = work[slot(8 * j + (jj ^ j))];
        xr[jj] = v.x;
        xi[jj] = v.y;
    }
    __syncwarp(gmask);
    dft8<INV>(xr, xi);
}

} // namespace fft64
} // namespace ffst
