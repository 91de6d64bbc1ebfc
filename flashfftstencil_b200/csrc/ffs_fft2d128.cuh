// 2D FP64 butterfly form on one 128 x 128 real tile per CTA: the per-thread pieces of
// the kernel (ffs_fft2d128.cu), host-callable so the decomposition can be run on the CPU.
//
// Work buffer: the tile's 64 row pairs r, each as one complex row z = row 2r + i row 2r+1
// (128 points), slot(r, x) = 128 r + (x ^ (r & 7)): 128 KB.
//
// FFT-128 of a line by a group of 8 threads.  Thread j holds points 8a + j (a = 0..15):
//   X[k1 + 16 k2] = sum_j w8^(j k2) [ w128^(j k1) sum_a x[8a + j] w16^(a k1) ]
// piece 1: DFT-16 over a in registers; put: Y_j[k1] times w128^(j k1) (a per-thread table,
// entry 8 k1 + j) into the line's exchange slot 8 k1 + (j ^ (k1 & 7)); get: thread t gathers
// Y_j[k1] for k1 = t and t + 8 over j and takes the two DFT-8 over j.  Thread t then holds
// frequencies t + 8m (m = 0..15), the same layout as its input points, so a forward transform
// feeds an inverse one with no reordering.  In every put and get the 8 threads of a group
// touch 8 distinct 16-byte bank groups, on row lines and on column lines alike (ColSlots).
//
// Pass A (rows): group r transforms row pair r (the two real rows packed as one complex
// row).  Pass B (columns): column kx = 1..63 gathers its half-spectrum values
//   A_2r[kx] = (Z_r[kx] + conj Z_r[128-kx]) / 2,  B_2r+1[kx] = (Z_r[kx] - conj Z_r[128-kx]) / 2i
// over y, transforms them, multiplies by S(ky, kx), transforms back and leaves A'_2r[kx]
// in slot (r, kx) and B'_2r+1[kx] in slot (r, 128-kx), the slots it read.  Columns 0 and 64
// are real along y and share one packed line (c = A[0] + i A[64]), separated after the
// forward transform by Hermitian symmetry.  Pass C (rows): group r rebuilds
//   Z'_r[x] = A'_2r[x] + i B'_2r+1[x]  (x <= 64),  conj A'[128-x] + i conj B'[128-x]  (x > 64)
// and its inverse transform is row 2r (real part) and row 2r+1 (imaginary part).
#pragma once
#include <cuda_runtime.h>

#include "ffs_dft32.cuh"

namespace ffst {
namespace f128 {

constexpr int N = 128;  // tile edge
constexpr int RP = 64;  // row pairs
constexpr int PTS = 16; // points per thread and line

__host__ __device__ __forceinline__ int slot(int r, int x) { return (r << 7) | (x ^ (r & 7)); }

// exchange slots of a line: row pair r; column kx in 1..63; the packed column of kx = 0, 64
struct RowSlots {
    int r;
    __host__ __device__ __forceinline__ int operator()(int e) const { return slot(r, e); }
};
// column line of x0 and x1 (column kx: kx and 128 - kx; the packed column: 0 and 64): index e
// in row (e & 7) | ((e >> 4) << 3), at x1 when bit 3 of e is set.  A put's 8 consecutive e
// then land in 8 consecutive rows of one column, and a get's 8 threads in rows of distinct
// e & 7 with x0 and x1 alternating (x0, x1 of equal parity): every access distinct bank groups.
struct ColSlots {
    int x0, x1;
    __host__ __device__ __forceinline__ int operator()(int e) const
    {
        return slot((e & 7) | ((e >> 4) << 3), ((e >> 3) & 1) ? x1 : x0);
    }
};
__host__ __device__ __forceinline__ ColSlots col_slots(int kx) { return kx == 0 ? ColSlots{0, 64} : ColSlots{kx, N - kx}; }

// Compiler-only fence: shared loads after it are not hoisted above it.  A gather of 16 points
// (32 shared loads) otherwise has every load in flight at once, 64 doubles live, and a
// 512-thread block (128 registers) spills.
__host__ __device__ __forceinline__ void hoist_fence()
{
#ifdef __CUDA_ARCH__
    asm volatile("" ::: "memory");
#endif
}

__host__ __device__ __forceinline__ void cmul(double &re, double &im, double wr, double wi)
{
    const double r = re * wr - im * wi;
    const double i = re * wi + im * wr;
    re = r;
    im = i;
}

// DFT-16 of 16 values in registers, natural order in and out (4 x 4: n = 4 n1 + n2,
// k = k1 + 4 k2; twiddle w16^(n2 k1) = w32^(2 n2 k1)).
template <bool INV>
__host__ __device__ __forceinline__ void dft16(double (&xr)[PTS], double (&xi)[PTS])
{
    using namespace dft32;
    dft4<0, 4, INV>(xr, xi);
    dft4<1, 4, INV>(xr, xi);
    dft4<2, 4, INV>(xr, xi);
    dft4<3, 4, INV>(xr, xi);
    rot<2, INV>(xr[5], xi[5]);
    rot<4, INV>(xr[6], xi[6]);
    rot<6, INV>(xr[7], xi[7]);
    rot<4, INV>(xr[9], xi[9]);
    rot<8, INV>(xr[10], xi[10]);
    rot<12, INV>(xr[11], xi[11]);
    rot<6, INV>(xr[13], xi[13]);
    rot<12, INV>(xr[14], xi[14]);
    rot<18, INV>(xr[15], xi[15]);
    dft4<0, 1, INV>(xr, xi);
    dft4<4, 1, INV>(xr, xi);
    dft4<8, 1, INV>(xr, xi);
    dft4<12, 1, INV>(xr, xi);
    double yr[PTS], yi[PTS];
#pragma unroll
    for (int s = 0; s < PTS; ++s) {
        yr[s] = xr[s];
        yi[s] = xi[s];
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) {
            xr[k1 + 4 * k2] = yr[4 * k1 + k2];
            xi[k1 + 4 * k2] = yi[4 * k1 + k2];
        }
}

// piece 1: DFT-16 over a (the twiddle w128^(j k1) is applied by line_put)
template <bool INV>
__host__ __device__ __forceinline__ void line_piece1(double (&xr)[PTS], double (&xi)[PTS])
{
    dft16<INV>(xr, xi);
}

// put: Y_j[k1] * w128^(j k1) into the line's exchange slot 8 k1 + (j ^ (k1 & 7)); each
// value is multiplied and stored in turn, so the registers free as the loop goes.
// tw[8 k1 + j] = w128^(j k1) = exp(-2 pi i j k1 / 128): for each k1 the 8 threads of a group
// read 8 consecutive entries (a table of w128^m indexed by j k1 put 2 to 8 of them on one
// bank group for even k1).
template <bool INV, class LS>
__host__ __device__ __forceinline__ void line_put(double (&xr)[PTS], double (&xi)[PTS], int j, const double2 *tw,
                                                  double2 *work, LS ls)
{
    work[ls(j)] = make_double2(xr[0], xi[0]);
#pragma unroll
    for (int k1 = 1; k1 < PTS; ++k1) {
        const double2 w = tw[8 * k1 + j];
        cmul(xr[k1], xi[k1], w.x, INV ? -w.y : w.y);
        work[ls(8 * k1 + (j ^ (k1 & 7)))] = make_double2(xr[k1], xi[k1]);
    }
}

// get: DFT-8 over j of Y_j[t] and Y_j[t + 8] (one after the other); frequency t + 8m lands
// in (xr, xi)[m]
template <bool INV, class LS>
__host__ __device__ __forceinline__ void line_get(double (&xr)[PTS], double (&xi)[PTS], int t, const double2 *work,
                                                  LS ls)
{
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
        double ar[8], ai[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
            const double2 u = work[ls(8 * (t + 8 * hh) + (jj ^ t))];
            ar[jj] = u.x;
            ai[jj] = u.y;
        }
        dft32::dft8<0, INV>(ar, ai);
#pragma unroll
        for (int k2 = 0; k2 < 8; ++k2) {
            xr[2 * k2 + hh] = ar[k2];
            xi[2 * k2 + hh] = ai[k2];
        }
    }
}

// pass B, column kx in 1..63: thread j's values at y = 8a + j (r = 4a + j/2)
__host__ __device__ __forceinline__ void col_gather(double (&xr)[PTS], double (&xi)[PTS], int kx, int j,
                                                    const double2 *work)
{
    const bool odd = j & 1;
#pragma unroll
    for (int a = 0; a < PTS; ++a) {
        const int r = 4 * a + (j >> 1);
        const double2 zk = work[slot(r, kx)], zm = work[slot(r, N - kx)];
        xr[a] = odd ? 0.5 * (zk.y + zm.y) : 0.5 * (zk.x + zm.x);
        xi[a] = odd ? -0.5 * (zk.x - zm.x) : 0.5 * (zk.y - zm.y);
        if (a % 4 == 3)
            hoist_fence();
    }
}

// pass B, column kx in 1..63, after the inverse transform: y = j + 8m (r = 4m + j/2)
__host__ __device__ __forceinline__ void col_scatter(const double (&xr)[PTS], const double (&xi)[PTS], int kx, int j,
                                                     double2 *work)
{
#pragma unroll
    for (int m = 0; m < PTS; ++m)
        work[slot(4 * m + (j >> 1), (j & 1) ? N - kx : kx)] = make_double2(xr[m], xi[m]);
}

// the packed column: c[y] = A_y[0] + i A_y[64], y = 8a + j
__host__ __device__ __forceinline__ void pack_gather(double (&xr)[PTS], double (&xi)[PTS], int j, const double2 *work)
{
    const bool odd = j & 1;
#pragma unroll
    for (int a = 0; a < PTS; ++a) {
        const int r = 4 * a + (j >> 1);
        const double2 z0 = work[slot(r, 0)], z64 = work[slot(r, 64)];
        xr[a] = odd ? z0.y : z0.x;
        xi[a] = odd ? z64.y : z64.x;
        if (a % 4 == 3)
            hoist_fence();
    }
}

// Index m' of C[128 - ky] in partner thread (8 - j) & 7, for ky = j + 8m: the value thread j
// sends at step m is its own index ((16 - m) & 15 for j == 0, 15 - m otherwise).
__host__ __device__ __forceinline__ constexpr int pack_partner_index(bool j_zero, int m)
{
    return j_zero ? ((16 - m) & 15) : 15 - m;
}

// Packed column, after the forward transform: C[ky] and Cm = C[-ky] -> the two real
// columns' spectra F0 = (C + conj Cm) / 2 and F64 = (C - conj Cm) / 2i, times S(ky, 0) and
// S(ky, 64), recombined as F0' + i F64'.
__host__ __device__ __forceinline__ void pack_spectrum(double &cr, double &ci, double mr, double mi, double2 s0,
                                                       double2 s64)
{
    double f0r = 0.5 * (cr + mr), f0i = 0.5 * (ci - mi);
    double f6r = 0.5 * (ci + mi), f6i = -0.5 * (cr - mr);
    cmul(f0r, f0i, s0.x, s0.y);
    cmul(f6r, f6i, s64.x, s64.y);
    cr = f0r - f6i;
    ci = f0i + f6r;
}

// pass C, row pair r: thread j's points x = 8a + j of Z'_r
__host__ __device__ __forceinline__ void row_gather_inverse(double (&xr)[PTS], double (&xi)[PTS], int r, int j,
                                                            const double2 *work)
{
#pragma unroll
    for (int a = 0; a < PTS; ++a) {
        const int x = 8 * a + j;
        if (x == 0 || x == 64) {
            const double2 v = work[slot(r, x)];
            xr[a] = v.x;
            xi[a] = v.y;
        } else if (a < 8) { // 1 <= x <= 63: A'[x] + i B'[x]
            const double2 pa = work[slot(r, x)], qb = work[slot(r, N - x)];
            xr[a] = pa.x - qb.y;
            xi[a] = pa.y + qb.x;
        } else { // 65 <= x <= 127: conj A'[128-x] + i conj B'[128-x]
            const double2 pa = work[slot(r, N - x)], qb = work[slot(r, x)];
            xr[a] = pa.x + qb.y;
            xi[a] = qb.x - pa.y;
        }
        if (a % 4 == 3)
            hoist_fence();
    }
}

} // namespace f128
} // namespace ffst
