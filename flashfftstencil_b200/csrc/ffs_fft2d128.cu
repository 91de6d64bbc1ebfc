// FP64 fused DFT-tile stencil kernel for 2D grids on a 128 x 128 real tile per CTA
// (butterflies on the FP64 pipe).  The per-thread pieces and the data layout are in
// ffs_fft2d128.cuh.
//
// Why a larger tile: with halo h = r tau the 64 x 64 tile keeps (64 - 2h)^2 cells of
// 64^2 (tau 8: 48^2) and the 128 x 128 tile (128 - 2h)^2 of 128^2 (tau 16: 96^2), so at
// twice the fused steps per pass it keeps the same fraction and does about 1.8x less
// butterfly work and 2.2x fewer shared-memory bytes per cell-step.  A real 128^2 tile
// held as 64 complex row pairs is 128 KB, one CTA of 512 threads per SM: 64 groups of 8,
// one line per group and pass (16 warps; 256 threads with two lines per group had no spills
// at 255 registers but measured 10-12 % slower):
//   A. row pair r from global memory (re = row 2r, im = row 2r+1), FFT-128;
//   B. column kx = 1..63 of the half spectrum (kx = 0: columns 0 and 64, packed as one
//      line), FFT-128, times S^tau / 128^2, inverse FFT-128;
//   C. row pair h/2 + q (q < u/2) rebuilt from the half spectrum, inverse FFT-128, cropped
//      stores of rows 2r and 2r+1.
// Two block barriers per tile (A -> B, B -> C): group g takes row pair h/2 + g (mod 64) in
// pass A, the pair it rebuilds in pass C, so C -> next A needs none, and the 64 - u/2 groups
// idle in pass C load the next tile meanwhile (Box2D9P 4096^2: 0.2504 -> 0.2419 ms per
// launch).  Within a group the line exchanges need only the group's own 8 lanes (__syncwarp
// on the group's mask).  The packed line multiplies by two spectrum
// columns, S(ky, 0) and S(ky, 64), which are staged in shared memory once per launch: read
// from L2 inside pass B, they held the packed line's warp, and at the barrier after pass B every
// other warp (the launch measured 10 % longer).
// Same overlap-save geometry, crop and band as the 64 x 64 forms, with single tiles instead
// of pairs along x.  Replaces rfft_2d (src/2D/rfft_2d/2d_rfft_1_async.cu:17-364) like them.
#include <algorithm>

#include "ffs_device.cuh"
#include "ffs_fft2d128.cuh"

namespace ffst {
namespace fft2d128 {

using namespace f128;

constexpr int NT = 512;                                          // 64 groups of 8 threads
constexpr int GROUPS = NT / 8;
static_assert(GROUPS == RP, "one row pair per group in pass A");
constexpr size_t WORK_BYTES = (size_t)RP * N * sizeof(double2);  // 128 KB
constexpr size_t SMEM_BYTES = WORK_BYTES + 3 * N * sizeof(double2); // + the 128th roots, S(ky, 0), S(ky, 64)
constexpr int kRootsOffset = 8 + 64; // the plan's tables: DFT-8 roots, 64th roots, 128th roots

struct Tile {
    int64_t lx, ly;
};

// 32-bit quotient (the launcher rejects 2^32 tiles or more): the 64-bit division's
// registers raised the kernel's spills from 60 to 140 bytes.
__device__ __forceinline__ Tile tile_of(const TileWork &p, int64_t w)
{
    Tile t;
    const uint32_t w32 = (uint32_t)w, npx = (uint32_t)p.npx, q = w32 / npx;
    const int64_t tx = p.t0[0] + (w32 - q * npx), ty = p.t0[1] + q;
    t.lx = tx * p.useful - p.halo;
    t.ly = ty * p.useful - p.halo;
    return t;
}

// Row pair r of tile t: z[8a + j] = row 2r + i row 2r+1; zeros outside a fixed-boundary
// grid, periodic wrap otherwise.  All loads are issued before the first use.
__device__ __forceinline__ void load_rows(double (&xr)[PTS], double (&xi)[PTS], const TileWork &p, const Tile &t,
                                          int r, int j)
{
    const int64_t gy0 = t.ly + 2 * r;
    const bool inside = t.lx >= 0 && t.lx + N <= p.nx && t.ly >= 0 && t.ly + N <= p.ny;
    if (inside) {
        const double *r0 = p.in + gy0 * p.nx + t.lx + j;
        const double *r1 = r0 + p.nx;
#pragma unroll
        for (int a = 0; a < PTS; ++a) {
            xr[a] = __ldcg(r0 + 8 * a);
            xi[a] = __ldcg(r1 + 8 * a);
        }
        return;
    }
    int64_t y0 = gy0, y1 = gy0 + 1;
    bool ok0 = y0 >= 0 && y0 < p.ny, ok1 = y1 >= 0 && y1 < p.ny;
    if (p.periodic) {
        y0 = wrap_near(y0, p.ny);
        y1 = wrap_near(y1, p.ny);
        ok0 = ok1 = true;
    }
#pragma unroll
    for (int a = 0; a < PTS; ++a) {
        int64_t gx = t.lx + 8 * a + j;
        bool okx = gx >= 0 && gx < p.nx;
        if (p.periodic) {
            gx = wrap_near(gx, p.nx);
            okx = true;
        }
        xr[a] = (ok0 && okx) ? __ldcg(p.in + y0 * p.nx + gx) : 0.0;
        xi[a] = (ok1 && okx) ? __ldcg(p.in + y1 * p.nx + gx) : 0.0;
    }
}

// One line transform of a group: piece 1, exchange through the line's slots, piece 3.
template <bool INV, class LS>
__device__ __forceinline__ void line_fft(double (&xr)[PTS], double (&xi)[PTS], int j, const double2 *roots,
                                         double2 *work, LS ls, unsigned gmask)
{
    line_piece1<INV>(xr, xi);
    __syncwarp(gmask); // every thread of the group has read the line's slots
    line_put<INV>(xr, xi, j, roots, work, ls);
    __syncwarp(gmask);
    line_get<INV>(xr, xi, j, work, ls);
    __syncwarp(gmask); // the slots may be written again
}

__global__ void __launch_bounds__(NT, 1) fft2d128_kernel(const TileWork p)
{
    extern __shared__ __align__(16) unsigned char smem[];
    double2 *work = reinterpret_cast<double2 *>(smem);
    double2 *roots = work + RP * N;
    const int tid = threadIdx.x, g = tid >> 3, j = tid & 7;
    const unsigned gmask = 0xffu << (tid & 24); // the 8 lanes of this group
    double2 *spec_pk = roots + N; // the spectrum's columns 0 and 64 (the packed line), S(ky, 0) at ky
    for (int i = tid; i < N; i += NT) { // twiddle of thread j and index k1 at 8 k1 + j: w128^(j k1)
        roots[i] = p.tables[kRootsOffset + (((i & 7) * (i >> 3)) & (N - 1))];
        spec_pk[i] = p.spec[i];
        spec_pk[N + i] = p.spec[64 * N + i];
    }
    __syncthreads();
    const int h = p.halo, u = p.useful;
    double xr[PTS], xi[PTS];
    for (int64_t w = blockIdx.x; w < p.nitems; w += gridDim.x) {
        const Tile t = tile_of(p, w);
        { // A: row pair r = h/2 + g (mod 64), forward: the pair this group rebuilds in pass C
            const int r = (h / 2 + g) & (RP - 1);
            load_rows(xr, xi, p, t, r, j);
            line_fft<false>(xr, xi, j, roots, work, RowSlots{r}, gmask);
#pragma unroll
            for (int m = 0; m < PTS; ++m)
                work[slot(r, j + 8 * m)] = make_double2(xr[m], xi[m]);
        }
        __syncthreads();
        for (int kx = g; kx < 64; kx += GROUPS) { // B: column kx (kx = 0: columns 0 and 64 packed)
            const bool packed = kx == 0;
            const ColSlots ls = col_slots(kx);
            if (packed)
                pack_gather(xr, xi, j, work);
            else
                col_gather(xr, xi, kx, j, work);
            line_fft<false>(xr, xi, j, roots, work, ls, gmask);
            if (packed) { // C[ky] through the line's own slots, C[128 - ky] read back
#pragma unroll
                for (int m = 0; m < PTS; ++m)
                    work[ls(j + 8 * m)] = make_double2(xr[m], xi[m]);
                __syncwarp(gmask);
#pragma unroll
                for (int m = 0; m < PTS; ++m) {
                    const int ky = j + 8 * m;
                    const double2 c = work[ls((N - ky) & (N - 1))];
                    pack_spectrum(xr[m], xi[m], c.x, c.y, spec_pk[ky], spec_pk[N + ky]);
                }
            } else {
                const double2 *sp = p.spec + kx * N + j; // S(ky, kx) at kx * 128 + ky
#pragma unroll
                for (int m = 0; m < PTS; ++m) {
                    const double2 sv = __ldg(sp + 8 * m);
                    f128::cmul(xr[m], xi[m], sv.x, sv.y);
                }
            }
            line_fft<true>(xr, xi, j, roots, work, ls, gmask);
            if (packed) {
                // Z'_r[0] = col0[2r] + i col0[2r+1], Z'_r[64] = col64[2r] + i col64[2r+1]: thread j
                // holds row y = j + 8m (r = 4m + j/2) and writes its half of both slots
                double *w0 = reinterpret_cast<double *>(work);
#pragma unroll
                for (int m = 0; m < PTS; ++m) {
                    const int r = 4 * m + (j >> 1);
                    w0[2 * slot(r, 0) + (j & 1)] = xr[m];
                    w0[2 * slot(r, 64) + (j & 1)] = xi[m];
                }
            } else {
                col_scatter(xr, xi, kx, j, work);
            }
        }
        __syncthreads();
        for (int q = g; q < u / 2; q += GROUPS) { // C: row pair h/2 + q, inverse, cropped stores
            const int r = h / 2 + q;
            row_gather_inverse(xr, xi, r, j, work);
            line_fft<true>(xr, xi, j, roots, work, RowSlots{r}, gmask);
            const int64_t gy0 = t.ly + 2 * r, gy1 = gy0 + 1;
            const bool y0_ok = gy0 >= p.vlo[1] && gy0 < p.vhi[1], y1_ok = gy1 >= p.vlo[1] && gy1 < p.vhi[1];
#pragma unroll
            for (int m = 0; m < PTS; ++m) {
                const int x = j + 8 * m;
                const int64_t gx = t.lx + x;
                if (x < h || x >= h + u || gx < p.vlo[0] || gx >= p.vhi[0])
                    continue;
                if (y0_ok)
                    p.out[gy0 * p.nx + gx] = xr[m];
                if (y1_ok)
                    p.out[gy1 * p.nx + gx] = xi[m];
            }
        }
        // no barrier: group g's next pass A writes only row pair h/2 + g (mod 64), the one it
        // read in pass C (for g >= u/2, one that no group reads in pass C), so the groups
        // idle in pass C start loading the next tile at once
    }
}

} // namespace fft2d128

size_t fft2d128_smem_bytes() { return fft2d128::SMEM_BYTES; }

cudaError_t prepare_fft2d128()
{
    return cudaFuncSetAttribute(fft2d128::fft2d128_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fft2d128::SMEM_BYTES);
}

cudaError_t launch_fft2d128(const TileWork &w, int grid, cudaStream_t s)
{
    if (w.nitems >= ((int64_t)1 << 32) || w.npx >= ((int64_t)1 << 32))
        return cudaErrorInvalidValue; // the kernel decodes tile indices in 32 bits
    fft2d128::fft2d128_kernel<<<grid, fft2d128::NT, fft2d128::SMEM_BYTES, s>>>(w);
    return cudaGetLastError();
}

} // namespace ffst
