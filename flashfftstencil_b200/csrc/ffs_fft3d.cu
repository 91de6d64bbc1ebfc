// FP64 fused DFT-tile stencil kernel for 3D grids on the FP64 pipe (radix-4 x 4
// butterflies, no tensor cores).
//
// B200 runs FP64 mma.sync at the plain FP64 FMA rate, so the DMMA form's DFT-16
// (two dense radix-4 GEMM stages, 32 FMAs per point) costs three times the FP64
// operations of a butterfly DFT-16 (about 10 per point).  A whole 16-point line
// fits in one thread's registers, so here every DFT-16 is done by one thread with
// no data exchange at all.  Per pair:
//   Z. thread (y, x) loads column (y, x) of both real tiles over z (a warp reads two
//      whole 128-byte rows per instruction; re = tile a, im = tile b), forward
//      DFT-16 along z in registers, stores to the work tile;
//   Y. thread (z, x): forward DFT-16 along y;
//   X. thread (z, y): forward DFT-16 along x, spectrum^tau / 16^3, inverse DFT-16;
//   Y'. thread (z, x) of a wanted x: inverse along y;
//   Z'. thread (y, x) of a wanted column: inverse along z, cropped stores (again two
//      whole rows per warp and instruction).
// Work tile slot (z, y, x) = 256 z + 16 y + (x ^ (y & 7)): in every pass the 8
// threads of a quarter warp read and write 8 distinct 16-byte bank groups.  Passes Y,
// X and Y' of plane z are all done by threads 16 z .. 16 z + 15 (one half warp), so
// only Z -> Y and Y' -> Z' need block barriers (two per pair); the rest are
// __syncwarp.  A CTA
// holds only its 64 KB work tile (the Hermitian half spectrum, 36 KB, is read through
// L1, which the CTAs of an SM share), so three CTAs of 256 threads share an SM and
// hide each other's global-load and barrier waits; the 80-register cap this needs
// spills about 150 bytes per thread and still measured 4 % faster than two CTAs.
// (One thread loading its own x-line from global memory made every warp instruction
// touch 32 rows; the z-columns are read and written as whole rows per warp instead.)
// Same tile geometry, halo, crop and band as the DMMA form (ffs_dmma3d.cuh).
// Replaces rfft_3d_8_nwarp (src/3D/rfft_3d/3d_rfft_N.cu:17-303) like that form.
#include <algorithm>

#include "ffs_dmma3d.cuh"

namespace ffst {
namespace fft3d {

constexpr int N = 16;
constexpr int VOL = N * N * N;
constexpr int NT = 256; // one thread per line
constexpr int HALF = N / 2 + 1; // spectrum columns kx = 0..8
constexpr size_t WORK_BYTES = (size_t)VOL * sizeof(double2);
constexpr size_t SPEC_BYTES = (size_t)N * N * HALF * sizeof(double2);
// Two layouts of the same passes, chosen per launch by its pair count:
//   CTAS = 3: a CTA holds only its 64 KB work tile and reads the Hermitian half
//     spectrum (36 KB) through L1, which the CTAs of an SM share; three CTAs per SM
//     hide each other's load and barrier waits, at an 80-register cap that spills
//     about 150 bytes per thread (the faster layout when every CTA has many pairs).
//   CTAS = 2: the spectrum is bulk-copied into shared memory behind the first loads
//     (100 KB per CTA, 128 registers, no spills): the lower latency per pair, for
//     launches with few pairs per CTA (small grids, batches of small problems).
template <int CTAS>
constexpr size_t smem_bytes()
{
    return CTAS == 3 ? WORK_BYTES + 16 : WORK_BYTES + SPEC_BYTES + 16;
}
static_assert(3 * smem_bytes<3>() <= 227 * 1024, "three CTAs per SM");
static_assert(2 * smem_bytes<2>() <= 227 * 1024, "two CTAs per SM");
// pairs per launch from which the three-CTA layout is used (8 pairs per CTA)
constexpr int64_t kThreeCtaPairsPerSm = 24;

__device__ __forceinline__ int slot(int z, int y, int x) { return (z << 8) | (y << 4) | (x ^ (y & 7)); }

// Complex multiply by the compile-time root w16^m (forward, w16 = exp(-2 pi i / 16))
// or its conjugate (inverse).
template <int M, bool INV>
__device__ __forceinline__ void rot16(double &re, double &im)
{
    constexpr int m = M & 15;
    if constexpr (m == 0)
        return;
    constexpr double C[16] = {1.0,
                              0.92387953251128675613,
                              0.70710678118654752440,
                              0.38268343236508977173,
                              0.0,
                              -0.38268343236508977173,
                              -0.70710678118654752440,
                              -0.92387953251128675613,
                              -1.0,
                              -0.92387953251128675613,
                              -0.70710678118654752440,
                              -0.38268343236508977173,
                              0.0,
                              0.38268343236508977173,
                              0.70710678118654752440,
                              0.92387953251128675613};
    // w16^m = cos(2 pi m / 16) - i sin(2 pi m / 16); sin(2 pi m / 16) = C[(m + 12) & 15]
    constexpr double c = C[m], s = INV ? -C[(m + 12) & 15] : C[(m + 12) & 15];
    // (re + i im)(c - i s)
    if constexpr (m == 4 || m == 12) { // -+i
        const double r = re;
        re = s * im;
        im = -s * r;
    } else if constexpr (m == 8) {
        re = -re;
        im = -im;
    } else {
        const double r = re * c + im * s;
        const double i = im * c - re * s;
        re = r;
        im = i;
    }
}

// DFT-4 over x[b], x[b + S], x[b + 2S], x[b + 3S] in place, natural order out.
template <int B, int S, bool INV>
__device__ __forceinline__ void dft4(double (&xr)[N], double (&xi)[N])
{
    const double t0r = xr[B] + xr[B + 2 * S], t0i = xi[B] + xi[B + 2 * S];
    const double t1r = xr[B] - xr[B + 2 * S], t1i = xi[B] - xi[B + 2 * S];
    const double t2r = xr[B + S] + xr[B + 3 * S], t2i = xi[B + S] + xi[B + 3 * S];
    const double t3r = xr[B + S] - xr[B + 3 * S], t3i = xi[B + S] - xi[B + 3 * S];
    xr[B] = t0r + t2r;
    xi[B] = t0i + t2i;
    xr[B + 2 * S] = t0r - t2r;
    xi[B + 2 * S] = t0i - t2i;
    // forward X1 = t1 - i t3, X3 = t1 + i t3; inverse swaps them
    if (!INV) {
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

template <int N2, int K1, bool INV>
__device__ __forceinline__ void tw(double (&xr)[N], double (&xi)[N])
{
    rot16<N2 * K1, INV>(xr[4 * K1 + N2], xi[4 * K1 + N2]);
}

// In-place DFT-16 of the line (xr, xi)[n]: X[k] = sum_n x[n] w16^(n k) (conjugate
// roots for the inverse), natural order out.  n = 4 n1 + n2, k = k1 + 4 k2: DFT-4
// over n1 for each n2 (result k1 lands in slot 4 k1 + n2), twiddle w16^(n2 k1),
// DFT-4 over n2 for each k1 (result k2 lands in slot 4 k1 + k2), then the 4 x 4
// index transpose is a renaming.
template <bool INV>
__device__ __forceinline__ void dft16(double (&xr)[N], double (&xi)[N])
{
    dft4<0, 4, INV>(xr, xi);
    dft4<1, 4, INV>(xr, xi);
    dft4<2, 4, INV>(xr, xi);
    dft4<3, 4, INV>(xr, xi);
    tw<1, 1, INV>(xr, xi);
    tw<2, 1, INV>(xr, xi);
    tw<3, 1, INV>(xr, xi);
    tw<1, 2, INV>(xr, xi);
    tw<2, 2, INV>(xr, xi);
    tw<3, 2, INV>(xr, xi);
    tw<1, 3, INV>(xr, xi);
    tw<2, 3, INV>(xr, xi);
    tw<3, 3, INV>(xr, xi);
    dft4<0, 1, INV>(xr, xi);
    dft4<4, 1, INV>(xr, xi);
    dft4<8, 1, INV>(xr, xi);
    dft4<12, 1, INV>(xr, xi);
    // slot 4 k1 + k2 holds X[k1 + 4 k2]: transpose the 4 x 4 index by renaming
    double yr[N], yi[N];
#pragma unroll
    for (int s = 0; s < N; ++s) {
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

// Column (y, x) of item `it` over z = 0..15 into registers: re from tile a, im from
// tile b; zeros outside a fixed-boundary grid, periodic wrap otherwise.  Thread
// (y, x) = (t >> 4, t & 15), so a warp reads two whole 128-byte rows per instruction;
// all loads are issued before the first use.
__device__ __forceinline__ void load_column(double (&re)[N], double (&im)[N], const TileWork &p,
                                            const dmma3d::Item &it, int y, int x)
{
    const bool inside = it.lz >= 0 && it.lz + N <= p.nz && it.ly >= 0 && it.ly + N <= p.ny && it.lx >= 0 &&
                        (it.has_b ? it.lxb + N : it.lx + N) <= p.nx;
    if (inside) { // the whole pair lies in the grid
        const int64_t plane = p.ny * p.nx;
        const double *base = p.in + (it.lz * p.ny + it.ly + y) * p.nx;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            re[k] = __ldcg(base + k * plane + it.lx + x);
            im[k] = it.has_b ? __ldcg(base + k * plane + it.lxb + x) : 0.0;
        }
        return;
    }
    int64_t gy = it.ly + y, ga = it.lx + x, gb = it.lxb + x;
    bool yok = gy >= 0 && gy < p.ny, aok = ga >= 0 && ga < p.nx, bok = it.has_b && gb >= 0 && gb < p.nx;
    if (p.periodic) {
        gy = wrap_near(gy, p.ny);
        ga = wrap_near(ga, p.nx);
        gb = wrap_near(gb, p.nx);
        yok = aok = true;
        bok = it.has_b;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        int64_t gz = it.lz + k;
        bool zok = gz >= 0 && gz < p.nz;
        if (p.periodic) {
            gz = wrap_near(gz, p.nz);
            zok = true;
        }
        const double *row = p.in + (gz * p.ny + gy) * p.nx;
        re[k] = (zok && yok && aok) ? __ldcg(row + ga) : 0.0;
        im[k] = (zok && yok && bok) ? __ldcg(row + gb) : 0.0;
    }
}

template <int CTAS>
__global__ void __launch_bounds__(NT, CTAS) fft3d_kernel(const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double2 *work = reinterpret_cast<double2 *>(smem);
    // CTAS = 3: the spectrum is read through L1; CTAS = 2: from a shared-memory copy
    const double2 *spec = CTAS == 3 ? p.spec : reinterpret_cast<const double2 *>(smem + WORK_BYTES);
    uint64_t *cbar = reinterpret_cast<uint64_t *>(smem + WORK_BYTES + SPEC_BYTES);

    const int t = threadIdx.x, hi = t >> 4, lo = t & 15;
    int64_t w = blockIdx.x;
    if (w >= p.nitems)
        return; // (the grid never exceeds the pair count; nothing was issued)
    bool spec_ready = CTAS == 3;
    if constexpr (CTAS == 2) {
        if (t == 0) { // the spectrum (needed from pass X on) arrives behind the first loads
            mbar_init(cbar, 1);
            fence_barrier_init();
            mbar_arrive_expect_tx(cbar, (uint32_t)SPEC_BYTES);
            bulk_load(reinterpret_cast<double2 *>(smem + WORK_BYTES), p.spec, (uint32_t)SPEC_BYTES, cbar);
        }
        __syncthreads();
    }
    const int u0 = p.halo, u1 = p.halo + p.useful; // wanted local positions per axis
    double xr[N], xi[N];
    for (; w < p.nitems; w += gridDim.x) {
        const dmma3d::Item it = dmma3d::item_of(p, w);
        { // Z: column (y, x) = (hi, lo) from global memory, forward along z
            load_column(xr, xi, p, it, hi, lo);
            dft16<false>(xr, xi);
#pragma unroll
            for (int i = 0; i < N; ++i)
                work[slot(i, hi, lo)] = make_double2(xr[i], xi[i]);
        }
        __syncthreads();
        { // Y: line (z, x) = (hi, lo), forward along y
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double2 v = work[slot(hi, i, lo)];
                xr[i] = v.x;
                xi[i] = v.y;
            }
            dft16<false>(xr, xi);
#pragma unroll
            for (int i = 0; i < N; ++i)
                work[slot(hi, i, lo)] = make_double2(xr[i], xi[i]);
        }
        __syncwarp(); // Y, X and Y' touch only plane z = hi, the 16 lanes of one half warp
        if (!spec_ready) {
            if (!mbar_wait_bounded(cbar, 0)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            spec_ready = true;
        }
        { // X: line (z, y) = (hi, lo): forward along x, spectrum, inverse along x
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double2 v = work[slot(hi, lo, i)];
                xr[i] = v.x;
                xi[i] = v.y;
            }
            dft16<false>(xr, xi);
            // frequency (kz, ky, kx) = (hi, lo, i) at spec[(kx * 16 + kz) * 16 + ky]; kx > 8 reads
            // conj S(16 - kx, -kz, -ky).  A warp's 32 lines read 32 consecutive entries (or two
            // reversed runs of 16) per kx: 16 sectors per load.
            const int direct = hi * N + lo, mirror = ((N - hi) & (N - 1)) * N + ((N - lo) & (N - 1));
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double2 *sp = i <= N / 2 ? spec + i * N * N + direct : spec + (N - i) * N * N + mirror;
                const double2 s = CTAS == 3 ? __ldg(sp) : *sp;
                cmul(xr[i], xi[i], s.x, i <= N / 2 ? s.y : -s.y);
            }
            dft16<true>(xr, xi);
#pragma unroll
            for (int i = 0; i < N; ++i)
                work[slot(hi, lo, i)] = make_double2(xr[i], xi[i]);
        }
        __syncwarp();
        if (lo >= u0 && lo < u1) { // Y': line (z, x) = (hi, lo) of a wanted x, inverse along y
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double2 v = work[slot(hi, i, lo)];
                xr[i] = v.x;
                xi[i] = v.y;
            }
            dft16<true>(xr, xi);
#pragma unroll
            for (int i = 0; i < N; ++i)
                work[slot(hi, i, lo)] = make_double2(xr[i], xi[i]);
        }
        __syncthreads();
        { // Z': column (y, x) = (hi, lo) when wanted, inverse along z, cropped stores
            const int64_t gy = it.ly + hi, ga = it.lx + lo, gb = it.lxb + lo;
            const bool a_ok = ga >= p.vlo[0] && ga < p.vhi[0];
            const bool b_ok = it.has_b && gb >= p.vlo[0] && gb < p.vhi[0];
            if (hi >= u0 && hi < u1 && gy >= p.vlo[1] && gy < p.vhi[1] && lo >= u0 && lo < u1 && (a_ok || b_ok)) {
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    const double2 v = work[slot(i, hi, lo)];
                    xr[i] = v.x;
                    xi[i] = v.y;
                }
                dft16<true>(xr, xi);
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    const int64_t gz = it.lz + i;
                    if (i < u0 || i >= u1 || gz < p.vlo[2] || gz >= p.vhi[2])
                        continue;
                    double *row = p.out + (gz * p.ny + gy) * p.nx;
                    if (a_ok)
                        row[ga] = xr[i];
                    if (b_ok)
                        row[gb] = xi[i];
                }
            }
        }
        // no barrier: the next pair's pass Z writes column (hi, lo) only, which this
        // thread alone has read in Z'
    }
}

} // namespace fft3d

size_t fft3d_smem_bytes() { return fft3d::smem_bytes<2>(); }

cudaError_t prepare_fft3d()
{
    cudaError_t e = cudaFuncSetAttribute(fft3d::fft3d_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fft3d::smem_bytes<3>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fft3d::fft3d_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)fft3d::smem_bytes<2>());
    return e;
}

// Three CTAs share each SM when the launch has at least 24 pairs per SM, else two.
int64_t fft3d_grid(int64_t nitems, int num_sms)
{
    const int per_sm = nitems >= fft3d::kThreeCtaPairsPerSm * num_sms ? 3 : 2;
    return std::min<int64_t>(nitems, (int64_t)per_sm * num_sms);
}

// `grid` is the SM count.
cudaError_t launch_fft3d(const TileWork &w, int grid, cudaStream_t s)
{
    const int64_t g = fft3d_grid(w.nitems, grid);
    if (w.nitems >= fft3d::kThreeCtaPairsPerSm * grid)
        fft3d::fft3d_kernel<3><<<(int)g, fft3d::NT, fft3d::smem_bytes<3>(), s>>>(w);
    else
        fft3d::fft3d_kernel<2><<<(int)g, fft3d::NT, fft3d::smem_bytes<2>(), s>>>(w);
    return cudaGetLastError();
}

} // namespace ffst
