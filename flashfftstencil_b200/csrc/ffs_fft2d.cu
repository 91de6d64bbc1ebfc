// FP64 fused DFT-tile stencil kernel for 2D grids on the FP64 pipe (radix-8
// butterflies, no tensor cores).
//
// On B200 an FP64 mma.sync.m8n8k4 runs at the rate of the plain FP64 FMA pipe
// (37.0 vs 36.8 TFLOP/s measured), so a DFT written as a dense GEMM pays for all
// of its 8 complex MACs per point and radix stage: 64 FMAs per point for a DFT-64.
// Butterflies compute the same DFT-64 in about 17 FP64 operations per point, and
// the kernel is then bound by shared-memory traffic instead.
//
// Tile 64 x 64 (same geometry and band as the DMMA form), two real tiles packed as
// one complex tile (re = left tile, im = right tile).  Per pair:
//   A. rows: forward DFT-64 along x of every row, read from the TMA staging planes;
//   B. columns: forward DFT-64 along y, multiply by spectrum^tau / 64^2, inverse
//      DFT-64 along y, all in registers;
//   C. rows: inverse DFT-64 along x of the wanted rows, cropped stores to global.
// Two work tiles let pass C of one pair run beside pass A of the next (C alone
// leaves the warps of the halo rows idle and the others latency-bound), so a pair
// costs two block barriers.  The spectrum is kept for kx = 0..32 only (Hermitian).
// Every DFT-64 is done by 8 threads (j = 0..7), each holding the 8 points 8a + j:
// a DFT-8 over a, the twiddle w64^(j k1), an 8 x 8 transpose through the line's
// own row or column of the work tile, a DFT-8 over j.  Thread k1 then holds
// frequency k1 + 8 k2 in register k2: natural order in, natural order out, so the
// inverse runs the same code with conjugate roots.
// Replaces rfft_2d_8_nwarp (src/2D/rfft_2d/2d_rfft_1_async.cu:17-364) like the
// DMMA form does; this form exists because the B200's FP64 tensor path has no
// throughput advantage over its FP64 FMA pipe.
#include <cstring>

#include "ffs_fft64.cuh"
#include "ffs_kernels.h"

namespace ffst {
namespace fft2d {

using namespace fft64;

constexpr int N = 64;
constexpr int NT = 512; // 64 groups of 8 threads: one line each per pass
constexpr size_t PLANE_BYTES = (size_t)N * N * sizeof(double);
constexpr size_t STAGE_BYTES = 2 * PLANE_BYTES;
constexpr size_t WORK_BYTES = (size_t)N * N * sizeof(double2);
constexpr int HALF = N / 2 + 1; // spectrum columns kx = 0..32
constexpr size_t SPEC_BYTES = (size_t)N * HALF * sizeof(double2);
constexpr size_t SMEM_BYTES = STAGE_BYTES + 2 * WORK_BYTES + SPEC_BYTES + 16;
static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");

// Staging plane (one real tile) as four TMA boxes of 16 x 64 doubles with the
// 128-byte swizzle: the 16-byte chunk (x & 15) >> 1 of row y moves to chunk
// ((x & 15) >> 1) ^ (y & 7) of that row's 128-byte line.
__device__ __forceinline__ int sidx(int y, int x)
{
    return ((x >> 4) << 10) | (y << 4) | (((((x >> 1) & 7) ^ (y & 7))) << 1) | (x & 1);
}

// Row of the tile that group q reads in pass A: the two groups of a half warp take
// rows r and r + 4, whose swizzled chunks are disjoint, so 8-byte staging reads are
// conflict-free.
__device__ __forceinline__ int row_a(int q) { return ((q >> 3) << 3) | ((q & 1) << 2) | ((q >> 1) & 3); }

struct Item {
    int64_t ly0, lxa, lxb;
    bool has_b;
};

__device__ __forceinline__ Item item_of(const TileWork &p, int64_t w)
{
    Item it;
    const int64_t pr = w % p.npx;
    const int64_t ty = p.t0[1] + w / p.npx, txa = p.t0[0] + 2 * pr;
    it.has_b = (2 * pr + 1) < p.nt[0];
    it.ly0 = ty * p.useful - p.halo;
    it.lxa = txa * p.useful - p.halo;
    it.lxb = it.lxa + p.useful;
    return it;
}

__device__ __forceinline__ bool tma_ok(const TileWork &p, const Item &it)
{
    if (!p.use_tma)
        return false;
    if (!p.periodic)
        return true; // out-of-range reads are zeros, only used by discarded cells
    const bool yin = it.ly0 >= 0 && it.ly0 + N <= p.ny;
    const bool ain = it.lxa >= 0 && it.lxa + N <= p.nx;
    const bool bin = !it.has_b || (it.lxb >= 0 && it.lxb + N <= p.nx);
    return yin && ain && bin;
}

// Plain (L1-bypassing) loads of item `it` into the staging planes, in the layout the
// TMA would have written; wraps periodically or reads zeros outside the grid.  Each
// thread issues all of its loads before its first store.
__device__ __forceinline__ void fill_plain(double *stage, const TileWork &p, const Item &it, int tid)
{
    constexpr int PER = N * N / NT;
    double re[PER], im[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        const int y = i >> 6, x = i & 63;
        int64_t gy = it.ly0 + y;
        const int64_t ga = it.lxa + x, gb = it.lxb + x;
        re[k] = 0.0;
        im[k] = 0.0;
        if (p.periodic) {
            gy = wrap_near(gy, p.ny);
            re[k] = __ldcg(p.in + gy * p.nx + wrap_near(ga, p.nx));
            if (it.has_b)
                im[k] = __ldcg(p.in + gy * p.nx + wrap_near(gb, p.nx));
        } else if (gy >= 0 && gy < p.ny) {
            if (ga >= 0 && ga < p.nx)
                re[k] = __ldcg(p.in + gy * p.nx + ga);
            if (it.has_b && gb >= 0 && gb < p.nx)
                im[k] = __ldcg(p.in + gy * p.nx + gb);
        }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        const int s = sidx(i >> 6, i & 63);
        stage[s] = re[k];
        stage[N * N + s] = im[k];
    }
}

// Pass A: forward along x of row row_a(q) of the staging planes into `work`.
__device__ __forceinline__ void pass_a(double2 *work, const double *stage, const Twiddle &tw, int q, int j,
                                       unsigned gmask)
{
    const int y = row_a(q);
    double xr[8], xi[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const int s = sidx(y, 8 * a + j);
        xr[a] = stage[s];
        xi[a] = stage[N * N + s];
    }
    auto slot = [&](int x) { return widx(y, x); };
    dft64_line<false>(xr, xi, tw, j, work, slot, gmask);
#pragma unroll
    for (int k = 0; k < 8; ++k)
        work[widx(y, j + 8 * k)] = make_double2(xr[k], xi[k]);
}

// Pass B: column kx = q: forward along y, spectrum, inverse along y.  Column kx > 32
// reads conj S(-ky, 64 - kx) from the stored half.
__device__ __forceinline__ void pass_b(double2 *work, const double2 *spec, const Twiddle &tw, int q, int j,
                                       unsigned gmask)
{
    const int c = q;
    const bool upper = c > N / 2;
    const int sx = upper ? N - c : c;
    auto slot = [&](int y) { return widx(y, c); };
    double xr[8], xi[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const double2 v = work[widx(8 * a + j, c)];
        xr[a] = v.x;
        xi[a] = v.y;
    }
    dft64_line<false>(xr, xi, tw, j, work, slot, gmask);
#pragma unroll
    for (int k = 0; k < 8; ++k) { // frequency (ky = j + 8 k, kx = c)
        const int ky = j + 8 * k;
        const double2 s = spec[(upper ? (N - ky) & (N - 1) : ky) * HALF + sx];
        cmul(xr[k], xi[k], s.x, upper ? -s.y : s.y);
    }
    dft64_line<true>(xr, xi, tw, j, work, slot, gmask);
#pragma unroll
    for (int k = 0; k < 8; ++k)
        work[widx(j + 8 * k, c)] = make_double2(xr[k], xi[k]);
}

// Pass C: inverse along x of row q of `work` when it is wanted; cropped stores.
__device__ __forceinline__ void pass_c(double2 *work, const TileWork &p, const Item &it, const Twiddle &tw, int q,
                                       int j, unsigned gmask)
{
    const int y = q;
    const int64_t gy = it.ly0 + y;
    if (y < p.halo || y >= p.halo + p.useful || gy < p.vlo[1] || gy >= p.vhi[1])
        return;
    double xr[8], xi[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const double2 v = work[widx(y, 8 * a + j)];
        xr[a] = v.x;
        xi[a] = v.y;
    }
    auto slot = [&](int x) { return widx(y, x); };
    dft64_line<true>(xr, xi, tw, j, work, slot, gmask);
    double *row = p.out + gy * p.nx;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int x = j + 8 * k;
        if (x < p.halo || x >= p.halo + p.useful)
            continue;
        const int64_t ga = it.lxa + x, gb = it.lxb + x;
        if (ga >= p.vlo[0] && ga < p.vhi[0])
            row[ga] = xr[k];
        if (it.has_b && gb >= p.vlo[0] && gb < p.vhi[0])
            row[gb] = xi[k];
    }
}

__global__ void __launch_bounds__(NT, 1) fft2d_kernel(const __grid_constant__ CUtensorMap tmap, const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double *stage = reinterpret_cast<double *>(smem);
    double2 *work0 = reinterpret_cast<double2 *>(smem + STAGE_BYTES);
    double2 *spec = reinterpret_cast<double2 *>(smem + STAGE_BYTES + 2 * WORK_BYTES);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES + 2 * WORK_BYTES + SPEC_BYTES);
    uint64_t *cbar = bar + 1; // the spectrum

    const int tid = threadIdx.x, q = tid >> 3, j = tid & 7;
    const unsigned gmask = 0xffu << (tid & 24);
    Twiddle tw;
    {
        const double2 *w64 = p.tables + 8; // w64[m] = exp(-2 pi i m / 64)
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const double2 v = w64[(j * k) & 63];
            tw.re[k] = v.x;
            tw.im[k] = v.y;
        }
    }
    auto issue = [&](const Item &it) {
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(bar, (uint32_t)STAGE_BYTES);
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            tma_load_2d(stage + b * 1024, &tmap, bar, (int)it.lxa + 16 * b, (int)it.ly0);
            tma_load_2d(stage + N * N + b * 1024, &tmap, bar, (int)it.lxb + 16 * b, (int)it.ly0);
        }
    };
    int64_t w = blockIdx.x;
    if (w >= p.nitems)
        return; // (the grid never exceeds the pair count; nothing was issued)
    // the first pair's tiles, then the spectrum (needed from pass B on), by async copies
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(cbar, 1);
        fence_barrier_init();
        const Item it = item_of(p, w);
        if (tma_ok(p, it))
            issue(it);
        mbar_arrive_expect_tx(cbar, (uint32_t)SPEC_BYTES);
        bulk_load(spec, p.spec, (uint32_t)SPEC_BYTES, cbar);
    }
    __syncthreads();

    uint32_t phase = 0;
    // stage the pair (TMA already issued, or plain loads); every thread returns ok
    auto staged = [&](const Item &it) -> bool {
        if (tma_ok(p, it)) {
            if (!mbar_wait_bounded(bar, phase))
                return false;
            phase ^= 1;
        } else {
            fill_plain(stage, p, it, tid);
            __syncthreads();
        }
        return true;
    };
    bool spec_ready = false;
    // a wait ran out: record it, and let the spectrum copy (if still pending) land
    // before the CTA exits
    auto fail = [&]() {
        record_error(p.status, kDevTimeoutTma);
        if (!spec_ready)
            (void)mbar_wait_bounded(cbar, 0);
    };
    Item it = item_of(p, w);
    if (!staged(it)) {
        fail();
        return;
    }
    pass_a(work0, stage, tw, q, j, gmask);
    for (int buf = 0;; buf ^= 1) {
        double2 *work = work0 + buf * (N * N);
        const int64_t wn = w + gridDim.x;
        __syncthreads(); // pass A of pair w done: staging planes free, rows complete
        if (tid == 0 && wn < p.nitems) {
            const Item nx_it = item_of(p, wn);
            if (tma_ok(p, nx_it))
                issue(nx_it);
        }
        if (!spec_ready) {
            if (!mbar_wait_bounded(cbar, 0)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            spec_ready = true;
        }
        pass_b(work, spec, tw, q, j, gmask);
        __syncthreads(); // columns complete
        pass_c(work, p, it, tw, q, j, gmask);
        if (wn >= p.nitems)
            break;
        // pass A of the next pair into the other work tile, beside this pair's pass C
        const Item nx = item_of(p, wn);
        if (!staged(nx)) {
            fail();
            return;
        }
        pass_a(work0 + (buf ^ 1) * (N * N), stage, tw, q, j, gmask);
        it = nx;
        w = wn;
    }
}

} // namespace fft2d

size_t fft2d_smem_bytes() { return fft2d::SMEM_BYTES; }

cudaError_t prepare_fft2d()
{
    return cudaFuncSetAttribute(fft2d::fft2d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fft2d::SMEM_BYTES);
}

cudaError_t launch_fft2d(const CUtensorMap *tmap, const TileWork &w, int grid, cudaStream_t s)
{
    CUtensorMap dummy;
    if (!tmap) {
        memset(&dummy, 0, sizeof(dummy));
        tmap = &dummy;
    }
    fft2d::fft2d_kernel<<<grid, fft2d::NT, fft2d::SMEM_BYTES, s>>>(*tmap, w);
    return cudaGetLastError();
}

} // namespace ffst
