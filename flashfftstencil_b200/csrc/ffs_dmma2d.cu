// FP64 fused DFT-tile stencil kernel for 2D grids (plain form, DMMA).
//
// One persistent CTA per SM walks tile pairs.  Per pair:
//   1. TMA (cp.async.bulk.tensor.2d, no multicast) stages two 64x64 FP64 halo
//      tiles of the natural row-major grid into shared memory; out-of-range
//      coordinates read zeros.  The next pair is prefetched while this one computes.
//   2. The two real tiles are interleaved into one complex tile (re = left tile,
//      im = right tile) in a swizzled layout that keeps every fragment access
//      below conflict-free for 128-bit shared loads/stores.
//   3. Forward 2D DFT-64x64: each 64-point DFT is two radix-8 stages, each an
//      8x8x8 complex product on mma.sync.m8n8k4.f64, with the 64th-root twiddle
//      applied in registers between them.  The second stage takes its A operand
//      straight from the first stage's accumulators by permuting the contraction
//      order of the DFT-8 matrix (the fragment-reuse idea of the reference,
//      src/2D/rfft_2d/2d_rfft_2.cu:113-116 with src/2D/create_fft_pfa_plan.cu:29).
//   4. Pointwise multiply by spectrum^tau / 64^2 (FP64, prepared on the host).
//   5. Inverse DFT, crop of the halo, direct store of the u x u interior.
// This replaces rfft_2d_8_nwarp (src/2D/rfft_2d/2d_rfft_1_async.cu:17-364): the
// reference uses 8x8 tiles, one step per launch and atomic overlap-add; here a
// tile carries tau fused steps and every output cell is written exactly once.
#include <cstring>

#include "ffs_device.cuh"
#include "ffs_kernels.h"

namespace ffst {
namespace dmma2d {

constexpr int N = 64;
constexpr int NT = 512;
constexpr int NWARP = NT / 32;
constexpr size_t STAGE_BYTES = 2ull * N * N * sizeof(double); // two dense TMA boxes
constexpr size_t WORK_BYTES = (size_t)N * N * sizeof(double2);
constexpr size_t SPEC_BYTES = (size_t)N * N * sizeof(double2);
constexpr size_t SMEM_BYTES = STAGE_BYTES + WORK_BYTES + SPEC_BYTES + 16;

// XOR swizzle of the complex work tile.  Element (y, x) lives at
// y*64 + (x ^ S(x>>3) ^ (y&7) ^ S(y>>3)); S bit-reverses the low two bits of
// the digit and doubles it.  With it, all eight access patterns used below
// (row/column x forward/inverse x load/store) touch eight distinct 16-byte
// bank groups per quarter warp.
__device__ __forceinline__ int S3(int h) { return ((h & 1) << 2) | (h & 2); }
__device__ __forceinline__ int widx(int y, int x) { return y * N + (x ^ (S3(x >> 3) ^ (y & 7) ^ S3(y >> 3))); }

struct LaneConst {
    double fa_re[2], fa_im[2], fa_nim[2]; // DFT-8[g][t + 4j]            (A operand)
    double fp_re[2], fp_im[2], fp_nim[2]; // DFT-8[2t + j][g]            (B operand, permuted k)
    double tw_re[2], tw_im[2];            // w64^(g * (2t + e))          (twiddles)
};

// D = A(const DFT-8, from registers) x B(data).  CONJ uses conj(A).
template <bool CONJ>
__device__ __forceinline__ void stage_constA(const LaneConst &c, const double bre[2], const double bim[2],
                                             double dre[2], double dim[2])
{
    dre[0] = dre[1] = dim[0] = dim[1] = 0.0;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double ai = CONJ ? c.fa_nim[j] : c.fa_im[j];
        const double nai = CONJ ? c.fa_im[j] : c.fa_nim[j];
        dmma(dre[0], dre[1], c.fa_re[j], bre[j]);
        dmma(dre[0], dre[1], nai, bim[j]);
        dmma(dim[0], dim[1], c.fa_re[j], bim[j]);
        dmma(dim[0], dim[1], ai, bre[j]);
    }
}

// D = A(data, k-step j = accumulator column 2t+j) x B(const permuted DFT-8).
template <bool CONJ>
__device__ __forceinline__ void stage_constB(const LaneConst &c, const double are[2], const double aim[2],
                                             double dre[2], double dim[2])
{
    dre[0] = dre[1] = dim[0] = dim[1] = 0.0;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double bi = CONJ ? c.fp_nim[j] : c.fp_im[j];
        const double nbi = CONJ ? c.fp_im[j] : c.fp_nim[j];
        dmma(dre[0], dre[1], are[j], c.fp_re[j]);
        dmma(dre[0], dre[1], aim[j], nbi);
        dmma(dim[0], dim[1], are[j], bi);
        dmma(dim[0], dim[1], aim[j], c.fp_re[j]);
    }
}

__device__ __forceinline__ void twiddle(const LaneConst &c, double re[2], double im[2], bool conj)
{
#pragma unroll
    for (int e = 0; e < 2; ++e)
        cmul(re[e], im[e], c.tw_re[e], conj ? -c.tw_im[e] : c.tw_im[e]);
}

// Store the two accumulator columns (2t, 2t+1) of an 8x8 block whose element
// (row g, col 2t+e) lands at index idx(e); the lane with odd g stores e=1 first
// so that each store instruction hits eight distinct bank groups.
template <typename IdxFn>
__device__ __forceinline__ void store_pair(double2 *buf, int g, const double re[2], const double im[2], IdxFn idx)
{
    const int e0 = g & 1;
    const double r0 = e0 ? re[1] : re[0], i0 = e0 ? im[1] : im[0];
    const double r1 = e0 ? re[0] : re[1], i1 = e0 ? im[0] : im[1];
    buf[idx(e0)] = make_double2(r0, i0);
    buf[idx(e0 ^ 1)] = make_double2(r1, i1);
}

// Forward DFT-64 along x of row y; output frequency k1 + 8*k2 at x-position 8*k1 + k2.
__device__ __forceinline__ void row_forward(double2 *work, int y, const LaneConst &c, int g, int t)
{
    double bre[2], bim[2], d1re[2], d1im[2], d2re[2], d2im[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double2 v = work[widx(y, 8 * (t + 4 * j) + g)];
        bre[j] = v.x;
        bim[j] = v.y;
    }
    stage_constA<false>(c, bre, bim, d1re, d1im);
    twiddle(c, d1re, d1im, false);
    stage_constB<false>(c, d1re, d1im, d2re, d2im);
    store_pair(work, g, d2re, d2im, [&](int e) { return widx(y, 8 * g + 2 * t + e); });
}

// Column px (an x-frequency position): forward DFT-64 along y, multiply by the
// spectrum column, inverse DFT-64 along y, back in place in natural y order.
__device__ __forceinline__ void column_pass(double2 *work, const double2 *spec, int px, const LaneConst &c, int g,
                                            int t)
{
    double bre[2], bim[2], are[2], aim[2], dre[2], dim[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double2 v = work[widx(8 * (t + 4 * j) + g, px)];
        bre[j] = v.x;
        bim[j] = v.y;
    }
    stage_constA<false>(c, bre, bim, are, aim);
    twiddle(c, are, aim, false);
    stage_constB<false>(c, are, aim, dre, dim);
    {   // spectrum (position 8*k1 + k2 along y), loaded in bank-friendly order
        const int e0 = g & 1;
        const double2 s0 = spec[px * N + 8 * g + 2 * t + e0];
        const double2 s1 = spec[px * N + 8 * g + 2 * t + (e0 ^ 1)];
        const double sr0 = e0 ? s1.x : s0.x, si0 = e0 ? s1.y : s0.y;
        const double sr1 = e0 ? s0.x : s1.x, si1 = e0 ? s0.y : s1.y;
        cmul(dre[0], dim[0], sr0, si0);
        cmul(dre[1], dim[1], sr1, si1);
    }
    stage_constB<true>(c, dre, dim, are, aim); // contract k2 -> a
    twiddle(c, are, aim, true);
    store_pair(work, g, are, aim, [&](int e) { return widx(8 * g + 2 * t + e, px); });
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double2 v = work[widx(8 * (t + 4 * j) + g, px)];
        bre[j] = v.x;
        bim[j] = v.y;
    }
    stage_constA<true>(c, bre, bim, dre, dim); // contract k1 -> b; y = a + 8b
    store_pair(work, g, dre, dim, [&](int e) { return widx(8 * g + 2 * t + e, px); });
}

// Inverse DFT-64 along x of row y; returns lane values at x = g + 8*(2t + e).
__device__ __forceinline__ void row_inverse(const double2 *work, int y, const LaneConst &c, int g, int t,
                                            double ore[2], double oim[2])
{
    double bre[2], bim[2], dre[2], dim[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double2 v = work[widx(y, 8 * g + t + 4 * j)];
        bre[j] = v.x;
        bim[j] = v.y;
    }
    stage_constA<true>(c, bre, bim, dre, dim); // contract k2 -> a (rows a = g)
    twiddle(c, dre, dim, true);
    stage_constB<true>(c, dre, dim, ore, oim); // contract k1 -> b
}

struct Item {
    int64_t ty, txa;
    int64_t ly0, lxa, lxb;
    bool has_b;
};

__device__ __forceinline__ Item item_of(const TileWork &p, int64_t w)
{
    Item it;
    const int64_t pr = w % p.npx;
    it.ty = p.t0[1] + w / p.npx;
    it.txa = p.t0[0] + 2 * pr;
    it.has_b = (2 * pr + 1) < p.nt[0];
    it.ly0 = it.ty * p.useful - p.halo;
    it.lxa = it.txa * p.useful - p.halo;
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

__device__ __forceinline__ int64_t wrapi(int64_t i, int64_t n)
{
    i %= n;
    return i < 0 ? i + n : i;
}

__global__ void __launch_bounds__(NT, 1) dmma2d_kernel(const __grid_constant__ CUtensorMap tmap, const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double *stage = reinterpret_cast<double *>(smem);
    double2 *work = reinterpret_cast<double2 *>(smem + STAGE_BYTES);
    double2 *spec = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    for (int i = tid; i < N * N; i += NT)
        spec[i] = p.spec[i];
    LaneConst c;
    {
        const double2 *f8 = p.tables, *w64 = p.tables + 8;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const double2 fa = f8[(g * (t + 4 * j)) & 7];
            const double2 fp = f8[((2 * t + j) * g) & 7];
            const double2 tw = w64[(g * (2 * t + j)) & 63];
            c.fa_re[j] = fa.x; c.fa_im[j] = fa.y; c.fa_nim[j] = -fa.y;
            c.fp_re[j] = fp.x; c.fp_im[j] = fp.y; c.fp_nim[j] = -fp.y;
            c.tw_re[j] = tw.x; c.tw_im[j] = tw.y;
        }
    }
    __syncthreads();

    auto issue = [&](const Item &it) {
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(bar, (uint32_t)STAGE_BYTES);
        tma_load_2d(stage, &tmap, bar, (int)it.lxa, (int)it.ly0);
        tma_load_2d(stage + N * N, &tmap, bar, (int)it.lxb, (int)it.ly0);
    };

    uint32_t phase = 0;
    int64_t w = blockIdx.x;
    if (tid == 0 && w < p.nitems) {
        const Item it = item_of(p, w);
        if (tma_ok(p, it))
            issue(it);
    }
    for (; w < p.nitems; w += gridDim.x) {
        const Item it = item_of(p, w);
        if (tma_ok(p, it)) {
            if (!mbar_wait_bounded(bar, phase)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            phase ^= 1;
            for (int i = tid; i < N * N; i += NT) {
                const int y = i >> 6, x = i & 63;
                work[widx(y, x)] = make_double2(stage[i], stage[N * N + i]);
            }
        } else {
            for (int i = tid; i < N * N; i += NT) {
                const int y = i >> 6, x = i & 63;
                int64_t gy = it.ly0 + y, ga = it.lxa + x, gb = it.lxb + x;
                double re = 0.0, im = 0.0;
                if (p.periodic) {
                    gy = wrapi(gy, p.ny);
                    re = p.in[gy * p.nx + wrapi(ga, p.nx)];
                    if (it.has_b)
                        im = p.in[gy * p.nx + wrapi(gb, p.nx)];
                } else if (gy >= 0 && gy < p.ny) {
                    if (ga >= 0 && ga < p.nx)
                        re = p.in[gy * p.nx + ga];
                    if (it.has_b && gb >= 0 && gb < p.nx)
                        im = p.in[gy * p.nx + gb];
                }
                work[widx(y, x)] = make_double2(re, im);
            }
        }
        __syncthreads();
        if (tid == 0 && w + gridDim.x < p.nitems) {
            const Item nx_it = item_of(p, w + gridDim.x);
            if (tma_ok(p, nx_it))
                issue(nx_it);
        }
        // forward DFT along x, every row
#pragma unroll 1
        for (int k = 0; k < N / NWARP; k += 2) {
            row_forward(work, warp + NWARP * k, c, g, t);
            row_forward(work, warp + NWARP * (k + 1), c, g, t);
        }
        __syncthreads();
#pragma unroll 1
        for (int k = 0; k < N / NWARP; ++k)
            column_pass(work, spec, warp + NWARP * k, c, g, t);
        __syncthreads();
        // inverse DFT along x and cropped store of the interior rows
#pragma unroll 1
        for (int k = 0; k < N / NWARP; ++k) {
            const int y = warp + NWARP * k;
            const int64_t gy = it.ly0 + y;
            if (y < p.halo || y >= p.halo + p.useful || gy < p.vlo[1] || gy >= p.vhi[1])
                continue;
            double ore[2], oim[2];
            row_inverse(work, y, c, g, t, ore, oim);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int x = g + 8 * (2 * t + e);
                if (x < p.halo || x >= p.halo + p.useful)
                    continue;
                const int64_t ga = it.lxa + x, gb = it.lxb + x;
                if (ga >= p.vlo[0] && ga < p.vhi[0])
                    p.out[gy * p.nx + ga] = ore[e];
                if (it.has_b && gb >= p.vlo[0] && gb < p.vhi[0])
                    p.out[gy * p.nx + gb] = oim[e];
            }
        }
        __syncthreads();
    }
}

} // namespace dmma2d

size_t dmma2d_smem_bytes() { return dmma2d::SMEM_BYTES; }
int dmma2d_tile() { return dmma2d::N; }

cudaError_t prepare_dmma2d()
{
    return cudaFuncSetAttribute(dmma2d::dmma2d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dmma2d::SMEM_BYTES);
}

cudaError_t launch_dmma2d(const CUtensorMap *tmap, const TileWork &w, int grid, cudaStream_t s)
{
    CUtensorMap dummy;
    if (!tmap) {
        memset(&dummy, 0, sizeof(dummy));
        tmap = &dummy;
    }
    dmma2d::dmma2d_kernel<<<grid, dmma2d::NT, dmma2d::SMEM_BYTES, s>>>(*tmap, w);
    return cudaGetLastError();
}

} // namespace ffst
