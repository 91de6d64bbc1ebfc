// Radix-8 DFT-64 building blocks on FP64 mma.sync.m8n8k4 shared by the
// fused tile kernels (2D tiles, and the 64 x 64 four-step 1D tile).
//
// An 8x8 complex block is spread over a warp as the m8n8k4 fragments: the
// lane with g = lane>>2, t = lane&3 holds accumulator elements (g, 2t+e),
// e in {0,1}.  A DFT-64 of a line is two radix-8 stages; the second stage
// feeds the first stage's accumulators straight back as its A operand by
// permuting the contraction order of the DFT-8 matrix.
#pragma once
#include "ffs_device.cuh"

namespace ffst {
namespace r64 {

constexpr int N = 64;

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

struct NoHook {
    __device__ __forceinline__ void operator()(int, double[2], double[2]) const {}
};

// Forward DFT-64 along x of row y; output frequency k1 + 8*k2 at x-position 8*k1 + k2.
// `post(y, re, im)` may rescale the lane's two outputs (k1 = g, k2 = 2t + e) before the store.
struct WorkLoader { // element (y, x) of the swizzled complex work tile
    const double2 *work;
    __device__ __forceinline__ double2 operator()(int y, int x) const { return work[widx(y, x)]; }
    __device__ __forceinline__ WorkLoader work_or(const double2 *w) const { return WorkLoader{work ? work : w}; }
};

struct StageLoader { // element (y, x) of two dense 64 x 64 FP64 planes (TMA staging: re, im)
    const double *stage;
    __device__ __forceinline__ double2 operator()(int y, int x) const
    {
        return make_double2(stage[y * N + x], stage[N * N + y * N + x]);
    }
    __device__ __forceinline__ StageLoader work_or(const double2 *) const { return *this; }
};

// `load(y, x)` supplies the input element; the output always goes to `work`.
template <typename Post = NoHook, typename Load = WorkLoader>
__device__ __forceinline__ void row_forward(double2 *work, int y, const LaneConst &c, int g, int t,
                                            Post post = Post(), Load load = Load{nullptr})
{
    double bre[2], bim[2], d1re[2], d1im[2], d2re[2], d2im[2];
    const Load ld = load.work_or(work);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double2 v = ld(y, 8 * (t + 4 * j) + g);
        bre[j] = v.x;
        bim[j] = v.y;
    }
    stage_constA<false>(c, bre, bim, d1re, d1im);
    twiddle(c, d1re, d1im, false);
    stage_constB<false>(c, d1re, d1im, d2re, d2im);
    post(y, d2re, d2im);
    store_pair(work, g, d2re, d2im, [&](int e) { return widx(y, 8 * g + 2 * t + e); });
}

// Columns pa and pb (x-frequency positions), interleaved for independent DMMA chains:
// forward DFT-64 along y, multiply by the spectrum column, inverse DFT-64 along y,
// back in place in natural y order.
__device__ __forceinline__ void column_pass2(double2 *work, const double2 *spec, int pa, int pb, const LaneConst &c,
                                             int g, int t)
{
    double bre[2][2], bim[2][2], are[2][2], aim[2][2], dre[2][2], dim[2][2];
    const int px[2] = {pa, pb};
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const double2 v = work[widx(8 * (t + 4 * j) + g, px[q])];
            bre[q][j] = v.x;
            bim[q][j] = v.y;
        }
#pragma unroll
    for (int q = 0; q < 2; ++q)
        stage_constA<false>(c, bre[q], bim[q], are[q], aim[q]);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        twiddle(c, are[q], aim[q], false);
        stage_constB<false>(c, are[q], aim[q], dre[q], dim[q]);
    }
    const int e0 = g & 1;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const double2 s0 = spec[px[q] * N + 8 * g + 2 * t + e0];
        const double2 s1 = spec[px[q] * N + 8 * g + 2 * t + (e0 ^ 1)];
        const double sr0 = e0 ? s1.x : s0.x, si0 = e0 ? s1.y : s0.y;
        const double sr1 = e0 ? s0.x : s1.x, si1 = e0 ? s0.y : s1.y;
        cmul(dre[q][0], dim[q][0], sr0, si0);
        cmul(dre[q][1], dim[q][1], sr1, si1);
    }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        stage_constB<true>(c, dre[q], dim[q], are[q], aim[q]);
        twiddle(c, are[q], aim[q], true);
        store_pair(work, g, are[q], aim[q], [&](int e) { return widx(8 * g + 2 * t + e, px[q]); });
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const double2 v = work[widx(8 * (t + 4 * j) + g, px[q])];
            bre[q][j] = v.x;
            bim[q][j] = v.y;
        }
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        stage_constA<true>(c, bre[q], bim[q], dre[q], dim[q]);
        store_pair(work, g, dre[q], dim[q], [&](int e) { return widx(8 * g + 2 * t + e, px[q]); });
    }
}

// Inverse DFT-64 along x of row y; returns lane values at x = g + 8*(2t + e).
// Split in two so a caller can load every row before any row is overwritten.
__device__ __forceinline__ void row_inverse_load(const double2 *work, int y, int g, int t, double bre[2],
                                                 double bim[2])
{
#pragma unroll
    for (int j = 0; j < 2; ++j) { // frequency k1 + 8*k2 with k1 = g, k2 = t + 4j
        const double2 v = work[widx(y, 8 * g + t + 4 * j)];
        bre[j] = v.x;
        bim[j] = v.y;
    }
}

__device__ __forceinline__ void row_inverse_compute(const LaneConst &c, double bre[2], double bim[2], double ore[2],
                                                    double oim[2])
{
    double dre[2], dim[2];
    stage_constA<true>(c, bre, bim, dre, dim); // contract k2 -> a (rows a = g)
    twiddle(c, dre, dim, true);
    stage_constB<true>(c, dre, dim, ore, oim); // contract k1 -> b
}

__device__ __forceinline__ void row_inverse(const double2 *work, int y, const LaneConst &c, int g, int t,
                                            double ore[2], double oim[2])
{
    double bre[2], bim[2], dre[2], dim[2];
    row_inverse_load(work, y, g, t, bre, bim);
    stage_constA<true>(c, bre, bim, dre, dim); // contract k2 -> a (rows a = g)
    twiddle(c, dre, dim, true);
    stage_constB<true>(c, dre, dim, ore, oim); // contract k1 -> b
}

__device__ __forceinline__ LaneConst lane_consts(const double2 *f8, const double2 *w64, int g, int t)
{
    LaneConst c;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const double2 fa = f8[(g * (t + 4 * j)) & 7];
        const double2 fp = f8[((2 * t + j) * g) & 7];
        const double2 tw = w64[(g * (2 * t + j)) & 63];
        c.fa_re[j] = fa.x;
        c.fa_im[j] = fa.y;
        c.fa_nim[j] = -fa.y;
        c.fp_re[j] = fp.x;
        c.fp_im[j] = fp.y;
        c.fp_nim[j] = -fp.y;
        c.tw_re[j] = tw.x;
        c.tw_im[j] = tw.y;
    }
    return c;
}

} // namespace r64
} // namespace ffst
