// 3D FP64-DMMA fused tile (16^3): per-item device functions shared by the
// persistent 3D kernel (ffs_dmma3d.cu) and the batched kernel.
//
// A DFT-16 along one axis is ONE pass over the tile, entirely in registers:
// position x = 4 x1 + x0, frequency k = f1 + 4 f0, and per pair of lines (r = 0, 1)
//   stage 1: Y[f1][x0, r] = sum_x1 X[4 x1 + x0, r] w4^(f1 x1)    (contract x1)
//   twiddle: Y *= w16^(f1 x0)
//   stage 2: Z[f0][f1, r] = sum_x0 Y[f1][x0, r] w4^(f0 x0)       (contract x0)
// Each stage is a real-block product [[Re F4, -Im F4], [Im F4, Re F4]] . [Xr; Xi]
// = two mma.sync.m8n8k4.f64 over 8 columns.  Stage 1's columns are (x0, r); after
// a lane-xor-16 shuffle that pairs real and imaginary rows, lane (g, t) holds the
// complex Y[f1 = g & 3][x0 = t, r = g >> 2] -- which is exactly stage 2's B
// fragment (k = x0 = t, column 4 r + f1 = g), so the two stages need no data
// movement between them; the twiddle is a per-lane constant.  Every element is
// read and written once per axis (the previous design, one radix-4 stage per
// pass, went through shared memory twice per axis).  Frequencies are stored in
// natural order, so the inverse pass is the same code with conjugate constants
// and the spectrum is natural (kz, ky, kx).
#pragma once
#include "ffs_device.cuh"
#include "ffs_kernels.h"

namespace ffst {
namespace dmma3d {

constexpr int N = 16;
constexpr int VOL = N * N * N;
constexpr int NT = 512;
constexpr size_t STAGE_BYTES = 2ull * VOL * sizeof(double);
constexpr size_t WORK_BYTES = (size_t)VOL * sizeof(double2);
constexpr size_t SPEC_BYTES = (size_t)VOL * sizeof(double2);
constexpr size_t SMEM_BYTES = STAGE_BYTES + WORK_BYTES + SPEC_BYTES + 16;

// Swizzle of the complex work tile, element e = 256 z + 16 y + x: XOR into the
// low three bits of x the bits (y0, x3 ^ y2 ^ z2, y1 ^ y3 ^ z1 ^ z3).  For every
// pass's load (position bits 2, 3 and the line bit r) and store (position bits
// 1, 2 and r) each quarter warp touches 8 distinct 16-byte bank groups, and the
// map is linear over GF(2): an address is a per-lane constant XOR a constant of
// the unrolled iteration.
__host__ __device__ constexpr int sw3(int e)
{
    const int h0 = (e >> 4) & 1;
    const int h1 = ((e >> 3) ^ (e >> 6) ^ (e >> 10)) & 1;
    const int h2 = ((e >> 5) ^ (e >> 7) ^ (e >> 9) ^ (e >> 11)) & 1;
    return e ^ (h0 | (h1 << 1) | (h2 << 2));
}

// Where TMA (128-byte swizzle, 16-double rows) puts element e of a staged real
// tile: the 16-byte chunk x >> 1 of row e >> 4 moves to chunk (x >> 1) ^ (row & 7).
// Also linear; the first pass's 8-byte loads hit 16 distinct slots per half warp.
__host__ __device__ constexpr int stage_idx(int e)
{
    return (e & ~15) | (((((e & 15) >> 1) ^ ((e >> 4) & 7)) << 1) | (e & 1));
}

struct Consts {
    double f0, f1;   // forward real-block DFT-4, lane (row g, k-col t) for the re and im k-steps
    double i0, i1;   // inverse (conjugate) real-block DFT-4
    double twr, twi; // forward twiddle w16^((g & 3) t) between the two stages
};

// tables[k] = w16^k.  Row g < 4 of the real-block DFT-4 is Re out f = g, else Im out f = g - 4.
__device__ __forceinline__ Consts make_consts(const double2 *tables, int g, int t)
{
    Consts c;
    const int k1 = g & 3;
    const double2 f = tables[(4 * k1 * t) & 15];
    const bool re_row = g < 4;
    c.f0 = re_row ? f.x : f.y;  // multiplies Xr[x1 = t]
    c.f1 = re_row ? -f.y : f.x; // multiplies Xi[x1 = t]
    c.i0 = re_row ? f.x : -f.y; // conjugate
    c.i1 = re_row ? f.y : f.x;
    const double2 w = tables[(k1 * t) & 15];
    c.twr = w.x;
    c.twi = w.y;
    return c;
}

enum Axis { kX = 0, kY = 1, kZ = 2 };
enum Src { kFromWork = 0, kFromStage = 1 };

// Element of line pair `it` (lines 2 it + r) at `pos` along the axis, in plane w
// (z-plane for the x and y passes, y-plane for the z pass).
template <int AX>
__host__ __device__ constexpr int elem(int w, int it, int pos, int r)
{
    return AX == kX ? (w << 8) | ((2 * it + r) << 4) | pos
                    : (AX == kY ? (w << 8) | (pos << 4) | (2 * it + r) : (pos << 8) | (w << 4) | (2 * it + r));
}

struct Item {
    int64_t lx, ly, lz, lxb;
    bool has_b;
};

__device__ __forceinline__ Item item_of(const TileWork &p, int64_t w)
{
    Item it;
    const int64_t pr = w % p.npx, rest = w / p.npx;
    const int64_t tx = p.t0[0] + 2 * pr, ty = p.t0[1] + rest % p.nt[1], tz = p.t0[2] + rest / p.nt[1];
    it.has_b = (2 * pr + 1) < p.nt[0];
    it.lx = tx * p.useful - p.halo;
    it.ly = ty * p.useful - p.halo;
    it.lz = tz * p.useful - p.halo;
    it.lxb = it.lx + p.useful;
    return it;
}

// Both DFT-16 stages of one direction on a batch of pairs held in registers.
template <int B>
__device__ __forceinline__ void dft16_regs(double (&re)[B], double (&im)[B], double a0, double a1, double twr,
                                           double twi, bool lo)
{
#pragma unroll
    for (int b = 0; b < B; ++b) {
        double d0 = 0.0, d1 = 0.0;
        dmma(d0, d1, a0, re[b]);
        dmma(d0, d1, a1, im[b]);
        double recv = __shfl_xor_sync(0xffffffffu, lo ? d1 : d0, 16);
        double xr = lo ? d0 : recv, xi = lo ? recv : d1;
        cmul(xr, xi, twr, twi);
        d0 = 0.0;
        d1 = 0.0;
        dmma(d0, d1, a0, xr);
        dmma(d0, d1, a1, xi);
        recv = __shfl_xor_sync(0xffffffffu, lo ? d1 : d0, 16);
        re[b] = lo ? d0 : recv;
        im[b] = lo ? recv : d1;
    }
}

// One DFT-16 pass along AX over the warp's 8 line pairs (4 in flight).  SRC: the
// swizzled work tile, or the two TMA-staged real tiles.  OUT: store the cropped
// interior to global memory (re -> tile a, im -> tile b) instead of writing back to
// the work tile.
template <int AX, bool INV, int SRC, bool OUT>
__device__ __forceinline__ void pass16(double2 *work, const double *stage, int w, const Consts &c, int g, int t,
                                       const TileWork &p, const Item &itm)
{
    constexpr int B = 4;
    const bool lo = g < 4;
    const int el = elem<AX>(w, 0, 4 * t + (g >> 1), g & 1);
    const int es = elem<AX>(w, 0, 2 * (t & 1) + (g >> 2) + 4 * (g & 3), t >> 1);
    const int lds = SRC == kFromStage ? stage_idx(el) : sw3(el);
    const int sts = sw3(es);
#pragma unroll
    for (int it0 = 0; it0 < 8; it0 += B) {
        double re[B], im[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int ei = elem<AX>(0, it0 + b, 0, 0);
            if constexpr (SRC == kFromStage) {
                const int k = lds ^ stage_idx(ei);
                re[b] = stage[k];
                im[b] = stage[VOL + k];
            } else {
                const double2 v = work[lds ^ sw3(ei)];
                re[b] = v.x;
                im[b] = v.y;
            }
        }
        if constexpr (INV)
            dft16_regs<B>(re, im, c.i0, c.i1, c.twr, -c.twi, lo);
        else
            dft16_regs<B>(re, im, c.f0, c.f1, c.twr, c.twi, lo);
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int ei = elem<AX>(0, it0 + b, 0, 0);
            if constexpr (OUT) { // x pass on z-plane w: element (w, y, x)
                const int e = es ^ ei;
                const int x = e & 15, y = (e >> 4) & 15;
                const int64_t gz = itm.lz + w, gy = itm.ly + y;
                if (y < p.halo || y >= p.halo + p.useful || gy < p.vlo[1] || gy >= p.vhi[1] || x < p.halo ||
                    x >= p.halo + p.useful)
                    continue;
                const int64_t row = (gz * p.ny + gy) * p.nx;
                const int64_t ga = itm.lx + x, gb = itm.lxb + x;
                if (ga >= p.vlo[0] && ga < p.vhi[0])
                    p.out[row + ga] = re[b];
                if (itm.has_b && gb >= p.vlo[0] && gb < p.vhi[0])
                    p.out[row + gb] = im[b];
            } else {
                work[sts ^ sw3(ei)] = make_double2(re[b], im[b]);
            }
        }
    }
}

// Forward z, spectrum, inverse z on the warp's y-plane w without a trip through
// shared memory: a pass leaves lane (g, t) holding position 2 (t & 1) + (g >> 2) +
// 4 (g & 3) of line t >> 1 and takes position 4 t + (g >> 1) of line g & 1, so one
// shuffle from lane 4 (t + 4 ((g >> 1) & 1)) + (g >> 2) + 2 (g & 1) turns the
// forward output into the inverse input.
__device__ __forceinline__ void pass16_z_round_trip(double2 *work, const double2 *spec, int w, const Consts &c,
                                                    int g, int t)
{
    constexpr int B = 4;
    const bool lo = g < 4;
    const int lds = sw3(elem<kZ>(w, 0, 4 * t + (g >> 1), g & 1));
    const int sts = sw3(elem<kZ>(w, 0, 2 * (t & 1) + (g >> 2) + 4 * (g & 3), t >> 1));
    const int src = 4 * (t + 4 * ((g >> 1) & 1)) + (g >> 2) + 2 * (g & 1);
#pragma unroll
    for (int it0 = 0; it0 < 8; it0 += B) {
        double re[B], im[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const double2 v = work[lds ^ sw3(elem<kZ>(0, it0 + b, 0, 0))];
            re[b] = v.x;
            im[b] = v.y;
        }
        dft16_regs<B>(re, im, c.f0, c.f1, c.twr, c.twi, lo);
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const double2 s = spec[sts ^ sw3(elem<kZ>(0, it0 + b, 0, 0))];
            cmul(re[b], im[b], s.x, s.y);
            re[b] = __shfl_sync(0xffffffffu, re[b], src);
            im[b] = __shfl_sync(0xffffffffu, im[b], src);
        }
        dft16_regs<B>(re, im, c.i0, c.i1, c.twr, -c.twi, lo);
#pragma unroll
        for (int b = 0; b < B; ++b)
            work[sts ^ sw3(elem<kZ>(0, it0 + b, 0, 0))] = make_double2(re[b], im[b]);
    }
}

__device__ __forceinline__ bool tma_ok(const TileWork &p, const Item &it)
{
    if (!p.use_tma)
        return false;
    if (!p.periodic)
        return true;
    const bool zin = it.lz >= 0 && it.lz + N <= p.nz, yin = it.ly >= 0 && it.ly + N <= p.ny;
    const bool ain = it.lx >= 0 && it.lx + N <= p.nx;
    const bool bin = !it.has_b || (it.lxb >= 0 && it.lxb + N <= p.nx);
    return zin && yin && ain && bin;
}

// Plain (L1-bypassing) loads of item `it` into the swizzled work tile.  Each thread
// issues all of its loads before its first store, so the memory latency is paid once
// per item rather than once per element (all NT threads of the CTA: VOL / NT each).
__device__ __forceinline__ void fill_plain(double2 *work, const TileWork &p, const Item &it, int tid)
{
    constexpr int PER = VOL / NT;
    double re[PER], im[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        const int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        const int64_t gz = it.lz + z, gy = it.ly + y, ga = it.lx + x, gb = it.lxb + x;
        re[k] = 0.0;
        im[k] = 0.0;
        if (p.periodic) {
            const int64_t row = (wrap_near(gz, p.nz) * p.ny + wrap_near(gy, p.ny)) * p.nx;
            re[k] = __ldcg(p.in + row + wrap_near(ga, p.nx));
            if (it.has_b)
                im[k] = __ldcg(p.in + row + wrap_near(gb, p.nx));
        } else if (gz >= 0 && gz < p.nz && gy >= 0 && gy < p.ny) {
            const int64_t row = (gz * p.ny + gy) * p.nx;
            if (ga >= 0 && ga < p.nx)
                re[k] = __ldcg(p.in + row + ga);
            if (it.has_b && gb >= 0 && gb < p.nx)
                im[k] = __ldcg(p.in + row + gb);
        }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k)
        work[sw3(tid + k * NT)] = make_double2(re[k], im[k]);
}

struct NoAction {
    __device__ void operator()() const {}
};

// The six passes of one tile pair (forward x, y, z with the spectrum; inverse z,
// y, x with the cropped store); needs exactly 16 warps.  Warp w owns z-plane w
// for the x and y passes and y-plane w for the z passes, so only two block
// barriers are needed.  `after_first_barrier` runs in every thread once no warp
// reads the staged input any more.
template <int SRC, class After = NoAction>
__device__ __forceinline__ void compute_item(double2 *work, const double *stage, const double2 *spec,
                                             const Consts &c, const TileWork &p, const Item &it, int warp, int g,
                                             int t, After after_first_barrier = After())
{
    pass16<kX, false, SRC, false>(work, stage, warp, c, g, t, p, it);
    __syncwarp();
    pass16<kY, false, kFromWork, false>(work, stage, warp, c, g, t, p, it);
    __syncthreads();
    after_first_barrier();
    pass16_z_round_trip(work, spec, warp, c, g, t);
    __syncthreads();
    if (warp >= p.halo && warp < p.halo + p.useful && it.lz + warp >= p.vlo[2] && it.lz + warp < p.vhi[2]) {
        pass16<kY, true, kFromWork, false>(work, stage, warp, c, g, t, p, it);
        __syncwarp();
        pass16<kX, true, kFromWork, true>(work, stage, warp, c, g, t, p, it);
    }
}

} // namespace dmma3d
} // namespace ffst
