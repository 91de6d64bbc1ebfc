// 3D FP64-DMMA fused tile (16^3, radix-4 x 4): per-item device functions shared
// by the persistent 3D kernel (ffs_dmma3d.cu) and the batched kernel.
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
constexpr size_t TW_BYTES = 16 * sizeof(double2);
constexpr size_t SMEM_BYTES = STAGE_BYTES + WORK_BYTES + SPEC_BYTES + TW_BYTES + 16;

// XOR swizzle of the 4096-element complex tile: with it every stage's 16-byte
// loads and stores below touch 8 distinct bank groups per quarter warp.
__device__ __forceinline__ int sw3(int i)
{
    const int m2 = ((i >> 7) ^ (i >> 4) ^ (i >> 11) ^ (i >> 8)) & 1;
    const int m1 = ((i >> 6) ^ (i >> 10)) & 1;
    const int m0 = ((i >> 3) ^ (i >> 5) ^ (i >> 9)) & 1;
    return i ^ ((m2 << 2) | (m1 << 1) | m0);
}

struct Consts {
    double f0, f1;   // forward real-block DFT-4, lane (row g, k-col t) for k-steps 0, 1
    double i0, i1;   // inverse (conjugate) real-block DFT-4
    const double2 *w16; // 16th roots of unity (shared memory)
};

enum Tw { kNoTw = 0, kFwdTw = 1, kInvTw = 2, kSpec = 3 };

// One radix-4 stage over 8 x (8 lines of 4 points) of a plane.  Contracted digit
// in bits (TH, TL); line id n = bit0 N0 | bit1 N1 | bit2 N2; iteration bits I0..I2.
// sw3 is linear over GF(2) and the plane, lane and iteration bit fields are
// disjoint, so every swizzled address is a per-lane constant XOR a compile-time
// constant of the (fully unrolled) iteration.
template <int I0, int I1, int I2>
__device__ __forceinline__ constexpr int iter_bits(int it)
{
    return ((it & 1) << I0) | (((it >> 1) & 1) << I1) | ((it >> 2) << I2);
}

template <int TH, int TL, int N0, int N1, int N2, int I0, int I1, int I2, bool INV, int TW>
__device__ __forceinline__ void stage(double2 *work, const double2 *spec, int plane, const Consts &c, int g, int t)
{
    const double a0 = INV ? c.i0 : c.f0, a1 = INV ? c.i1 : c.f1;
    const int ld_off = ((t >> 1) << TH) | ((t & 1) << TL) | ((g & 1) << N0) | (((g >> 1) & 1) << N1) |
                       ((g >> 2) << N2);
    const int dig = g & 3;             // output digit of this lane after the regroup
    const int nn = 2 * t + (g >> 2);   // output line id
    const int st_off = ((dig >> 1) << TH) | ((dig & 1) << TL) | ((nn & 1) << N0) | (((nn >> 1) & 1) << N1) |
                       ((nn >> 2) << N2);
    const int lds = sw3(plane | ld_off), sts = sw3(plane | st_off);
    const int lane_idx = plane | st_off; // logical index of the output, less the iteration bits
    const bool lo = g < 4;
#pragma unroll
    for (int it = 0; it < 8; ++it) {
        const int ib = iter_bits<I0, I1, I2>(it);
        const int sib = sw3(ib); // folds to a constant
        const double2 v = work[lds ^ sib];
        double d0 = 0.0, d1 = 0.0;
        dmma(d0, d1, a0, v.x);
        dmma(d0, d1, a1, v.y);
        const double recv = __shfl_xor_sync(0xffffffffu, lo ? d1 : d0, 16);
        double re = lo ? d0 : recv;
        double im = lo ? recv : d1;
        if (TW == kFwdTw) { // after stage 1: w16^(b * k1), b in the two bits below TL
            const int b = ((lane_idx >> (TL - 2)) & 3) ^ ((ib >> (TL - 2)) & 3);
            const double2 w = c.w16[b * dig];
            cmul(re, im, w.x, w.y);
        } else if (TW == kInvTw) { // after inverse stage 2: conj w16^(b * k1), k1 in the two bits above TH
            const int k1 = ((lane_idx >> (TL + 2)) & 3) ^ ((ib >> (TL + 2)) & 3);
            const double2 w = c.w16[dig * k1];
            cmul(re, im, w.x, -w.y);
        } else if (TW == kSpec) {
            const double2 s = spec[sts ^ sib];
            cmul(re, im, s.x, s.y);
        }
        work[sts ^ sib] = make_double2(re, im);
    }
}

// Final stage (inverse stage 1 along x on z-plane zp): outputs go straight to global memory.
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

__device__ __forceinline__ void last_stage(const double2 *work, int plane, const Consts &c, int g, int t,
                                           const TileWork &p, const Item &itm)
{
    // x inverse stage 1: contract k1 (bits 3,2) -> a; lines n = (x1, x0, y2); iterations y0, y1, y3
    constexpr int TH = 3, TL = 2, N0 = 1, N1 = 0, N2 = 6, I0 = 4, I1 = 5, I2 = 7;
    const int ld_off = ((t >> 1) << TH) | ((t & 1) << TL) | ((g & 1) << N0) | (((g >> 1) & 1) << N1) |
                       ((g >> 2) << N2);
    const int dig = g & 3, nn = 2 * t + (g >> 2);
    const int st_off = ((dig >> 1) << TH) | ((dig & 1) << TL) | ((nn & 1) << N0) | (((nn >> 1) & 1) << N1) |
                       ((nn >> 2) << N2);
    const int lds = sw3(plane | ld_off);
    const int x = st_off & 15, ylane = (st_off >> 4) & 15;
    const int z = plane >> 8;
    const int64_t gz = itm.lz + z;
    const bool lo = g < 4;
    const bool zok = z >= p.halo && z < p.halo + p.useful && gz >= p.vlo[2] && gz < p.vhi[2];
    const int64_t ga = itm.lx + x, gb = itm.lxb + x;
    const bool xa = x >= p.halo && x < p.halo + p.useful && ga >= p.vlo[0] && ga < p.vhi[0];
    const bool xb = itm.has_b && x >= p.halo && x < p.halo + p.useful && gb >= p.vlo[0] && gb < p.vhi[0];
#pragma unroll
    for (int it = 0; it < 8; ++it) {
        const int ib = iter_bits<I0, I1, I2>(it);
        const double2 v = work[lds ^ sw3(ib)];
        double d0 = 0.0, d1 = 0.0;
        dmma(d0, d1, c.i0, v.x);
        dmma(d0, d1, c.i1, v.y);
        const double recv = __shfl_xor_sync(0xffffffffu, lo ? d1 : d0, 16);
        const double re = lo ? d0 : recv;
        const double im = lo ? recv : d1;
        const int y = ylane | (ib >> 4);
        const int64_t gy = itm.ly + y;
        if (!zok || y < p.halo || y >= p.halo + p.useful || gy < p.vlo[1] || gy >= p.vhi[1])
            continue;
        const int64_t row = (gz * p.ny + gy) * p.nx;
        if (xa)
            p.out[row + ga] = re;
        if (xb)
            p.out[row + gb] = im;
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

__device__ __forceinline__ int64_t wrapi(int64_t i, int64_t n)
{
    i %= n;
    return i < 0 ? i + n : i;
}

// Plain (L1-bypassing) loads of item `it` into the swizzled work tile.
__device__ __forceinline__ void fill_plain(double2 *work, const TileWork &p, const Item &it, int tid, int nthreads)
{
    for (int i = tid; i < VOL; i += nthreads) {
        const int x = i & 15, y = (i >> 4) & 15, z = i >> 8;
        int64_t gz = it.lz + z, gy = it.ly + y, ga = it.lx + x, gb = it.lxb + x;
        double re = 0.0, im = 0.0;
        if (p.periodic) {
            const int64_t row = (wrapi(gz, p.nz) * p.ny + wrapi(gy, p.ny)) * p.nx;
            re = __ldcg(p.in + row + wrapi(ga, p.nx));
            if (it.has_b)
                im = __ldcg(p.in + row + wrapi(gb, p.nx));
        } else if (gz >= 0 && gz < p.nz && gy >= 0 && gy < p.ny) {
            const int64_t row = (gz * p.ny + gy) * p.nx;
            if (ga >= 0 && ga < p.nx)
                re = __ldcg(p.in + row + ga);
            if (it.has_b && gb >= 0 && gb < p.nx)
                im = __ldcg(p.in + row + gb);
        }
        work[sw3(i)] = make_double2(re, im);
    }
}

// The 12 radix-4 stages of one tile pair with the spectrum multiply and the
// cropped store; needs exactly 16 warps (warp = plane index).
__device__ __forceinline__ void compute_item(double2 *work, const double2 *spec, const Consts &c, const TileWork &p,
                                             const Item &it, int warp, int g, int t)
{
        // x and y forward on z-plane `warp`
        const int zp = warp << 8, yp = warp << 4;
        stage<3, 2, 1, 0, 6, 4, 5, 7, false, kFwdTw>(work, spec, zp, c, g, t);
        __syncwarp();
        stage<1, 0, 2, 6, 7, 3, 4, 5, false, kNoTw>(work, spec, zp, c, g, t);
        __syncwarp();
        stage<7, 6, 5, 0, 2, 1, 3, 4, false, kFwdTw>(work, spec, zp, c, g, t);
        __syncwarp();
        stage<5, 4, 6, 1, 0, 2, 3, 7, false, kNoTw>(work, spec, zp, c, g, t);
        __syncthreads();
        // z forward, spectrum, z inverse on y-plane `warp`
        stage<11, 10, 9, 2, 0, 1, 3, 8, false, kFwdTw>(work, spec, yp, c, g, t);
        __syncwarp();
        stage<9, 8, 10, 1, 0, 2, 3, 11, false, kSpec>(work, spec, yp, c, g, t);
        __syncwarp();
        stage<9, 8, 10, 1, 0, 2, 3, 11, true, kInvTw>(work, spec, yp, c, g, t);
        __syncwarp();
        stage<11, 10, 9, 2, 0, 1, 3, 8, true, kNoTw>(work, spec, yp, c, g, t);
        __syncthreads();
        // y and x inverse on z-plane `warp`, the last stage stores the cropped interior
        if (zp >> 8 >= p.halo && zp >> 8 < p.halo + p.useful) {
            stage<5, 4, 6, 1, 0, 2, 3, 7, true, kInvTw>(work, spec, zp, c, g, t);
            __syncwarp();
            stage<7, 6, 5, 0, 2, 1, 3, 4, true, kNoTw>(work, spec, zp, c, g, t);
            __syncwarp();
            stage<1, 0, 2, 6, 7, 3, 4, 5, true, kInvTw>(work, spec, zp, c, g, t);
            __syncwarp();
            last_stage(work, zp, c, g, t, p, it);
        }
}

} // namespace dmma3d
} // namespace ffst
