// Direct FP64 stepping of fixed-boundary band boxes: device function shared by
// the band kernel (ffs_band.cu) and the batched kernel.
#pragma once
#include "ffs_device.cuh"
#include "ffs_kernels.h"

namespace ffst {
namespace band {

constexpr int kWarpCells = 8; // cells per lane of the one-warp 1-D path

// One warp steps a 1-D box whose staged region [L, L + ext) has at most 32 * K cells,
// entirely in registers: lane l holds cells [lK, lK + K), the R cells beyond each end
// of its chunk come from the neighbouring lanes by shuffles, so a time step needs no
// barrier (a block-wide one per step dominated the generic path for these boxes).
// Same update rule as the generic path: the ring and the cells whose taps leave the
// staged region keep their value.
template <int R, int K>
__device__ __forceinline__ void process_box_1d_warp(const BandWork &p, const BandBox &bx, int64_t L, int ext)
{
    const int lane = threadIdx.x & 31;
    double w[2 * R + 1];
#pragma unroll
    for (int k = 0; k < 2 * R + 1; ++k)
        w[k] = p.weights[k];
    double v[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int c = lane * K + j;
        v[j] = c < ext ? __ldcg(p.in + L + c) : 0.0;
    }
    const int lo = (int)max((int64_t)R, (int64_t)R - L);                  // staged coordinates
    const int hi = (int)min((int64_t)ext - R, (int64_t)(p.n[0] - R) - L); // exclusive
    for (int s = 0; s < p.tau; ++s) {
        double lft[R], rgt[R];
#pragma unroll
        for (int m = 1; m <= R; ++m) {
            lft[m - 1] = __shfl_up_sync(0xffffffffu, v[K - m], 1);   // cell lK - m
            rgt[m - 1] = __shfl_down_sync(0xffffffffu, v[m - 1], 1); // cell lK + K - 1 + m
        }
        double nv[K];
#pragma unroll
        for (int j = 0; j < K; ++j) {
            const int c = lane * K + j;
            double acc = 0.0;
#pragma unroll
            for (int dx = -R; dx <= R; ++dx) {
                const int idx = j + dx;
                const double x = idx < 0 ? lft[-idx - 1] : (idx >= K ? rgt[idx - K] : v[idx]);
                acc += w[dx + R] * x;
            }
            nv[j] = (c >= lo && c < hi) ? acc : v[j];
        }
#pragma unroll
        for (int j = 0; j < K; ++j)
            v[j] = nv[j];
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
        const int64_t gx = L + lane * K + j;
        if (gx >= bx.lo[0] && gx < bx.lo[0] + bx.ext[0])
            p.out[gx] = v[j];
    }
}

// Quotient t / d for 0 <= t < 2^22 without an integer division: a float reciprocal gives
// the quotient to within one, and the remainder's sign corrects it.
struct QuickDiv {
    int d;
    float inv;
    __device__ __forceinline__ explicit QuickDiv(int d_) : d(d_), inv(1.0f / (float)d_) {}
    __device__ __forceinline__ int operator()(int t) const
    {
        int q = __float2int_rz((float)t * inv);
        const int rem = t - q * d;
        q += rem >= d ? 1 : 0;
        q -= rem < 0 ? 1 : 0;
        return q;
    }
};

// Direct stepping of band box `box` with `nthreads` threads; `smem` holds
// band_smem_bytes(max_vol, ntaps) bytes.
// NTAPS > 0: the stencil has exactly NTAPS non-zero taps, held in registers for all tau
// steps (weights and offsets otherwise come from shared memory at every tap of every step).
// ROWS: 2-D 3 x 3 boxes may step by warp rows (below); a separate instantiation, since that
// path's registers (64 against 48) cost the other boxes occupancy.
template <int DIM, int NTAPS = 0, bool ROWS = false>
__device__ __forceinline__ void process_box(const BandWork &p, int box, unsigned char *smem, int nthreads)
{
    const BandBox bx = p.boxes[box];
    const int tau = p.tau, r = p.r;
    const int64_t rt = (int64_t)p.r * p.tau;
    if constexpr (DIM == 1) { // small 1-D boxes: one warp, registers and shuffles
        const int64_t lo = bx.lo[0] - rt < 0 ? 0 : bx.lo[0] - rt;
        const int64_t hi = bx.lo[0] + bx.ext[0] + rt > p.n[0] ? p.n[0] : bx.lo[0] + bx.ext[0] + rt;
        const int ext = (int)(hi - lo);
        if (ext <= 32 * kWarpCells && r >= 1 && r <= 4) {
            if (threadIdx.x < 32) {
                switch (r) {
                case 1: process_box_1d_warp<1, kWarpCells>(p, bx, lo, ext); break;
                case 2: process_box_1d_warp<2, kWarpCells>(p, bx, lo, ext); break;
                case 3: process_box_1d_warp<3, kWarpCells>(p, bx, lo, ext); break;
                default: process_box_1d_warp<4, kWarpCells>(p, bx, lo, ext); break;
                }
            }
            return;
        }
    }

    int64_t L[3];
    int ext[3];
    int vol = 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d < DIM) {
            L[d] = bx.lo[d] - rt < 0 ? 0 : bx.lo[d] - rt;
            const int64_t hi = bx.lo[d] + bx.ext[d] + rt;
            ext[d] = (int)((hi > p.n[d] ? p.n[d] : hi) - L[d]);
        } else {
            L[d] = 0;
            ext[d] = 1;
        }
        vol *= ext[d];
    }
    if (vol > p.max_vol) { // the host sizes shared memory for the largest box; refuse otherwise
        if (threadIdx.x == 0)
            record_error(p.status, kDevBadConfig);
        return;
    }
    // staged region is dense with the box's own loaded extents as strides
    const int ex = ext[0], exy = ext[0] * ext[1];
    const int64_t plane = (p.max_vol + 1) & ~(int64_t)1; // keeps the int4 taps 16-byte aligned
    double *buf0 = reinterpret_cast<double *>(smem);
    double *buf1 = buf0 + plane;
    double *wts = buf1 + plane;
    int *toff = reinterpret_cast<int *>(wts + ((p.ntaps + 1) & ~1));
    for (int i = threadIdx.x; i < p.ntaps; i += nthreads) {
        const int4 tp = p.taps[i];
        wts[i] = p.weights[tp.w];
        toff[i] = tp.z * exy + tp.y * ex + tp.x;
    }
    for (int i = threadIdx.x; i < vol; i += nthreads) {
        const int z = DIM == 3 ? i / exy : 0;
        const int rem = i - z * exy;
        const int y = DIM >= 2 ? rem / ex : 0;
        const int x = rem - y * ex;
        buf0[i] = __ldcg(p.in + ((L[2] + z) * p.n[1] + (L[1] + y)) * p.n[0] + (L[0] + x));
    }
    __syncthreads();
    double tap_w[NTAPS > 0 ? NTAPS : 1];
    int tap_o[NTAPS > 0 ? NTAPS : 1];
    if constexpr (NTAPS > 0) {
#pragma unroll
        for (int k = 0; k < NTAPS; ++k) {
            tap_w[k] = wts[k];
            tap_o[k] = toff[k];
        }
    }
    // Per-dim bounds of the cells updated at step s (0-based): never the ring; on a side where
    // the staged region ends at a cut through the grid (not at the grid's face) only cells at
    // least (s + 1) r from that end, since only those feed the box's values after the tau
    // steps (the box lies r tau inside every cut end).  The region shrinks by r per step.
    bool cut_lo[3], cut_hi[3];
    int ring_lo[3], ring_hi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (d < DIM) {
            cut_lo[d] = L[d] > 0;
            cut_hi[d] = L[d] + ext[d] < p.n[d];
            ring_lo[d] = (int)max((int64_t)r, (int64_t)r - L[d]);                      // the grid's ring
            ring_hi[d] = (int)min((int64_t)ext[d] - r, (int64_t)(p.n[d] - r) - L[d]); // (exclusive)
        } else {
            cut_lo[d] = cut_hi[d] = false;
            ring_lo[d] = 0;
            ring_hi[d] = 1;
        }
    }
    int ulo[3], uhi[3];
    auto bounds = [&](int s) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            ulo[d] = cut_lo[d] ? max(ring_lo[d], (s + 1) * r) : ring_lo[d];
            uhi[d] = cut_hi[d] ? min(ring_hi[d], ext[d] - (s + 1) * r) : ring_hi[d];
        }
    };
    // Each thread steps kCells cells at a time (cells base + c * nthreads): the tap loop is
    // outermost, so a tap's weight and offset (broadcast shared loads) serve all kCells cells
    // and their kCells accumulations are independent chains.  Per cell the taps are summed in
    // the same order as one cell at a time.  When the staged box fits in one such chunk per
    // thread (up to kCells * nthreads cells), the cells' positions are decoded once for all
    // tau steps.  Cells outside the step's bounds keep their value (they are not read later
    // by any cell that is still updated).
    constexpr int kCells = 4;
    const QuickDiv by_ex(ex), by_exy(exy); // (staged regions hold at most ~13 K cells)
    auto decode = [&](int base, int (&idx)[kCells], int (&pos)[kCells][3]) {
#pragma unroll
        for (int c = 0; c < kCells; ++c) {
            const int i = base + c * nthreads;
            const int z = DIM == 3 ? by_exy(i) : 0;
            const int rem = i - z * exy;
            const int y = DIM >= 2 ? by_ex(rem) : 0;
            idx[c] = i;
            pos[c][0] = rem - y * ex;
            pos[c][1] = y;
            pos[c][2] = z;
        }
    };
    auto step = [&](const int (&idx)[kCells], const int (&pos)[kCells][3], const double *src, double *dst) {
        bool upd[kCells];
#pragma unroll
        for (int c = 0; c < kCells; ++c)
            upd[c] = idx[c] < vol && pos[c][0] >= ulo[0] && pos[c][0] < uhi[0] && pos[c][1] >= ulo[1] &&
                     pos[c][1] < uhi[1] && pos[c][2] >= ulo[2] && pos[c][2] < uhi[2];
        double acc[kCells];
#pragma unroll
        for (int c = 0; c < kCells; ++c)
            acc[c] = 0.0;
        if constexpr (NTAPS > 0) {
#pragma unroll
            for (int k = 0; k < NTAPS; ++k)
#pragma unroll
                for (int c = 0; c < kCells; ++c)
                    if (upd[c])
                        acc[c] += tap_w[k] * src[idx[c] + tap_o[k]];
        } else {
            for (int k = 0; k < p.ntaps; ++k) {
                const double w = wts[k];
                const int o = toff[k];
#pragma unroll
                for (int c = 0; c < kCells; ++c)
                    if (upd[c])
                        acc[c] += w * src[idx[c] + o];
            }
        }
#pragma unroll
        for (int c = 0; c < kCells; ++c)
            if (idx[c] < vol) // cells not updated keep their value
                dst[idx[c]] = upd[c] ? acc[c] : src[idx[c]];
    };
    double *src = buf0, *dst = buf1;
    bool stepped = false;
    if constexpr (DIM == 2 && NTAPS == 9 && ROWS) {
        // All nine taps of a 3 x 3 box (r = 1 with 9 non-zero taps): a warp takes a unit of 32
        // consecutive x and 4 consecutive y, one column of 4 cells per lane.  The 6 rows
        // y0 - 1 .. y0 + 4 are read once each at x - 1, x and x + 1 (18 shared loads for 4
        // cells, against 36 tap by tap), lanes on consecutive x.  Each cell sums its taps in
        // the tap list's order (dy, then dx), as the tap-by-tap path does.  An updated cell lies
        // at least r inside the staged region, so every row and column read here is in it.
        // Only for staged widths that fill whole warps: 16- and 48-wide regions left lanes idle
        // (the 64 x 64 tile's boxes at tau 8 ran 3 % slower this way, Box2D9P 4096^2 898 -> 870
        // GStencil/s), while the 128 x 128 tile's at tau 16, 32 and 64 wide, ran 1000-1016 ->
        // 1039-1051, and 8192^2 1166-1170 -> 1185-1186.
        if (r == 1 && (ex & 31) == 0) {
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = nthreads >> 5;
            const int ey = ext[1], nstrips = (ex + 31) >> 5, nunits = nstrips * ((ey + 3) >> 2);
            const QuickDiv by_strips(nstrips);
            for (int s = 0; s < tau; ++s) {
                bounds(s);
                for (int u = warp; u < nunits; u += nwarps) {
                    const int yb = by_strips(u), x = (u - yb * nstrips) * 32 + lane, y0 = yb * 4;
                    if (x >= ex)
                        continue;
                    const bool xin = x >= ulo[0] && x < uhi[0];
                    bool upd[4];
                    double acc[4];
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int y = y0 + c;
                        upd[c] = xin && y < ey && y >= ulo[1] && y < uhi[1];
                        acc[c] = 0.0;
                    }
#pragma unroll
                    for (int j = 0; j < 6; ++j) { // row y0 - 1 + j feeds cells c = j - 2 .. j (dy = j - 1 - c)
                        bool need = false;
#pragma unroll
                        for (int c = 0; c < 4; ++c)
                            if (c >= j - 2 && c <= j)
                                need |= upd[c];
                        if (!need)
                            continue;
                        const double *row = src + (y0 - 1 + j) * ex + x;
                        const double vm = row[-1], v0 = row[0], vp = row[1];
#pragma unroll
                        for (int c = 0; c < 4; ++c)
                            if (c >= j - 2 && c <= j && upd[c]) {
                                const int k = 3 * (j - c); // tap (dy, -1) of the list
                                acc[c] += tap_w[k] * vm;
                                acc[c] += tap_w[k + 1] * v0;
                                acc[c] += tap_w[k + 2] * vp;
                            }
                    }
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const int i = (y0 + c) * ex + x;
                        if (y0 + c < ey) // cells not updated keep their value
                            dst[i] = upd[c] ? acc[c] : src[i];
                    }
                }
                __syncthreads();
                double *tmp = src;
                src = dst;
                dst = tmp;
            }
            stepped = true;
        }
    }
    if (stepped) {
    } else if (vol <= nthreads * kCells) {
        int idx[kCells], pos[kCells][3];
        decode(threadIdx.x, idx, pos);
        for (int s = 0; s < tau; ++s) {
            bounds(s);
            step(idx, pos, src, dst);
            __syncthreads();
            double *tmp = src;
            src = dst;
            dst = tmp;
        }
    } else if (vol <= 2 * nthreads * kCells) { // two chunks per thread, decoded once
        int idx0[kCells], pos0[kCells][3], idx1[kCells], pos1[kCells][3];
        decode(threadIdx.x, idx0, pos0);
        decode(threadIdx.x + nthreads * kCells, idx1, pos1);
        for (int s = 0; s < tau; ++s) {
            bounds(s);
            step(idx0, pos0, src, dst);
            step(idx1, pos1, src, dst);
            __syncthreads();
            double *tmp = src;
            src = dst;
            dst = tmp;
        }
    } else {
        for (int s = 0; s < tau; ++s) {
            bounds(s);
            for (int base = threadIdx.x; base < vol; base += nthreads * kCells) {
                int idx[kCells], pos[kCells][3];
                decode(base, idx, pos);
                step(idx, pos, src, dst);
            }
            __syncthreads();
            double *tmp = src;
            src = dst;
            dst = tmp;
        }
    }
    const int bex = bx.ext[0], bexy = bx.ext[0] * bx.ext[1];
    const int bvol = bexy * bx.ext[2];
    for (int i = threadIdx.x; i < bvol; i += nthreads) {
        const int z = DIM == 3 ? i / bexy : 0;
        const int rem = i - z * bexy;
        const int y = DIM >= 2 ? rem / bex : 0;
        const int x = rem - y * bex;
        const int64_t gx = bx.lo[0] + x, gy = bx.lo[1] + y, gz = bx.lo[2] + z;
        const int li = (int)(((gz - L[2]) * ext[1] + (gy - L[1])) * ext[0] + (gx - L[0]));
        p.out[(gz * p.n[1] + gy) * p.n[0] + gx] = src[li];
    }
}

} // namespace band
} // namespace ffst
