// Fused DFT-tile stencil kernel for 3D grids on tcgen05 tensor cores:
//   FORM_OZAKI: Ozaki-scheme FP64 emulation with INT8 slices (kind::i8, exact
//               INT32 accumulation in TMEM), FP64 only for slice recombination;
//   FORM_BF16:  3-way BF16 split with FP32 accumulation (kind::f16), summed in FP64.
// (The reference's 3D kernel is FP64 only: src/3D/rfft_3d/3d_rfft_N.cu:17-303.)
//
// A complex 16^3 tile pair (re = the tile at x, im = its x neighbour) goes through
// six DFT-16 stages: forward x, y, z, spectrum multiply, inverse z, y, x.  A stage
// transforms all 256 lines of the tile along one axis as two GEMMs of 128 lines,
//   D[l][n] = sum_k A[l][k] * B[n][k]
//   A (data, 128 lines x 32 K): line l's 16 complex values, k = 2 * position + part;
//   B (the constant DFT-16, shared memory): row n = 32 i + 2 f + part of slice i,
//     B[2f][2x] = Re F, B[2f][2x+1] = -Im F, B[2f+1][2x] = Im F, B[2f+1][2x+1] = Re F,
//     F[f][x] = w16^(f x);
//   D (TMEM lane l): the line's 16 transformed complex values, column 2 f + part.
// Ozaki: data slice j is multiplied by DFT slices 0 .. s-1-j in ONE instruction
// (N = 32 (s - j)) whose accumulator starts 32 j columns further on, so data slice
// j times DFT slice i lands in accumulator d = i + j.  Every diagonal sum is exact
// in INT32 TMEM (balanced base-256 digits, see ffs_ozaki.cuh) and no operand is
// zero-padded.  Each line carries a power-of-two scale 2^e (its largest
// magnitude); values are split as digits of v * 2^(6 - e) and the DFT as digits of
// F * 2^6, so a line is recombined as V = 2^(e - 12) * sum_d 256^(-d) D_d.
// BF16: x = hi + mid + lo; pieces with i + j <= s - 1 in short FP32 accumulations
// (hi x hi per K-step, each later diagonal in its own accumulator), summed in FP64
// when read.
// The inverse DFT is G v = conj(F conj(v)): the spectrum product is conjugated and
// the last stage's output conjugated back, so only F is stored.
//
// Between stages on different axes the values go through an FP64 tile in shared
// memory, element (a, b, c) at a * 256 + b * 16 + (c ^ (b & 7)): for every access
// pattern below, each group of 8 lanes touches 8 distinct 16-byte bank groups.
// Forward z -> inverse z transforms the same lines and skips the round trip.
#include <cuda_bf16.h>

#include "ffs_device.cuh"
#include "ffs_kernels.h"
#include "ffs_ozaki.cuh"
#include "ffs_tcgen05.cuh"

namespace ffst {
namespace tc3d {

constexpr int NT = 512; // 16 warps
constexpr int LINES = 256;

template <int FORM>
struct Cfg;
template <>
struct Cfg<kFormOzaki> {
    static constexpr int KB = 32;                    // bytes per operand row (32 int8)
    static constexpr int A_SLICE = LINES * KB;       // 8 KiB: data slice, both 128-line blocks
    static constexpr int F_SLICE = 32 * KB;          // 1 KiB: DFT slice
    static constexpr int BLOCK = 128 * KB;           // second 128-line block
};
template <>
struct Cfg<kFormBf16> {
    static constexpr int KB = 64;                    // 32 bf16
    static constexpr int A_SLICE = LINES * KB;       // 16 KiB
    static constexpr int F_SLICE = 32 * KB;          // 2 KiB
    static constexpr int BLOCK = 128 * KB;
};

// TMEM columns of one 128-line block's accumulators (32 each).  Ozaki: one per
// diagonal.  BF16: the hi x hi products of each of the two K-steps in accumulators 0
// and 1, diagonal d >= 1 in accumulator d + 1, summed in FP64 when read: short FP32
// accumulations, since an FP32 accumulator rounds at every MMA it absorbs.
template <int FORM, int S>
__host__ __device__ constexpr int block_cols()
{
    return FORM == kFormOzaki ? 32 * S : 32 * (S + 1);
}

constexpr size_t TILE_BYTES = 4096 * sizeof(double2);
template <int FORM>
__host__ __device__ constexpr size_t smem_bytes(int slices)
{
    // tile + spectrum + data slices + DFT slices + 2 x 256 scales + 2 x 256 maxima + barrier
    return 2 * TILE_BYTES + (size_t)slices * (Cfg<FORM>::A_SLICE + Cfg<FORM>::F_SLICE) + 2 * LINES * sizeof(int) +
           2 * LINES * sizeof(double) + 64;
}

__device__ __forceinline__ int tidx(int a, int b, int c) { return a * 256 + b * 16 + (c ^ (b & 7)); }

// Write positions [8h, 8h + 8) of operand row `row` (v = re, im interleaved) for every slice.
template <int FORM, int S>
__device__ __forceinline__ void write_a_row(unsigned char *A, int row, int h, const double (&v)[16], int e)
{
    constexpr int KB = Cfg<FORM>::KB;
    if constexpr (FORM == kFormOzaki) {
        const double sc = oz::pow2(6 - e);
        uint64_t U[16];
#pragma unroll
        for (int c = 0; c < 16; ++c)
            U[c] = oz::digit_bytes<S>(v[c] * sc);
        uint32_t w[S][4];
        oz::digit_words<S, 16>(U, w);
#pragma unroll
        for (int i = 0; i < S; ++i)
            *reinterpret_cast<uint4 *>(A + i * Cfg<FORM>::A_SLICE + tc::operand_offset(row, 16 * h, KB)) =
                make_uint4(w[i][0], w[i][1], w[i][2], w[i][3]);
    } else {
        (void)e;
        uint32_t w[S][8];
#pragma unroll
        for (int c = 0; c < 16; c += 2) {
            float r0 = (float)v[c], r1 = (float)v[c + 1];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                const __nv_bfloat162 pr = __floats2bfloat162_rn(r0, r1);
                w[i][c >> 1] = *reinterpret_cast<const uint32_t *>(&pr);
                r0 -= __low2float(pr);
                r1 -= __high2float(pr);
            }
        }
#pragma unroll
        for (int i = 0; i < S; ++i)
#pragma unroll
            for (int hh = 0; hh < 2; ++hh)
                *reinterpret_cast<uint4 *>(A + i * Cfg<FORM>::A_SLICE +
                                           tc::operand_offset(row, 32 * h + 16 * hh, KB)) =
                    make_uint4(w[i][4 * hh], w[i][4 * hh + 1], w[i][4 * hh + 2], w[i][4 * hh + 3]);
    }
}

// All MMAs of one stage (both 128-line blocks), issued by one thread, then a commit.
template <int FORM, int S>
__device__ __forceinline__ void issue_stage(const unsigned char *A, const unsigned char *F, uint32_t tmem,
                                            uint64_t *bar)
{
    constexpr int KB = Cfg<FORM>::KB;
    const uint64_t adesc0 = tc::smem_desc(smem_u32(A), 128, 8 * KB);
    const uint64_t fdesc0 = tc::smem_desc(smem_u32(F), 128, 8 * KB);
    constexpr uint64_t AS = Cfg<FORM>::A_SLICE >> 4, FS = Cfg<FORM>::F_SLICE >> 4, BS = Cfg<FORM>::BLOCK >> 4;
    constexpr int COLS = block_cols<FORM, S>();
    if constexpr (FORM == kFormOzaki) {
#pragma unroll
        for (int j = 0; j < S; ++j) { // data slice j x DFT slices 0 .. S-1-j -> accumulators j .. S-1
            const uint32_t idesc = tc::idesc_i8(128, 32 * (S - j));
#pragma unroll
            for (int b = 0; b < 2; ++b)
                tc::mma_i8(tmem + b * COLS + 32 * j, adesc0 + j * AS + b * BS, fdesc0, idesc, j > 0);
        }
    } else {
        constexpr uint32_t idesc = tc::idesc_bf16(128, 32);
        constexpr uint64_t KS = 256 >> 4; // 16 bf16 per MMA = two 16-byte core-matrix columns
#pragma unroll
        for (int dgl = 0; dgl < S; ++dgl)
#pragma unroll
            for (int i = 0; i <= dgl; ++i) { // data piece i, DFT piece dgl - i
                const int j = dgl - i;
#pragma unroll
                for (int b = 0; b < 2; ++b)
#pragma unroll
                    for (int ks = 0; ks < 2; ++ks) {
                        const int a = dgl == 0 ? ks : dgl + 1;
                        const bool first = dgl == 0 || (i == 0 && ks == 0);
                        tc::mma_f16(tmem + b * COLS + 32 * a, adesc0 + i * AS + b * BS + ks * KS,
                                    fdesc0 + j * FS + ks * KS, idesc, !first);
                    }
            }
    }
    tc::commit(bar);
}

// This thread's 16 accumulator columns (8 complex values) of its line, recombined.
template <int FORM, int S>
__device__ __forceinline__ void read_line(uint32_t taddr, int e, double (&v)[16])
{
    if constexpr (FORM == kFormOzaki) {
        const double sc = oz::pow2(e - 12);
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            uint32_t acc[S][8];
#pragma unroll
            for (int d = 0; d < S; ++d)
                tc::ld8(taddr + 32 * d + 8 * hh, acc[d]);
            tc::ld_wait();
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                uint32_t a[S];
#pragma unroll
                for (int d = 0; d < S; ++d)
                    a[d] = acc[d][c];
                v[8 * hh + c] = oz::combine<S>(a) * sc;
            }
        }
    } else {
        (void)e;
#pragma unroll
        for (int c = 0; c < 16; ++c)
            v[c] = 0.0;
#pragma unroll
        for (int a = S; a >= 0; --a) { // the small diagonals first
            uint32_t acc[16];
            tc::ld16(taddr + 32 * a, acc);
            tc::ld_wait();
#pragma unroll
            for (int c = 0; c < 16; ++c)
                v[c] += (double)__uint_as_float(acc[c]);
        }
    }
}

__device__ __forceinline__ int line_exponent(const double (&v)[16], double partner_max)
{
    double mx = partner_max;
#pragma unroll
    for (int c = 0; c < 16; ++c)
        mx = fmax(mx, fabs(v[c]));
    return mx > 0.0 ? oz::exponent_above(mx) : 0;
}

__device__ __forceinline__ double local_max(const double (&v)[16])
{
    double mx = 0.0;
#pragma unroll
    for (int c = 0; c < 16; ++c)
        mx = fmax(mx, fabs(v[c]));
    return mx;
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

// Cell (gz, gy, gx) of the input; outside the grid: wrapped (periodic) or 0 (fixed,
// whose outer cells are recomputed by the band kernel).
__device__ __forceinline__ double fetch(const TileWork &p, int64_t gz, int64_t gy, int64_t gx)
{
    if (p.periodic)
        return __ldg(p.in + (wrap_near(gz, p.nz) * p.ny + wrap_near(gy, p.ny)) * p.nx + wrap_near(gx, p.nx));
    if (gz < 0 || gz >= p.nz || gy < 0 || gy >= p.ny || gx < 0 || gx >= p.nx)
        return 0.0;
    return __ldg(p.in + (gz * p.ny + gy) * p.nx + gx);
}

template <int FORM, int S>
__global__ void __launch_bounds__(NT, 1) tc3d_kernel(const TileWork p, const unsigned char *f_slices)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double2 *tile = reinterpret_cast<double2 *>(smem);
    double2 *spec = reinterpret_cast<double2 *>(smem + TILE_BYTES);
    unsigned char *A = smem + 2 * TILE_BYTES;
    unsigned char *F = A + S * Cfg<FORM>::A_SLICE;
    int *escale = reinterpret_cast<int *>(F + S * Cfg<FORM>::F_SLICE); // [2][256]
    double *smax = reinterpret_cast<double *>(escale + 2 * LINES);     // [2][256]
    uint64_t *bar = reinterpret_cast<uint64_t *>(smax + 2 * LINES);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // split role: line ls (16 per warp), half hs (positions 8 hs .. 8 hs + 7); partner = lane ^ 16
    const int ls = warp * 16 + (lane & 15), hs = lane >> 4;
    // recombine role: TMEM lane quadrant q = warp & 3, block b, half hr; line lr
    const int q = warp & 3, g = warp >> 2, b = g >> 1, hr = g & 1;
    const int lr = 128 * b + 32 * q + lane;
    constexpr int COLS = block_cols<FORM, S>();

    {   // constants: DFT slices and the spectrum (natural order kz, ky, kx)
        const uint4 *src = reinterpret_cast<const uint4 *>(f_slices);
        uint4 *dst = reinterpret_cast<uint4 *>(F);
        for (int i = tid; i < S * Cfg<FORM>::F_SLICE / 16; i += NT)
            dst[i] = src[i];
        for (int i = tid; i < 4096; i += NT)
            spec[i] = p.spec[i];
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    if (warp == 0)
        tc::tmem_alloc(tslot, 512);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + b * COLS + 16 * hr;
    uint32_t phase = 0;
    bool failed = false;

    auto run_stage = [&]() -> bool {
        fence_proxy_async_shared();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_stage<FORM, S>(A, F, tmem, bar);
        }
        const bool ok = mbar_wait_bounded(bar, phase);
        phase ^= 1;
        const bool any_fail = __syncthreads_or(!ok) != 0;
        tc::fence_after_sync();
        return !any_fail;
    };
    // split role: operand row ls from v (positions 8 hs ..), scale into escale[buf]
    auto split = [&](const double (&v)[16], int buf) {
        const double pm = __shfl_xor_sync(0xffffffffu, local_max(v), 16);
        const int e = line_exponent(v, pm);
        if (hs == 0)
            escale[buf * LINES + ls] = e;
        write_a_row<FORM, S>(A, ls, hs, v, e);
    };

    for (int64_t w = blockIdx.x; w < p.nitems && !failed; w += gridDim.x) {
        const Item it = item_of(p, w);
        {   // stage 0 operand: lines (z, y) along x, straight from global memory
            const int z = ls >> 4, y = ls & 15;
            const int64_t gz = it.lz + z, gy = it.ly + y;
            double v[16];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int x = 8 * hs + c;
                v[2 * c] = fetch(p, gz, gy, it.lx + x);
                v[2 * c + 1] = it.has_b ? fetch(p, gz, gy, it.lxb + x) : 0.0;
            }
            split(v, 0);
        }
#pragma unroll 1
        for (int st = 0; st < 6; ++st) {
            if (!run_stage()) {
                failed = true;
                break;
            }
            double v[16];
            read_line<FORM, S>(taddr, escale[(st & 1) * LINES + lr], v);
            const int la = lr >> 4, lb = lr & 15; // line coordinates (outer, inner)
            if (st == 2) {
                // forward z done: line (ky, kx), positions kz.  W' = conj(W * S^tau / 16^3),
                // then straight into the inverse-z operand (same lines)
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const double2 s = spec[(8 * hr + c) * 256 + lr];
                    const double re = v[2 * c], im = v[2 * c + 1];
                    v[2 * c] = re * s.x - im * s.y;
                    v[2 * c + 1] = -(re * s.y + im * s.x);
                }
                smax[hr * LINES + lr] = local_max(v);
                __syncthreads();
                const int e = line_exponent(v, smax[(hr ^ 1) * LINES + lr]);
                if (hr == 0)
                    escale[LINES + lr] = e;
                write_a_row<FORM, S>(A, lr, hr, v, e);
                continue;
            }
            if (st == 5) { // inverse x done: line (z, y), positions x; out = conj, cropped
                const int64_t gz = it.lz + la, gy = it.ly + lb;
                const bool rowok = la >= p.halo && la < p.halo + p.useful && gz >= p.vlo[2] && gz < p.vhi[2] &&
                                   lb >= p.halo && lb < p.halo + p.useful && gy >= p.vlo[1] && gy < p.vhi[1];
                if (rowok) {
                    double *row = p.out + (gz * p.ny + gy) * p.nx;
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        const int x = 8 * hr + c;
                        if (x < p.halo || x >= p.halo + p.useful)
                            continue;
                        const int64_t ga = it.lx + x, gb = it.lxb + x;
                        if (ga >= p.vlo[0] && ga < p.vhi[0])
                            row[ga] = v[2 * c];
                        if (it.has_b && gb >= p.vlo[0] && gb < p.vhi[0])
                            row[gb] = -v[2 * c + 1];
                    }
                }
                continue;
            }
            // into the FP64 tile: st 0 line (z, y) -> (z, y, kx); st 1 line (z, kx) -> (z, ky, kx);
            // st 3 line (ky, kx) -> (z, ky, kx); st 4 line (z, kx) -> (z, y, kx)
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int f = 8 * hr + c;
                const int i = st == 0 ? tidx(la, lb, f) : (st == 3 ? tidx(f, la, lb) : tidx(la, f, lb));
                tile[i] = make_double2(v[2 * c], v[2 * c + 1]);
            }
            __syncthreads();
            // next operand from the tile: st 1 and 4 lines (z, kx) along y; st 2 lines (ky, kx)
            // along z; st 5 lines (z, y) along x
            {
                const int sa = ls >> 4, sb = ls & 15;
                double u[16];
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const int pos = 8 * hs + c;
                    const int i = (st == 0 || st == 3) ? tidx(sa, pos, sb)
                                                       : (st == 1 ? tidx(pos, sa, sb) : tidx(sa, sb, pos));
                    const double2 t2 = tile[i];
                    u[2 * c] = t2.x;
                    u[2 * c + 1] = t2.y;
                }
                split(u, (st + 1) & 1);
            }
        }
    }
    if (failed && tid == 0)
        record_error(p.status, kDevTimeoutMma);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0)
        tc::tmem_dealloc(tmem, 512);
}

} // namespace tc3d

size_t tc3d_smem_bytes(int form, int slices)
{
    return form == kFormOzaki ? tc3d::smem_bytes<kFormOzaki>(slices) : tc3d::smem_bytes<kFormBf16>(slices);
}

#define FFS_TC3D_CASES(X) X(kFormOzaki, 4) X(kFormOzaki, 5) X(kFormOzaki, 6) X(kFormOzaki, 7) X(kFormOzaki, 8) \
    X(kFormBf16, 2) X(kFormBf16, 3)

cudaError_t prepare_tc3d()
{
    cudaError_t e = cudaSuccess;
#define FFS_SET(F, S)                                                                                             \
    if (e == cudaSuccess)                                                                                         \
        e = cudaFuncSetAttribute(tc3d::tc3d_kernel<F, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                                 (int)tc3d::smem_bytes<F>(S));
    FFS_TC3D_CASES(FFS_SET)
#undef FFS_SET
    return e;
}

cudaError_t launch_tc3d(int form, int slices, const TileWork &w, const unsigned char *f_slices, int grid,
                        cudaStream_t s)
{
#define FFS_LAUNCH(F, S)                                                                                          \
    if (form == F && slices == S) {                                                                               \
        tc3d::tc3d_kernel<F, S><<<grid, tc3d::NT, tc3d::smem_bytes<F>(S), s>>>(w, f_slices);                     \
        return cudaGetLastError();                                                                                \
    }
    FFS_TC3D_CASES(FFS_LAUNCH)
#undef FFS_LAUNCH
    return cudaErrorInvalidValue;
}

} // namespace ffst
