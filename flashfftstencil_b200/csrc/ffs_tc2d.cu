// Fused DFT-tile stencil kernel for 2D grids on tcgen05 tensor cores:
//   FORM_OZAKI: Ozaki-scheme FP64 emulation with INT8 slices (kind::i8, exact
//               INT32 accumulation in TMEM), FP64 only for slice recombination;
//   FORM_BF16:  3-way BF16 split with FP32 accumulation (kind::f16) for ~1e-7 work.
//
// A complex 64 x 64 tile pair (re = left tile, im = right tile) goes through
// four dense DFT-64 GEMMs, each   D[m][n] = sum_k A[m][k] * B[n][k]   with
//   A (128 x 128, constant, in shared memory): the real-block DFT-64 matrix with
//     interleaved rows, m = 2f + part: A[2f][x] = Re F[f][x], A[2f][64+x] = -Im F[f][x],
//     A[2f+1][x] = Im F[f][x], A[2f+1][64+x] = Re F[f][x]   (F[f][x] = w64^(f x));
//   B (64 x 128, data): row n = a line of the tile, k = (part, position along the line);
//   D (128 lanes x 64 columns in TMEM): lane m = (frequency f, part), column n.
// The thread that owns TMEM lane m holds a whole row of D, which is exactly
// row f of the next stage's B: no transposition through memory.  Stages:
//   1. forward over x  (B rows = y)   -> D1[(kx,p)][y]
//   2. forward over y  (B rows = kx)  -> D2[(ky,p)][kx] = W;  W' = W * S^tau / 64^2
//   3. inverse over x  (B rows = ky, conj(W'))  -> D3[(x,p)][ky]
//   4. inverse over y  (B rows = x)   -> D4[(y,p)][x];  out[y][x] = conj(D4)
// (G = conj(F): G v = conj(F conj(v)), so only F is stored.)
//
// Ozaki: every B row n carries a power-of-two scale 2^e_n (its max magnitude);
// values are split into s balanced base-256 digits (ffs_ozaki.cuh) and the DFT
// matrix likewise; products of digit i (data) and j (DFT) with i + j = d
// accumulate into INT32 TMEM accumulator d (exact: |sum| < 2^24), and the row is
// recombined in FP64: V = 2^(e_n - 12) * sum_d 256^(-d) D_d.
// (Ozaki scheme: see ffs_ozaki.cuh.)
// BF16: x = hi + mid + lo (bf16 each, 24 significant bits), products with
// i + j <= slices-1 accumulate into one FP32 accumulator (Henry, Tang &
// Heinecke, "Leveraging the bfloat16 AI datatype for higher-precision
// computations", ARITH 2019).
#include <cuda_bf16.h>

#include <cstring>

#include "ffs_device.cuh"
#include "ffs_kernels.h"
#include "ffs_ozaki.cuh"
#include "ffs_tcgen05.cuh"

namespace ffst {
namespace tc2d {

constexpr int N = 64;
constexpr int NT = 512;  // 16 warps: TMEM lane quadrant = warp & 3, column quarter = warp >> 2
constexpr int CW = 16;   // columns of D per thread
constexpr int M = 128;
constexpr int KE = 128; // contraction length in elements (re half + im half)

template <int FORM>
struct Cfg;
template <>
struct Cfg<kFormOzaki> {
    static constexpr int EB = 1;                    // bytes per operand element
    static constexpr int KB = KE * EB;              // 128 bytes per operand row
    static constexpr int A_SLICE = M * KB;          // 16 KiB
    static constexpr int B_SLICE = N * KB;          // 8 KiB
    static constexpr int KSTEPS = KB / 32;          // 4 MMAs of K = 32
};
template <>
struct Cfg<kFormBf16> {
    static constexpr int EB = 2;
    static constexpr int KB = KE * EB;              // 256 bytes
    static constexpr int A_SLICE = M * KB;          // 32 KiB
    static constexpr int B_SLICE = N * KB;          // 16 KiB
    static constexpr int KSTEPS = KB / 32;          // 8 MMAs of K = 16
};

// At least 120 KiB so that one CTA occupies an SM: each CTA allocates all 512
// TMEM columns for its lifetime, so two co-resident CTAs would wait on each other.
template <int FORM>
__host__ __device__ constexpr size_t smem_bytes(int slices)
{
    const size_t need = (size_t)slices * (Cfg<FORM>::A_SLICE + Cfg<FORM>::B_SLICE) + 2 * 64 * sizeof(int) +
                        4 * 128 * sizeof(double) + 64;
    return need > 120 * 1024 ? need : 120 * 1024;
}

struct Shared {
    unsigned char *A, *B;
    int *escale;       // [2][64] per-B-row exponent (Ozaki)
    double *smax;      // [4][128] per-lane quarter-row maxima
    uint64_t *bar;
    uint32_t *tslot;
};

using oz::exponent_above;
using oz::pow2;

// Write the CW consecutive K elements [k0, k0 + CW) of B row `row` for every slice.
// Ozaki: digits of v * 2^(6 - e); BF16: hi/mid/lo pieces of (float) v.
template <int FORM, int S>
__device__ __forceinline__ void write_b_row(unsigned char *B, int row, int k0, const double (&v)[CW], int e)
{
    if constexpr (FORM == kFormOzaki) {
        const double sc = pow2(6 - e);
        uint64_t U[CW];
#pragma unroll
        for (int c = 0; c < CW; ++c)
            U[c] = oz::digit_bytes<S>(v[c] * sc);
        uint32_t w[S][CW / 4];
        oz::digit_words<S, CW>(U, w);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            uint4 *dst = reinterpret_cast<uint4 *>(B + i * Cfg<FORM>::B_SLICE +
                                                  tc::operand_offset(row, k0, Cfg<FORM>::KB));
            *dst = make_uint4(w[i][0], w[i][1], w[i][2], w[i][3]);
        }
    } else {
        (void)e;
        uint32_t w[S][8];
#pragma unroll
        for (int c = 0; c < CW; c += 2) {
            float r0 = (float)v[c], r1 = (float)v[c + 1];
#pragma unroll
            for (int i = 0; i < S; ++i) {
                const __nv_bfloat162 p = __floats2bfloat162_rn(r0, r1);
                w[i][c >> 1] = *reinterpret_cast<const uint32_t *>(&p);
                r0 -= __low2float(p);
                r1 -= __high2float(p);
            }
        }
        // CW bf16 = 32 bytes = 2 chunks of 16 B
#pragma unroll
        for (int i = 0; i < S; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint4 *dst = reinterpret_cast<uint4 *>(B + i * Cfg<FORM>::B_SLICE +
                                                      tc::operand_offset(row, 2 * (k0 + 8 * h), Cfg<FORM>::KB));
                *dst = make_uint4(w[i][4 * h], w[i][4 * h + 1], w[i][4 * h + 2], w[i][4 * h + 3]);
            }
    }
}

// All MMAs of one stage, issued by a single thread, then a commit to `bar`.  The
// descriptor's start-address field is the byte address >> 4 (14 bits hold every
// shared-memory address), so operand offsets are added to base descriptors.
template <int FORM, int S>
__device__ __forceinline__ void issue_stage(const Shared &sh, uint32_t tmem)
{
    constexpr int KB = Cfg<FORM>::KB;
    const uint64_t adesc0 = tc::smem_desc(smem_u32(sh.A), 128, 8 * KB);
    const uint64_t bdesc0 = tc::smem_desc(smem_u32(sh.B), 128, 8 * KB);
    constexpr uint64_t AS = Cfg<FORM>::A_SLICE >> 4, BS = Cfg<FORM>::B_SLICE >> 4, KS = 256 >> 4;
    if constexpr (FORM == kFormOzaki) {
        constexpr uint32_t idesc = tc::idesc_i8(M, N);
#pragma unroll
        for (int dgl = 0; dgl < S; ++dgl) {
#pragma unroll
            for (int i = 0; i <= dgl; ++i) { // data slice i, DFT slice dgl - i
                const int j = dgl - i;
#pragma unroll
                for (int ks = 0; ks < Cfg<FORM>::KSTEPS; ++ks)
                    tc::mma_i8(tmem + 64 * dgl, adesc0 + j * AS + ks * KS, bdesc0 + i * BS + ks * KS, idesc,
                               i > 0 || ks > 0);
            }
        }
    } else {
        constexpr uint32_t idesc = tc::idesc_bf16(M, N);
#pragma unroll
        for (int dgl = 0; dgl < S; ++dgl) // pieces with i + j <= S - 1, one FP32 accumulator
#pragma unroll
            for (int i = 0; i <= dgl; ++i) {
                const int j = dgl - i;
#pragma unroll
                for (int ks = 0; ks < Cfg<FORM>::KSTEPS; ++ks)
                    tc::mma_f16(tmem, adesc0 + j * AS + ks * KS, bdesc0 + i * BS + ks * KS, idesc,
                                dgl > 0 || i > 0 || ks > 0);
            }
    }
    tc::commit(sh.bar);
}

// TMEM row of this thread (lane m, columns [CW q, CW q + CW)) recombined to doubles.
template <int FORM, int S>
__device__ __forceinline__ void read_row(uint32_t tmem, uint32_t lane_base, int q, const int *escale,
                                         double (&v)[CW])
{
    if constexpr (FORM == kFormOzaki) {
#pragma unroll
        for (int h = 0; h < CW / 8; ++h) { // 8 columns at a time
            uint32_t acc[S][8];
#pragma unroll
            for (int d = 0; d < S; ++d)
                tc::ld8(tmem + lane_base + 64 * d + CW * q + 8 * h, acc[d]);
            tc::ld_wait();
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                uint32_t a[S];
#pragma unroll
                for (int d = 0; d < S; ++d)
                    a[d] = acc[d][c];
                const int n = CW * q + 8 * h + c;
                v[8 * h + c] = oz::combine<S>(a) * pow2(escale[n] - 12);
            }
        }
    } else {
        uint32_t acc[CW];
        tc::ld16(tmem + lane_base + CW * q, acc);
        tc::ld_wait();
#pragma unroll
        for (int c = 0; c < CW; ++c)
            v[c] = (double)__uint_as_float(acc[c]);
    }
}

// Row maximum across the 2 parts (lanes m, m^1) and the 4 column quarters (warps w + 4j).
__device__ __forceinline__ double row_max(const double (&v)[CW], int m, int q, double *smax)
{
    double mx = 0.0;
#pragma unroll
    for (int c = 0; c < CW; ++c)
        mx = fmax(mx, fabs(v[c]));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    smax[q * 128 + m] = mx;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j)
        mx = fmax(mx, smax[j * 128 + m]);
    return mx;
}

struct Item {
    int64_t ly0, lxa, lxb;
    bool has_b;
};

__device__ __forceinline__ Item item_of(const TileWork &p, int64_t w)
{
    Item it;
    const int64_t pr = w % p.npx;
    const int64_t ty = p.t0[1] + w / p.npx;
    const int64_t txa = p.t0[0] + 2 * pr;
    it.has_b = (2 * pr + 1) < p.nt[0];
    it.ly0 = ty * p.useful - p.halo;
    it.lxa = txa * p.useful - p.halo;
    it.lxb = it.lxa + p.useful;
    return it;
}

template <int FORM, int S>
__global__ void __launch_bounds__(NT, 1) tc2d_kernel(const TileWork p, const unsigned char *a_slices)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    Shared sh;
    sh.A = smem;
    sh.B = smem + S * Cfg<FORM>::A_SLICE;
    sh.escale = reinterpret_cast<int *>(sh.B + S * Cfg<FORM>::B_SLICE);
    sh.smax = reinterpret_cast<double *>(sh.escale + 128);
    sh.bar = reinterpret_cast<uint64_t *>(sh.smax + 512);
    sh.tslot = reinterpret_cast<uint32_t *>(sh.bar + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quad = warp & 3, cq = warp >> 2;
    const int m = 32 * quad + lane;       // TMEM lane = D row
    const int f = m >> 1, part = m & 1;   // frequency / position and re-im part of this row
    const uint32_t lane_base = (uint32_t)(32 * quad) << 16;

    {   // constant DFT slices -> shared memory (16-byte copies)
        const uint4 *src = reinterpret_cast<const uint4 *>(a_slices);
        uint4 *dst = reinterpret_cast<uint4 *>(sh.A);
        for (int i = tid; i < S * Cfg<FORM>::A_SLICE / 16; i += NT)
            dst[i] = src[i];
    }
    if (tid == 0) {
        mbar_init(sh.bar, 1);
        fence_barrier_init();
    }
    if (warp == 0)
        tc::tmem_alloc(sh.tslot, 512);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *sh.tslot;
    uint32_t phase = 0;
    bool failed = false;

    // one stage: operands written -> MMAs -> wait; false (in every thread) if any wait timed out
    auto run_stage = [&]() -> bool {
        fence_proxy_async_shared();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_stage<FORM, S>(sh, tmem);
        }
        const bool ok = mbar_wait_bounded(sh.bar, phase);
        phase ^= 1;
        const bool any_fail = __syncthreads_or(!ok) != 0;
        tc::fence_after_sync();
        return !any_fail;
    };

    for (int64_t w = blockIdx.x; w < p.nitems && !failed; w += gridDim.x) {
        const Item it = item_of(p, w);
        int *esc = sh.escale; // [0]: scales of the current B, [64]: next
        // ---- stage 1 operand: B[y][(part, x)] = tile(part)[y][x] ----
        {
            const int y = tid >> 3, pp = (tid >> 2) & 1, qq = tid & 3; // row, part, quarter of the row
            const int64_t gy0 = it.ly0 + y;
            const int64_t gx0 = (pp ? it.lxb : it.lxa) + CW * qq;
            double v[CW];
            const bool have = pp == 0 || it.has_b;
            const bool inside = gy0 >= 0 && gy0 < p.ny && gx0 >= 0 && gx0 + CW <= p.nx;
            const double *row = p.in + (inside ? gy0 * p.nx + gx0 : 0);
            // 16-byte loads only where the row segment starts on a 16-byte boundary
            // (an odd nx puts every other row on an 8-byte one)
            if (have && inside && (reinterpret_cast<uintptr_t>(row) & 15) == 0) {
                const double2 *src = reinterpret_cast<const double2 *>(row);
#pragma unroll
                for (int c = 0; c < CW / 2; ++c) {
                    const double2 t2 = src[c];
                    v[2 * c] = t2.x;
                    v[2 * c + 1] = t2.y;
                }
            } else {
#pragma unroll
                for (int c = 0; c < CW; ++c) {
                    int64_t gy = gy0, gx = gx0 + c;
                    double x = 0.0;
                    if (have) {
                        if (p.periodic)
                            x = p.in[wrap_near(gy, p.ny) * p.nx + wrap_near(gx, p.nx)];
                        else if (gy >= 0 && gy < p.ny && gx >= 0 && gx < p.nx)
                            x = p.in[gy * p.nx + gx];
                    }
                    v[c] = x;
                }
            }
            double mx = 0.0;
#pragma unroll
            for (int c = 0; c < CW; ++c)
                mx = fmax(mx, fabs(v[c]));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
            const int e = mx > 0.0 ? exponent_above(mx) : 0;
            if ((tid & 7) == 0)
                esc[y] = e;
            write_b_row<FORM, S>(sh.B, y, 64 * pp + CW * qq, v, e);
        }
        // ---- stages 1..4 ----
#pragma unroll 1
        for (int st = 0; st < 4 && !failed; ++st) {
            if (!run_stage()) {
                failed = true;
                break;
            }
            double v[CW];
            read_row<FORM, S>(tmem, lane_base, cq, esc, v);
            tc::ld_wait();
            if (st == 1) { // W' = W * S^tau / 64^2, then conj for the inverse
#pragma unroll
                for (int c = 0; c < CW; ++c) {
                    const double other = __shfl_xor_sync(0xffffffffu, v[c], 1);
                    const double re = part ? other : v[c], im = part ? v[c] : other;
                    const double2 s = __ldg(p.spec + f * N + CW * cq + c);
                    const double pr_ = re * s.x - im * s.y, pi_ = re * s.y + im * s.x;
                    v[c] = part ? -pi_ : pr_;
                }
            }
            if (st < 3) {
                int *nesc = (esc == sh.escale) ? sh.escale + 64 : sh.escale;
                const double mx = row_max(v, m, cq, sh.smax);
                const int e = mx > 0.0 ? exponent_above(mx) : 0;
                if (part == 0 && cq == 0)
                    nesc[f] = e;
                write_b_row<FORM, S>(sh.B, f, 64 * part + CW * cq, v, e);
                esc = nesc;
            } else { // out[y][x] = conj(D4[(y, part)][x]), crop to the interior
                const int y = f;
                const int64_t gy = it.ly0 + y;
                if (y >= p.halo && y < p.halo + p.useful && gy >= p.vlo[1] && gy < p.vhi[1] &&
                    (part == 0 || it.has_b)) {
                    const int64_t base = gy * p.nx + (part ? it.lxb : it.lxa);
#pragma unroll
                    for (int c = 0; c < CW; ++c) {
                        const int x = CW * cq + c;
                        const int64_t gx = (part ? it.lxb : it.lxa) + x;
                        if (x >= p.halo && x < p.halo + p.useful && gx >= p.vlo[0] && gx < p.vhi[0])
                            p.out[base + x] = part ? -v[c] : v[c];
                    }
                }
                tc::fence_before_sync();
                __syncthreads();
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

} // namespace tc2d

size_t tc2d_smem_bytes(int form, int slices)
{
    return form == kFormOzaki ? tc2d::smem_bytes<kFormOzaki>(slices) : tc2d::smem_bytes<kFormBf16>(slices);
}

#define FFS_TC2D_CASES(X) X(kFormOzaki, 4) X(kFormOzaki, 5) X(kFormOzaki, 6) X(kFormOzaki, 7) X(kFormOzaki, 8) \
    X(kFormBf16, 2) X(kFormBf16, 3)

cudaError_t prepare_tc2d()
{
    cudaError_t e = cudaSuccess;
#define FFS_SET(F, S)                                                                                             \
    if (e == cudaSuccess)                                                                                         \
        e = cudaFuncSetAttribute(tc2d::tc2d_kernel<F, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,            \
                                 (int)tc2d::smem_bytes<F>(S));
    FFS_TC2D_CASES(FFS_SET)
#undef FFS_SET
    return e;
}

cudaError_t launch_tc2d(int form, int slices, const TileWork &w, const unsigned char *a_slices, int grid,
                        cudaStream_t s)
{
#define FFS_LAUNCH(F, S)                                                                                          \
    if (form == F && slices == S) {                                                                               \
        tc2d::tc2d_kernel<F, S><<<grid, tc2d::NT, tc2d::smem_bytes<F>(S), s>>>(w, a_slices);                     \
        return cudaGetLastError();                                                                                \
    }
    FFS_TC2D_CASES(FFS_LAUNCH)
#undef FFS_LAUNCH
    return cudaErrorInvalidValue;
}

} // namespace ffst
