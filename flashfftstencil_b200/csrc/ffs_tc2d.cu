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
// i + j <= slices-1 (Henry, Tang & Heinecke, "Leveraging the bfloat16 AI datatype
// for higher-precision computations", ARITH 2019) in short FP32 accumulations: hi x hi
// in four K-chunks, each later diagonal in its own accumulator, summed in FP64 when
// read (one accumulator for all 48 MMAs of a stage measured 10x the error).
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

// Shared memory: DFT slices A, `slots` B operands, per-slot row exponents
// ([slots][2][64] int16: current and next operand), quarter-row exponents
// ([4][128] int16), one mbarrier per slot, the TMEM address.  At least 120 KiB so
// that one CTA occupies an SM: each CTA allocates all 512 TMEM columns for its
// lifetime, so two co-resident CTAs would wait on each other.
template <int FORM>
__host__ __device__ constexpr size_t smem_need(int S, int slots)
{
    return (size_t)S * Cfg<FORM>::A_SLICE + (size_t)slots * S * Cfg<FORM>::B_SLICE + (size_t)slots * 128 * 2 +
           512 * 2 + (size_t)slots * 8 + 16;
}

// Tile pairs in flight per CTA: two when two B operands fit beside the DFT slices
// (every form but Ozaki with 8 slices).
template <int FORM>
__host__ __device__ constexpr int slots_for(int S)
{
    return smem_need<FORM>(S, 2) <= 227 * 1024 ? 2 : 1;
}

template <int FORM>
__host__ __device__ constexpr size_t smem_bytes(int S)
{
    const size_t need = smem_need<FORM>(S, slots_for<FORM>(S));
    return need > 120 * 1024 ? need : 120 * 1024;
}

using oz::exponent_above;
using oz::pow2;

// BF16 accumulators (64 TMEM columns each): the hi x hi products of K-steps
// [2c, 2c + 2) in accumulator c < kBf16Chunks, diagonal d >= 1 in kBf16Chunks + d - 1.
// Short FP32 accumulations: an FP32 accumulator rounds at every MMA it absorbs, and one
// accumulator for all products of a stage absorbs 48 of them (6 products x 8 K-steps).
constexpr int kBf16Chunks = 4;
__host__ __device__ constexpr int bf16_acc(int dgl, int ks)
{
    return dgl == 0 ? ks / (8 / kBf16Chunks) : kBf16Chunks + dgl - 1;
}

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

// All MMAs of one stage of one tile pair (operand B at `B`), issued by a single
// thread, then a commit to `bar`.  The descriptor's start-address field is the
// byte address >> 4 (14 bits hold every shared-memory address), so operand
// offsets are added to base descriptors.
template <int FORM, int S>
__device__ __forceinline__ void issue_stage(const unsigned char *A, const unsigned char *B, uint32_t tmem,
                                            uint64_t *bar)
{
    constexpr int KB = Cfg<FORM>::KB;
    const uint64_t adesc0 = tc::smem_desc(smem_u32(A), 128, 8 * KB);
    const uint64_t bdesc0 = tc::smem_desc(smem_u32(B), 128, 8 * KB);
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
        // pieces with i + j <= S - 1 in FP32 accumulators: hi x hi in kBf16Chunks K-chunks, each
        // later diagonal in one of its own (bf16_acc), summed in FP64 when read
        constexpr uint32_t idesc = tc::idesc_bf16(M, N);
#pragma unroll
        for (int dgl = 0; dgl < S; ++dgl)
#pragma unroll
            for (int i = 0; i <= dgl; ++i) {
                const int j = dgl - i;
#pragma unroll
                for (int ks = 0; ks < Cfg<FORM>::KSTEPS; ++ks) {
                    constexpr int per = Cfg<FORM>::KSTEPS / kBf16Chunks;
                    const bool first = dgl == 0 ? ks % per == 0 : (i == 0 && ks == 0);
                    tc::mma_f16(tmem + 64 * bf16_acc(dgl, ks), adesc0 + j * AS + ks * KS, bdesc0 + i * BS + ks * KS,
                                idesc, !first);
                }
            }
    }
    tc::commit(bar);
}

// TMEM row of this thread (lane m, columns [CW q, CW q + CW)) recombined to doubles.
template <int FORM, int S>
__device__ __forceinline__ void read_row(uint32_t tmem, uint32_t lane_base, int q, const int16_t *escale,
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
                v[8 * h + c] = oz::combine<S>(a) * pow2((int)escale[n] - 12);
            }
        }
    } else {
#pragma unroll
        for (int c = 0; c < CW; ++c)
            v[c] = 0.0;
#pragma unroll
        for (int a = kBf16Chunks + S - 2; a >= 0; --a) { // the small diagonals first
            uint32_t acc[CW];
            tc::ld16(tmem + lane_base + 64 * a + CW * q, acc);
            tc::ld_wait();
#pragma unroll
            for (int c = 0; c < CW; ++c)
                v[c] += (double)__uint_as_float(acc[c]);
        }
    }
}

constexpr int kNoExp = -32768; // exponent slot of an all-zero quarter row

// Power-of-two scale exponent of a row (smallest e with every |value| < 2^e, 0 for a
// zero row) across the 2 parts (lanes m, m^1) and the 4 column quarters (warps w + 4j).
__device__ __forceinline__ int row_exp(const double (&v)[CW], int m, int q, int16_t *sexp)
{
    double mx = 0.0;
#pragma unroll
    for (int c = 0; c < CW; ++c)
        mx = fmax(mx, fabs(v[c]));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    const int e = mx > 0.0 ? exponent_above(mx) : kNoExp;
    sexp[q * 128 + m] = (int16_t)e;
    __syncthreads();
    int r = e;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        r = max(r, (int)sexp[j * 128 + m]);
    return r == kNoExp ? 0 : r;
}

struct Item {
    int64_t ly0, lxa, lxb;
    bool has_b;
};

// A slot of the two-pair pipeline: its current pair (-1: none left), next stage, which half
// of its row exponents belongs to its current operand, and its mbarrier phase.
struct SlotState {
    int64_t w;
    int st, cur;
    uint32_t ph;
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

// Stage-1 operand of a tile pair from global memory: B[y][(part, x)] = tile(part)[y][x]
// with per-row scale exponents in esc[y].  No barrier inside.
template <int FORM, int S>
__device__ __forceinline__ void load_operand(const TileWork &p, const Item &it, unsigned char *B, int16_t *esc,
                                             int tid)
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
        esc[y] = (int16_t)e;
    write_b_row<FORM, S>(B, y, 64 * pp + CW * qq, v, e);
}

// Two-slot software pipeline.  The CTA's tile pairs w = blockIdx.x + k * gridDim.x run
// through SLOTS slots, one pair each, with its own B operand and row exponents; TMEM
// holds the accumulators of one stage of one pair.  As soon as every thread has read a
// slot's accumulators, the MMAs of the other slot's next stage are issued, so they run
// while this slot's values are recombined, multiplied, re-split and written (or stored
// and the slot's next pair loaded).  One MMA group is in flight at a time; all slot
// bookkeeping is block-uniform.
template <int FORM, int S>
__global__ void __launch_bounds__(NT, 1) tc2d_kernel(const TileWork p, const unsigned char *a_slices)
{
    constexpr int SLOTS = slots_for<FORM>(S);
    constexpr int BSZ = S * Cfg<FORM>::B_SLICE;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *A = smem;
    unsigned char *Bbuf = smem + S * Cfg<FORM>::A_SLICE;
    int16_t *escale = reinterpret_cast<int16_t *>(Bbuf + SLOTS * BSZ); // [SLOTS][2][64]
    int16_t *sexp = escale + SLOTS * 128;                               // [4][128]
    uint64_t *bar = reinterpret_cast<uint64_t *>(sexp + 512);          // [SLOTS]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + SLOTS);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int quad = warp & 3, cq = warp >> 2;
    const int m = 32 * quad + lane;       // TMEM lane = D row
    const int f = m >> 1, part = m & 1;   // frequency / position and re-im part of this row
    const uint32_t lane_base = (uint32_t)(32 * quad) << 16;

    {   // constant DFT slices -> shared memory (16-byte copies)
        const uint4 *src = reinterpret_cast<const uint4 *>(a_slices);
        uint4 *dst = reinterpret_cast<uint4 *>(A);
        for (int i = tid; i < S * Cfg<FORM>::A_SLICE / 16; i += NT)
            dst[i] = src[i];
    }
    if (tid == 0) {
        for (int k = 0; k < SLOTS; ++k)
            mbar_init(bar + k, 1);
        fence_barrier_init();
    }
    if (warp == 0)
        tc::tmem_alloc(tslot, 512);

    // slot state, block-uniform (two named states and selects: an array indexed by the
    // slot number would live in local memory)
    int64_t next_w = blockIdx.x;
    SlotState st0{next_w < p.nitems ? next_w : -1, 0, 0, 0}, st1{-1, 0, 0, 0};
    next_w += gridDim.x;
    if (SLOTS == 2) {
        st1.w = next_w < p.nitems ? next_w : -1;
        next_w += gridDim.x;
    }
    if (st0.w >= 0)
        load_operand<FORM, S>(p, item_of(p, st0.w), Bbuf, escale, tid);
    if (st1.w >= 0)
        load_operand<FORM, S>(p, item_of(p, st1.w), Bbuf + BSZ, escale + 128, tid);
    fence_proxy_async_shared();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;
    int inflight = -1;
    if (st0.w >= 0) {
        if (tid == 0)
            issue_stage<FORM, S>(A, Bbuf, tmem, bar);
        inflight = 0;
    }
    bool failed = false;

    while (inflight >= 0) {
        const int c = inflight;
        SlotState cs = c ? st1 : st0; // written back at the end of the step
        const bool ok = mbar_wait_bounded(bar + c, cs.ph);
        cs.ph ^= 1;
        if (__syncthreads_or(!ok) != 0) {
            failed = true;
            break;
        }
        tc::fence_after_sync();
        double v[CW];
        read_row<FORM, S>(tmem, lane_base, cq, escale + c * 128 + cs.cur * 64, v);
        tc::fence_before_sync();
        __syncthreads(); // every thread has read the accumulators: TMEM is free
        inflight = -1;
        if constexpr (SLOTS == 2) {
            const int o = c ^ 1;
            if ((o ? st1.w : st0.w) >= 0) {
                if (tid == 0) {
                    tc::fence_after_sync();
                    issue_stage<FORM, S>(A, Bbuf + o * BSZ, tmem, bar + o);
                }
                inflight = o;
            }
        }
        unsigned char *B = Bbuf + c * BSZ;
        if (cs.st < 3) {
            if (cs.st == 1) { // W' = W * S^tau / 64^2, then conj for the inverse
#pragma unroll
                for (int k = 0; k < CW; ++k) {
                    const double other = __shfl_xor_sync(0xffffffffu, v[k], 1);
                    const double re = part ? other : v[k], im = part ? v[k] : other;
                    const double2 sp = __ldg(p.spec + f * N + CW * cq + k);
                    const double pr_ = re * sp.x - im * sp.y, pi_ = re * sp.y + im * sp.x;
                    v[k] = part ? -pi_ : pr_;
                }
            }
            const int e = row_exp(v, m, cq, sexp);
            if (part == 0 && cq == 0)
                escale[c * 128 + (cs.cur ^ 1) * 64 + f] = (int16_t)e;
            write_b_row<FORM, S>(B, f, 64 * part + CW * cq, v, e);
            cs.cur ^= 1;
            ++cs.st;
        } else { // out[y][x] = conj(D4[(y, part)][x]), crop to the interior
            const Item it = item_of(p, cs.w);
            const int y = f;
            const int64_t gy = it.ly0 + y;
            if (y >= p.halo && y < p.halo + p.useful && gy >= p.vlo[1] && gy < p.vhi[1] &&
                (part == 0 || it.has_b)) {
                const int64_t base = gy * p.nx + (part ? it.lxb : it.lxa);
#pragma unroll
                for (int k = 0; k < CW; ++k) {
                    const int x = CW * cq + k;
                    const int64_t gx = (part ? it.lxb : it.lxa) + x;
                    if (x >= p.halo && x < p.halo + p.useful && gx >= p.vlo[0] && gx < p.vhi[0])
                        p.out[base + x] = part ? -v[k] : v[k];
                }
            }
            // this slot's next pair: its stage-1 operand while the other slot's MMAs run
            cs.w = next_w < p.nitems ? next_w : -1;
            next_w += gridDim.x;
            cs.st = 0;
            cs.cur = 0;
            if (cs.w >= 0)
                load_operand<FORM, S>(p, item_of(p, cs.w), B, escale + c * 128, tid);
        }
        fence_proxy_async_shared();
        tc::fence_before_sync();
        __syncthreads(); // slot c's operand is complete
        if (c)
            st1 = cs;
        else
            st0 = cs;
        if (inflight < 0 && cs.w >= 0) {
            if (tid == 0) {
                tc::fence_after_sync();
                issue_stage<FORM, S>(A, B, tmem, bar + c);
            }
            inflight = c;
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
