// FP64 fused DFT-tile stencil kernel for 1D grids (plain form, DMMA).
//
// Tile n = 4096 = 64 x 64 cells (tile-local index j = 64a + b), two tiles
// adjacent along x packed as one complex tile.  The 4096-point DFT is the
// four-step form: a DFT-64 over a for every b (each DFT-64 two radix-8
// mma.sync.m8n8k4.f64 stages), the 4096th-root twiddle w^(b*k1), then per k1
// a DFT-64 over b, the spectrum^tau multiply and the inverse DFT-64 over b,
// the conjugate twiddle, and the inverse DFT-64 back to a.  The interior
// u = 4096 - 2*halo cells are stored with coalesced writes.
//
// Replaces rfft_pfa_stencil_8_nwarp (src/1D/rfftstencil_pfa/rfft_8_pfa_fastcomplex.cu:17-340),
// which runs one 56-point prime-factor tile (8 x 7) per warp with a random
// 29/31-tap kernel standing in for 14/7/5 fused steps and atomics on overlap.
#include <cstring>

#include "ffs_device.cuh"
#include "ffs_kernels.h"
#include "ffs_radix64.cuh"

namespace ffst {
namespace dmma1d {

using namespace r64;
constexpr int TILE = N * N; // 4096
constexpr int NT = 512;
constexpr int NWARP = NT / 32;
constexpr int T1N = 448; // w4096^m, m <= 63*7
constexpr int T2N = 512; // w512^m
constexpr size_t STAGE_BYTES = 2ull * TILE * sizeof(double);
constexpr size_t WORK_BYTES = (size_t)TILE * sizeof(double2);
constexpr size_t SPEC_BYTES = (size_t)TILE * sizeof(double2);
constexpr size_t TW_BYTES = (size_t)(T1N + T2N) * sizeof(double2);
constexpr size_t SMEM_BYTES = STAGE_BYTES + WORK_BYTES + SPEC_BYTES + TW_BYTES + 16;

// Natural-order (a, b) slot used for the cropped write-back; conflict-free for
// the per-lane writes (a = g + 16t + 8e, fixed b) and for row-contiguous reads.
__device__ __forceinline__ int nat_idx(int a, int b) { return a * N + (b ^ ((a & 1) | ((a >> 3) & 6))); }

struct Item {
    int64_t lxa, lxb;
    bool has_b;
};

__device__ __forceinline__ Item item_of(const TileWork &p, int64_t w)
{
    Item it;
    const int64_t txa = p.t0[0] + 2 * w;
    it.has_b = (2 * w + 1) < p.nt[0];
    it.lxa = txa * p.useful - p.halo;
    it.lxb = it.lxa + p.useful;
    return it;
}

__device__ __forceinline__ bool bulk_ok(const TileWork &p, const Item &it)
{
    if (!p.use_tma)
        return false;
    const bool ain = it.lxa >= 0 && it.lxa + TILE <= p.nx;
    const bool bin = !it.has_b || (it.lxb >= 0 && it.lxb + TILE <= p.nx);
    return ain && bin;
}

__device__ __forceinline__ int64_t wrapi(int64_t i, int64_t n)
{
    i %= n;
    return i < 0 ? i + n : i;
}

// w4096^(b*k1) with k1 = g + 8*c2: T1[b*g] * T2[b*c2]
__device__ __forceinline__ void tw4096(const double2 *t1, const double2 *t2, int b, int g, int c2, double &wr,
                                       double &wi)
{
    const double2 x = t1[b * g];
    const double2 y = t2[(b * c2) & (T2N - 1)];
    wr = x.x * y.x - x.y * y.y;
    wi = x.x * y.y + x.y * y.x;
}

struct FwdTwiddle {
    const double2 *t1, *t2;
    int g, t;
    __device__ __forceinline__ void operator()(int b, double re[2], double im[2]) const
    {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            double wr, wi;
            tw4096(t1, t2, b, g, 2 * t + e, wr, wi);
            cmul(re[e], im[e], wr, wi);
        }
    }
};

__global__ void __launch_bounds__(NT, 1) dmma1d_kernel(const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double *stage = reinterpret_cast<double *>(smem);
    double2 *work = reinterpret_cast<double2 *>(smem + STAGE_BYTES);
    double2 *spec = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES);
    double2 *t1 = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES);
    double2 *t2 = t1 + T1N;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES + TW_BYTES);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    for (int i = tid; i < TILE; i += NT)
        spec[i] = p.spec[i];
    for (int i = tid; i < T1N + T2N; i += NT)
        t1[i] = p.tables[8 + 64 + i];
    const LaneConst c = lane_consts(p.tables, p.tables + 8, g, t);
    __syncthreads();

    auto issue = [&](const Item &it) {
        fence_proxy_async_shared();
        mbar_arrive_expect_tx(bar, it.has_b ? (uint32_t)STAGE_BYTES : (uint32_t)(STAGE_BYTES / 2));
        bulk_load(stage, p.in + it.lxa, TILE * sizeof(double), bar);
        if (it.has_b)
            bulk_load(stage + TILE, p.in + it.lxb, TILE * sizeof(double), bar);
    };

    uint32_t phase = 0;
    int64_t w = blockIdx.x;
    if (tid == 0 && w < p.nitems) {
        const Item it = item_of(p, w);
        if (bulk_ok(p, it))
            issue(it);
    }
    for (; w < p.nitems; w += gridDim.x) {
        const Item it = item_of(p, w);
        // stage -> work, transposed: SMEM row b holds the line a = 0..63 of x[64a + b]
        if (bulk_ok(p, it)) {
            if (!mbar_wait_bounded(bar, phase)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            phase ^= 1;
            for (int i = tid; i < TILE; i += NT) {
                const int a = i >> 6, b = i & 63;
                work[widx(b, a)] = make_double2(stage[i], it.has_b ? stage[TILE + i] : 0.0);
            }
        } else {
            for (int i = tid; i < TILE; i += NT) {
                const int a = i >> 6, b = i & 63;
                const int64_t ga = it.lxa + i, gb = it.lxb + i;
                double re = 0.0, im = 0.0;
                if (p.periodic) {
                    re = p.in[wrapi(ga, p.nx)];
                    if (it.has_b)
                        im = p.in[wrapi(gb, p.nx)];
                } else {
                    if (ga >= 0 && ga < p.nx)
                        re = p.in[ga];
                    if (it.has_b && gb >= 0 && gb < p.nx)
                        im = p.in[gb];
                }
                work[widx(b, a)] = make_double2(re, im);
            }
        }
        __syncthreads();
        if (tid == 0 && w + gridDim.x < p.nitems) {
            const Item nx_it = item_of(p, w + gridDim.x);
            if (bulk_ok(p, nx_it))
                issue(nx_it);
        }
        // 1. DFT-64 over a for every b, then w4096^(b*k1)
        const FwdTwiddle fwd{t1, t2, g, t};
#pragma unroll 1
        for (int k = 0; k < N / NWARP; k += 2) {
            row_forward(work, warp + NWARP * k, c, g, t, fwd);
            row_forward(work, warp + NWARP * (k + 1), c, g, t, fwd);
        }
        __syncthreads();
        // 2. per k1: DFT-64 over b, spectrum, inverse DFT-64 over b
#pragma unroll 1
        for (int k = 0; k < N / NWARP; ++k)
            column_pass(work, spec, warp + NWARP * k, c, g, t);
        __syncthreads();
        // 3. conj twiddle and inverse DFT-64 over k1 -> a; load every row first, then
        //    write natural order over the same buffer
        double bre[N / NWARP][2], bim[N / NWARP][2];
#pragma unroll
        for (int k = 0; k < N / NWARP; ++k) {
            const int b = warp + NWARP * k;
            row_inverse_load(work, b, g, t, bre[k], bim[k]);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                double wr, wi;
                tw4096(t1, t2, b, g, t + 4 * j, wr, wi);
                cmul(bre[k][j], bim[k][j], wr, -wi);
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < N / NWARP; ++k) {
            const int b = warp + NWARP * k;
            double ore[2], oim[2];
            row_inverse_compute(c, bre[k], bim[k], ore, oim);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int a = g + 8 * (2 * t + e);
                work[nat_idx(a, b)] = make_double2(ore[e], oim[e]);
            }
        }
        __syncthreads();
        // 4. cropped, coalesced store of the interior
        for (int i = tid; i < TILE; i += NT) {
            if (i < p.halo || i >= p.halo + p.useful)
                continue;
            const double2 v = work[nat_idx(i >> 6, i & 63)];
            const int64_t ga = it.lxa + i, gb = it.lxb + i;
            if (ga >= p.vlo[0] && ga < p.vhi[0])
                p.out[ga] = v.x;
            if (it.has_b && gb >= p.vlo[0] && gb < p.vhi[0])
                p.out[gb] = v.y;
        }
        __syncthreads();
    }
}

} // namespace dmma1d

size_t dmma1d_smem_bytes() { return dmma1d::SMEM_BYTES; }
int dmma1d_tile() { return dmma1d::TILE; }

cudaError_t prepare_dmma1d()
{
    return cudaFuncSetAttribute(dmma1d::dmma1d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dmma1d::SMEM_BYTES);
}

cudaError_t launch_dmma1d(const TileWork &w, int grid, cudaStream_t s)
{
    dmma1d::dmma1d_kernel<<<grid, dmma1d::NT, dmma1d::SMEM_BYTES, s>>>(w);
    return cudaGetLastError();
}

} // namespace ffst
