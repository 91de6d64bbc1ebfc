// FP64 fused DFT-tile stencil kernel for 1D grids on the FP64 pipe (four-step
// DFT-4096 of radix-8 butterflies, no tensor cores).
//
// Tile 4096 = 64 x 64 (same geometry, halo and band as the DMMA form), two real tiles
// packed as one complex tile (re = tile a, im = tile b).  The tile is held as the
// 64 x 64 work matrix W[b][a] = x[64 a + b], and
//   X[k1 + 64 k2] = sum_b w64^(b k2) w4096^(b k1) sum_a x[64 a + b] w64^(a k1):
//   A. rows b: forward DFT-64 over a (-> k1), times w4096^(b k1);
//   B. columns k1: forward DFT-64 over b (-> k2), spectrum S[k1 + 64 k2], inverse;
//   C. rows b: times w4096^(-b k1), inverse DFT-64 over k1 (-> a), cropped stores of
//      x[64 a + b].
// Each DFT-64 is the shared radix-8 group code (ffs_fft64.cuh).  The twiddle is
// w4096^(b (j + 8 k)) = T1[b j] T2[b k] (w4096^m, m < 448; w512^m), from the plan's
// tables.  Staging: each 64-point row of both tiles is one 512-byte bulk copy into a
// row of 66 doubles (528 B), so the column-strided reads of pass A hit 16 distinct
// bank pairs per half warp; edge tiles take plain loads into the same layout.  The
// spectrum is the Hermitian half k = 0..2048 at slot k + (k >> 6) (conflict-free for
// the column reads of pass B).
// Replaces rfft_pfa_stencil_8_nwarp (src/1D/rfftstencil_pfa/rfft_8_pfa_fastcomplex.cu:
// 17-340) like the DMMA form does.
#include "ffs_dmma1d.cuh"
#include "ffs_fft64.cuh"

namespace ffst {
namespace fft1d {

using fft64::Twiddle;
using fft64::widx;
constexpr int N = 64;
constexpr int TILE = N * N;
constexpr int NT = 512; // 64 groups of 8 threads: one line each per pass
constexpr int PITCH = 66; // doubles per staged row (528 B: 16-byte aligned, 4 banks of skew)
constexpr int PLANE = N * PITCH;
constexpr size_t STAGE_BYTES = 2ull * PLANE * sizeof(double);
constexpr size_t WORK_BYTES = (size_t)TILE * sizeof(double2);
constexpr int HALF_SLOTS = 2088; // k = 0..2048 at slot k + (k >> 6) <= 2080, rounded up to a multiple of 8
constexpr size_t SPEC_BYTES = (size_t)HALF_SLOTS * sizeof(double2);
constexpr int T1N = dmma1d::T1N, T2N = dmma1d::T2N;
constexpr size_t TW_BYTES = (size_t)(T1N + T2N) * sizeof(double2);
constexpr size_t SMEM_BYTES = STAGE_BYTES + WORK_BYTES + SPEC_BYTES + TW_BYTES + 16;
static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");

__device__ __forceinline__ int sslot(int k) { return k + (k >> 6); }

// Staged tiles: whole 4096-point tiles inside the grid are bulk-copied row by row.
__device__ __forceinline__ bool rows_ok(const TileWork &p, const dmma1d::Item &it)
{
    if (!p.use_tma)
        return false;
    const bool ain = it.lxa >= 0 && it.lxa + TILE <= p.nx;
    const bool bin = !it.has_b || (it.lxb >= 0 && it.lxb + TILE <= p.nx);
    return ain && bin;
}

// Plain loads of item `it` into the staging layout; zeros outside a fixed-boundary
// grid, periodic wrap otherwise.  All loads of a thread before its first store.
__device__ __forceinline__ void fill_stage(double *stage, const TileWork &p, const dmma1d::Item &it, int tid)
{
    constexpr int PER = TILE / NT;
    double re[PER], im[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        int64_t ga = it.lxa + i, gb = it.lxb + i;
        bool aok = ga >= 0 && ga < p.nx, bok = it.has_b && gb >= 0 && gb < p.nx;
        if (p.periodic) {
            ga = wrap_near(ga, p.nx);
            gb = wrap_near(gb, p.nx);
            aok = true;
            bok = it.has_b;
        }
        re[k] = aok ? __ldcg(p.in + ga) : 0.0;
        im[k] = bok ? __ldcg(p.in + gb) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int i = tid + k * NT;
        const int s = (i >> 6) * PITCH + (i & 63);
        stage[s] = re[k];
        stage[PLANE + s] = im[k];
    }
}

__device__ __forceinline__ void twiddle(double &re, double &im, const double2 *t1, const double2 *t2, int b, int j,
                                        int k, bool conj)
{
    const double2 u = t1[b * j], v = t2[b * k];
    double wr = u.x * v.x - u.y * v.y, wi = u.x * v.y + u.y * v.x;
    cmul(re, im, wr, conj ? -wi : wi);
}

__global__ void __launch_bounds__(NT, 1) fft1d_kernel(const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double *stage = reinterpret_cast<double *>(smem);
    double2 *work = reinterpret_cast<double2 *>(smem + STAGE_BYTES);
    double2 *spec = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES);
    double2 *t1 = reinterpret_cast<double2 *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES);
    double2 *t2 = t1 + T1N;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGE_BYTES + WORK_BYTES + SPEC_BYTES + TW_BYTES);
    uint64_t *cbar = bar + 1; // spectrum and twiddle tables

    const int tid = threadIdx.x, q = tid >> 3, j = tid & 7, lane = tid & 31;
    const unsigned gmask = 0xffu << (tid & 24);
    int64_t w = blockIdx.x;
    if (w >= p.nitems)
        return; // (the grid never exceeds the pair count; nothing was issued)
    // the 128 row copies of a pair: warp 0 issues them after its lane 0 set the byte count
    auto issue = [&](const dmma1d::Item &it) {
        if (lane == 0) {
            fence_proxy_async_shared();
            mbar_arrive_expect_tx(bar, (uint32_t)((it.has_b ? 2 : 1) * TILE * sizeof(double)));
        }
        __syncwarp();
        for (int r = lane; r < 2 * N; r += 32) {
            const int t = r >> 6, row = r & 63;
            if (t == 1 && !it.has_b)
                continue;
            bulk_load(stage + t * PLANE + row * PITCH, p.in + (t ? it.lxb : it.lxa) + row * N,
                      (uint32_t)(N * sizeof(double)), bar);
        }
    };
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(cbar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid < 32) {
        const dmma1d::Item it = dmma1d::item_of(p, w);
        if (rows_ok(p, it))
            issue(it);
        if (tid == 0) { // constants behind the first pair's rows
            mbar_arrive_expect_tx(cbar, (uint32_t)(SPEC_BYTES + TW_BYTES));
            bulk_load(spec, p.spec, (uint32_t)SPEC_BYTES, cbar);
            bulk_load(t1, p.tables + 8 + 64, (uint32_t)TW_BYTES, cbar);
        }
    }
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
    uint32_t phase = 0;
    bool consts_ready = false;
    for (; w < p.nitems; w += gridDim.x) {
        const dmma1d::Item it = dmma1d::item_of(p, w);
        if (rows_ok(p, it)) {
            if (!mbar_wait_bounded(bar, phase)) {
                record_error(p.status, kDevTimeoutTma);
                if (!consts_ready)
                    (void)mbar_wait_bounded(cbar, 0);
                return;
            }
            phase ^= 1;
        } else {
            fill_stage(stage, p, it, tid);
            __syncthreads();
        }
        if (!consts_ready) {
            if (!mbar_wait_bounded(cbar, 0)) {
                record_error(p.status, kDevTimeoutTma);
                return;
            }
            consts_ready = true;
        }
        double xr[8], xi[8];
        { // A: row b = q: x[64 a + b] for a = 8 i + j, forward over a, times w4096^(b k1)
            const int b = q;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int s = (8 * i + j) * PITCH + b;
                xr[i] = stage[s];
                xi[i] = it.has_b ? stage[PLANE + s] : 0.0; // (a lone tile's partner plane is not copied)
            }
            auto slot = [&](int x) { return widx(b, x); };
            fft64::dft64_line<false>(xr, xi, tw, j, work, slot, gmask);
#pragma unroll
            for (int k = 0; k < 8; ++k) { // k1 = j + 8 k
                twiddle(xr[k], xi[k], t1, t2, b, j, k, false);
                work[widx(b, j + 8 * k)] = make_double2(xr[k], xi[k]);
            }
        }
        __syncthreads();
        // the staged rows are consumed: warp 0 starts the next pair's copies
        if (tid < 32 && w + gridDim.x < p.nitems) {
            const dmma1d::Item nx_it = dmma1d::item_of(p, w + gridDim.x);
            if (rows_ok(p, nx_it))
                issue(nx_it);
        }
        { // B: column k1 = c: forward over b (-> k2), spectrum, inverse
            const int c = q;
            auto slot = [&](int y) { return widx(y, c); };
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const double2 v = work[widx(8 * a + j, c)];
                xr[a] = v.x;
                xi[a] = v.y;
            }
            fft64::dft64_line<false>(xr, xi, tw, j, work, slot, gmask);
#pragma unroll
            for (int k = 0; k < 8; ++k) { // frequency c + 64 (j + 8 k); > 2048 reads conj S[4096 - k]
                const int f = c + 64 * (j + 8 * k);
                const bool upper = f > TILE / 2;
                const double2 s = spec[sslot(upper ? TILE - f : f)];
                cmul(xr[k], xi[k], s.x, upper ? -s.y : s.y);
            }
            fft64::dft64_line<true>(xr, xi, tw, j, work, slot, gmask);
#pragma unroll
            for (int k = 0; k < 8; ++k)
                work[widx(j + 8 * k, c)] = make_double2(xr[k], xi[k]);
        }
        __syncthreads();
        { // C: row b = q: times w4096^(-b k1), inverse over k1 (-> a), x[64 a + b]
            const int b = q;
#pragma unroll
            for (int i = 0; i < 8; ++i) { // k1 = 8 i + j
                const double2 v = work[widx(b, 8 * i + j)];
                xr[i] = v.x;
                xi[i] = v.y;
                twiddle(xr[i], xi[i], t1, t2, b, j, i, true);
            }
            auto slot = [&](int x) { return widx(b, x); };
            fft64::dft64_line<true>(xr, xi, tw, j, work, slot, gmask);
#pragma unroll
            for (int k = 0; k < 8; ++k) { // a = j + 8 k: position 64 a + b
                const int pos = 64 * (j + 8 * k) + b;
                if (pos < p.halo || pos >= p.halo + p.useful)
                    continue;
                const int64_t ga = it.lxa + pos, gb = it.lxb + pos;
                if (ga >= p.vlo[0] && ga < p.vhi[0])
                    p.out[ga] = xr[k];
                if (it.has_b && gb >= p.vlo[0] && gb < p.vhi[0])
                    p.out[gb] = xi[k];
            }
        }
        __syncthreads();
    }
}

} // namespace fft1d

size_t fft1d_smem_bytes() { return fft1d::SMEM_BYTES; }

cudaError_t prepare_fft1d()
{
    return cudaFuncSetAttribute(fft1d::fft1d_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fft1d::SMEM_BYTES);
}

cudaError_t launch_fft1d(const TileWork &w, int grid, cudaStream_t s)
{
    fft1d::fft1d_kernel<<<grid, fft1d::NT, fft1d::SMEM_BYTES, s>>>(w);
    return cudaGetLastError();
}

} // namespace ffst
