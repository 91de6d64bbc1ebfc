// FP64 fused DFT-tile stencil kernel for 3D grids with a 32^3 tile held across a
// cluster of four CTAs in distributed shared memory (butterflies on the FP64 pipe).
//
// A 32^3 complex tile pair (re = tile a, im = tile b, 512 KB) does not fit one SM's
// shared memory, so the four CTAs of a cluster (one per SM) each hold 8 of its 32
// planes, 128 KB, and transform the axes whose lines they hold; the third axis is
// read across the cluster.  A DFT-32 line fits one thread's registers
// (ffs_dft32.cuh), so every transform is one thread per line, 256 lines per CTA:
//   Z.  thread (yl, x) of CTA c loads column (y = 8c + yl, x) of both real tiles over
//       z (a warp reads two whole 256-byte rows per instruction), forward along z,
//       into plane slab A: slot (z, yl, x);
//   X.  thread (z, yl): forward along x in place;
//   --  cluster barrier: every CTA's slab holds the z- and x-transformed planes;
//   Y.  thread (zl, x) of CTA c gathers the y line at kz = 8c + zl, kx = x from all
//       four CTAs' slabs (ld.shared::cluster), forward along y, times the spectrum
//       S^tau / 32^3 (natural order, read through L1/L2 coalesced along kx), inverse
//       along y, and keeps the wanted y positions;
//   --  cluster barrier: no CTA reads the A slabs any more;
//   the wanted y positions go to slab B: slot (zl, yu, x);
//   X'. thread (zl, yu): inverse along x, the wanted x written back;
//   --  cluster barrier;
//   Z'. each wanted (y, x) column, a quarter of them per CTA, gathered over z from
//       all four CTAs, inverse along z, cropped stores;
//   --  cluster barrier before the next pair overwrites the slabs.
// Against the 16^3 tile (ffs_fft3d.cu) the halo costs less: at tau 2 (halo 2) a
// pair yields 2 * 28^3 cells for 2 * 32^3 loaded, against 2 * 12^3 for 2 * 16^3, so
// there are 21 % fewer butterfly operations and 37 % fewer loaded cells per output
// cell and pass; at tau 4 (halo 4, 24^3 kept) the pass count halves.
// Slot swizzles: line L of a slab holds its 32 points at L * 32 + (x ^ (L & 7)), so
// a quarter warp reading one point of 8 consecutive lines, or 8 consecutive points
// of one line, touches 8 distinct 16-byte bank groups.
// Same tile geometry (item_of), halo, crop and band as the 16^3 forms, with n = 32.
// Replaces rfft_3d_8_nwarp (src/3D/rfft_3d/3d_rfft_N.cu:17-303) like the 16^3 forms.
#include <algorithm>

#include "ffs_dft32.cuh"
#include "ffs_dmma3d.cuh"

namespace ffst {
namespace fft3d32 {

constexpr int N = 32;
constexpr int CL = 4;       // CTAs per cluster
constexpr int PL = N / CL;  // planes per CTA
constexpr int NT = 256;     // one thread per line
constexpr size_t SLAB_BYTES = (size_t)N * PL * N * sizeof(double2); // 128 KB
static_assert(PL * N == NT, "one thread per line of a slab");

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_index()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_count()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
// All threads of all CTAs of the cluster; release/acquire orders the shared-memory
// writes before it with the cluster-wide reads after it.
__device__ __forceinline__ void cluster_sync()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t map_to_rank(uint32_t saddr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}
__device__ __forceinline__ double2 ld_cluster(uint32_t addr)
{
    double2 v;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr) : "memory");
    return v;
}

// slot of point i of slab line L
__device__ __forceinline__ int slot(int L, int i) { return (L << 5) | (i ^ (L & 7)); }

// Column (y, x) of item `it` over z = 0..31 into registers: re from tile a, im from
// tile b; zeros outside a fixed-boundary grid, periodic wrap otherwise.
__device__ __forceinline__ void load_column(double (&re)[N], double (&im)[N], const TileWork &p,
                                            const dmma3d::Item &it, int y, int x)
{
    const bool inside = it.lz >= 0 && it.lz + N <= p.nz && it.ly >= 0 && it.ly + N <= p.ny && it.lx >= 0 &&
                        (it.has_b ? it.lxb + N : it.lx + N) <= p.nx;
    if (inside) { // the whole pair lies in the grid
        const int64_t plane = p.ny * p.nx;
        const double *base = p.in + (it.lz * p.ny + it.ly + y) * p.nx;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            re[k] = __ldcg(base + k * plane + it.lx + x);
            im[k] = it.has_b ? __ldcg(base + k * plane + it.lxb + x) : 0.0;
        }
        return;
    }
    int64_t gy = it.ly + y, ga = it.lx + x, gb = it.lxb + x;
    bool yok = gy >= 0 && gy < p.ny, aok = ga >= 0 && ga < p.nx, bok = it.has_b && gb >= 0 && gb < p.nx;
    if (p.periodic) {
        gy = wrap_near(gy, p.ny);
        ga = wrap_near(ga, p.nx);
        gb = wrap_near(gb, p.nx);
        yok = aok = true;
        bok = it.has_b;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        int64_t gz = it.lz + k;
        bool zok = gz >= 0 && gz < p.nz;
        if (p.periodic) {
            gz = wrap_near(gz, p.nz);
            zok = true;
        }
        const double *row = p.in + (gz * p.ny + gy) * p.nx;
        re[k] = (zok && yok && aok) ? __ldcg(row + ga) : 0.0;
        im[k] = (zok && yok && bok) ? __ldcg(row + gb) : 0.0;
    }
}

__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(NT, 1) fft3d32_kernel(const TileWork p)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    double2 *slab = reinterpret_cast<double2 *>(smem);
    const int c = (int)cluster_rank();
    uint32_t peer[CL]; // the slab of each CTA of the cluster, in the cluster's shared window
#pragma unroll
    for (int r = 0; r < CL; ++r)
        peer[r] = map_to_rank(smem_u32(slab), (uint32_t)r);
    const int t = threadIdx.x;
    const int u0 = p.halo, u = p.useful, u1 = p.halo + p.useful; // wanted local positions per axis
    double xr[N], xi[N];
    // every CTA of a cluster takes the same items, so all reach the same cluster barriers
    for (int64_t w = cluster_index(); w < p.nitems; w += cluster_count()) {
        const dmma3d::Item it = dmma3d::item_of(p, w);
        { // Z: column (y, x) = (PL c + yl, x), forward along z, into slab line (z, yl)
            const int yl = t >> 5, x = t & 31;
            load_column(xr, xi, p, it, PL * c + yl, x);
            dft32::dft32<false>(xr, xi);
#pragma unroll
            for (int z = 0; z < N; ++z)
                slab[slot(z * PL + yl, x)] = make_double2(xr[z], xi[z]);
        }
        __syncthreads();
        { // X: line L = (z, yl) = t, forward along x in place
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double2 v = slab[slot(t, i)];
                xr[i] = v.x;
                xi[i] = v.y;
            }
            dft32::dft32<false>(xr, xi);
#pragma unroll
            for (int i = 0; i < N; ++i)
                slab[slot(t, i)] = make_double2(xr[i], xi[i]);
        }
        cluster_sync();
        const int zl = t >> 5, x = t & 31;
        { // Y: the y line at (kz, kx) = (PL c + zl, x) from the four slabs
            const int kz = PL * c + zl;
#pragma unroll
            for (int r = 0; r < CL; ++r)
#pragma unroll
                for (int yl = 0; yl < PL; ++yl) {
                    const double2 v = ld_cluster(peer[r] + 16u * (uint32_t)slot(kz * PL + yl, x));
                    xr[PL * r + yl] = v.x;
                    xi[PL * r + yl] = v.y;
                }
            dft32::dft32<false>(xr, xi);
            const double2 *sp = p.spec + (size_t)kz * N * N + x; // S(kz, ky, kx) at (kz * 32 + ky) * 32 + kx
#pragma unroll
            for (int ky = 0; ky < N; ++ky) {
                const double2 s = __ldg(sp + ky * N);
                cmul(xr[ky], xi[ky], s.x, s.y);
            }
            dft32::dft32<true>(xr, xi);
        }
        cluster_sync();
        // the wanted y positions into slab B: line (zl, yu) = zl * u + yu
#pragma unroll
        for (int y = 0; y < N; ++y)
            if (y >= u0 && y < u1)
                slab[slot(zl * u + (y - u0), x)] = make_double2(xr[y], xi[y]);
        __syncthreads();
        if (t < PL * u) { // X': line (zl, yu) = t, inverse along x, the wanted x written back
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double2 v = slab[slot(t, i)];
                xr[i] = v.x;
                xi[i] = v.y;
            }
            dft32::dft32<true>(xr, xi);
#pragma unroll
            for (int i = 0; i < N; ++i)
                if (i >= u0 && i < u1)
                    slab[slot(t, i)] = make_double2(xr[i], xi[i]);
        }
        cluster_sync();
        { // Z': wanted column j = (yu, xu), a quarter per CTA, gathered over z, inverse along z
            const int per = (u * u + CL - 1) / CL;
            const int j = c * per + t;
            if (t < per && j < u * u) {
                const int yu = j / u, xu = j - yu * u;
                const int64_t gy = it.ly + u0 + yu, ga = it.lx + u0 + xu, gb = it.lxb + u0 + xu;
                const bool a_ok = ga >= p.vlo[0] && ga < p.vhi[0];
                const bool b_ok = it.has_b && gb >= p.vlo[0] && gb < p.vhi[0];
                if (gy >= p.vlo[1] && gy < p.vhi[1] && (a_ok || b_ok)) {
#pragma unroll
                    for (int r = 0; r < CL; ++r)
#pragma unroll
                        for (int zz = 0; zz < PL; ++zz) {
                            const double2 v = ld_cluster(peer[r] + 16u * (uint32_t)slot(zz * u + yu, u0 + xu));
                            xr[PL * r + zz] = v.x;
                            xi[PL * r + zz] = v.y;
                        }
                    dft32::dft32<true>(xr, xi);
#pragma unroll
                    for (int z = 0; z < N; ++z) {
                        const int64_t gz = it.lz + z;
                        if (z < u0 || z >= u1 || gz < p.vlo[2] || gz >= p.vhi[2])
                            continue;
                        double *row = p.out + (gz * p.ny + gy) * p.nx;
                        if (a_ok)
                            row[ga] = xr[z];
                        if (b_ok)
                            row[gb] = xi[z];
                    }
                }
            }
        }
        cluster_sync(); // the next pair overwrites the slabs the other CTAs read above
    }
}

int g_max_clusters[64]; // per device: clusters of this kernel that fit at once (0 = not queried)

} // namespace fft3d32

size_t fft3d32_smem_bytes() { return fft3d32::SLAB_BYTES; }

cudaError_t prepare_fft3d32()
{
    cudaError_t e = cudaFuncSetAttribute(fft3d32::fft3d32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fft3d32::SLAB_BYTES);
    int dev = 0;
    if (e == cudaSuccess)
        e = cudaGetDevice(&dev);
    if (e == cudaSuccess && dev >= 0 && dev < 64) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(fft3d32::CL * 64, 1, 1);
        cfg.blockDim = dim3(fft3d32::NT, 1, 1);
        cfg.dynamicSmemBytes = fft3d32::SLAB_BYTES;
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, fft3d32::fft3d32_kernel, &cfg) == cudaSuccess && n > 0)
            fft3d32::g_max_clusters[dev] = n;
        else
            (void)cudaGetLastError(); // the launch then assumes one cluster per four SMs
    }
    return e;
}

// `num_sms` bounds the clusters when the occupancy query was not made.
cudaError_t launch_fft3d32(const TileWork &w, int num_sms, cudaStream_t s)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    const int fit = (dev >= 0 && dev < 64 && fft3d32::g_max_clusters[dev] > 0) ? fft3d32::g_max_clusters[dev]
                                                                                : num_sms / fft3d32::CL;
    const int64_t clusters = std::max<int64_t>(1, std::min<int64_t>(w.nitems, fit));
    fft3d32::fft3d32_kernel<<<(int)(clusters * fft3d32::CL), fft3d32::NT, fft3d32::SLAB_BYTES, s>>>(w);
    return cudaGetLastError();
}

} // namespace ffst
