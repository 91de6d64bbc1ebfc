// Host-side launch interface of the sm_100a kernels (internal to libffs.so).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ffst {

// Codes a kernel writes into the plan's device status word.
enum DeviceError : int {
    kDevOk = 0,
    kDevTimeoutTma = 1,
    kDevTimeoutMma = 2,
    kDevBadConfig = 3,
    kDevTimeoutDep = 4,
};

// Tile-pair work description shared by the fused DFT-tile kernels.  Tiles of
// edge n overlap by `halo` cells per side; each produces a u = n - 2*halo edge of
// outputs.  Two tiles adjacent along x are packed as the real and imaginary
// parts of one complex tile (the reference's "two real tiles per complex tile",
// src/2D/rfft_2d/2d_rfft_1_async.cu:73-92).
struct TileWork {
    const double *in;
    double *out;
    const double2 *spec;   // spectrum^tau / n^d, in the kernel's frequency-position order
    const double2 *tables; // DFT-8 roots (8) then n-th roots of unity (n or n^2 for 1D)
    int *status;           // device error word (0 = ok)
    int64_t nx, ny, nz;
    int halo, useful;
    int64_t t0[3];   // first tile index per dim (x, y, z)
    int64_t nt[3];   // tiles per dim in the range (x, y, z)
    int64_t npx;     // tile pairs along x = ceil(nt[0] / 2)
    int64_t nitems;  // npx * nt[1] * nt[2]
    int64_t vlo[3], vhi[3]; // store window per dim (spectrally exact cells)
    int periodic;
    int use_tma;
};

cudaError_t prepare_dmma2d(); // sets the shared-memory attribute on the current device
cudaError_t launch_dmma2d(const CUtensorMap *tmap, const TileWork &w, int grid, cudaStream_t s);
size_t dmma2d_smem_bytes();
int dmma2d_tile();

// 2D FP64 radix-8 butterfly form (same tile geometry and spectrum layout as tc2d).
cudaError_t prepare_fft2d();
cudaError_t launch_fft2d(const CUtensorMap *tmap, const TileWork &w, int grid, cudaStream_t s);
size_t fft2d_smem_bytes();

// 3D FP64 butterfly form (two CTAs per SM; `grid` is the SM count bound).
cudaError_t prepare_fft3d();
cudaError_t launch_fft3d(const TileWork &w, int grid, cudaStream_t s);
int64_t fft3d_grid(int64_t nitems, int num_sms); // the CTA count launch_fft3d uses
size_t fft3d_smem_bytes();
// 2D FP64 butterfly form on one 128 x 128 real tile per CTA (single tiles, not pairs).
cudaError_t prepare_fft2d128();
cudaError_t launch_fft2d128(const TileWork &w, int grid, cudaStream_t s);
size_t fft2d128_smem_bytes();
// 3D FP64 butterfly form on a 32^3 tile held by a cluster of four CTAs (one per SM).
cudaError_t prepare_fft3d32();
cudaError_t launch_fft3d32(const TileWork &w, int num_sms, cudaStream_t s);
size_t fft3d32_smem_bytes();

// 1D FP64 butterfly form (four-step DFT-4096 of radix-8 lines).
cudaError_t prepare_fft1d();
cudaError_t launch_fft1d(const TileWork &w, int grid, cudaStream_t s);
size_t fft1d_smem_bytes();

cudaError_t prepare_dmma1d();
cudaError_t launch_dmma1d(const TileWork &w, int grid, cudaStream_t s);
size_t dmma1d_smem_bytes();
int dmma1d_tile();

cudaError_t prepare_dmma3d();
cudaError_t launch_dmma3d(const CUtensorMap *tmap, const TileWork &w, int grid, cudaStream_t s);
size_t dmma3d_smem_bytes();
int dmma3d_tile();

// tcgen05 2D and 3D forms (Ozaki INT8 slices / 3-way BF16 split).
constexpr int kFormOzaki = 2;
constexpr int kFormBf16 = 3;
cudaError_t prepare_tc2d();
cudaError_t launch_tc2d(int form, int slices, const TileWork &w, const unsigned char *a_slices, int grid,
                        cudaStream_t s);
size_t tc2d_smem_bytes(int form, int slices);
cudaError_t prepare_tc3d();
cudaError_t launch_tc3d(int form, int slices, const TileWork &w, const unsigned char *f_slices, int grid,
                        cudaStream_t s);
size_t tc3d_smem_bytes(int form, int slices);

// Direct FP64 time stepping of boxes near a fixed boundary.
struct BandBox {
    int64_t lo[3]; // box origin (x, y, z)
    int32_t ext[3]; // box extents
};
struct BandWork {
    const double *in;
    double *out;
    const double *weights; // dense (2r+1)^dim, device
    const BandBox *boxes;
    int nboxes;
    int dim, r, tau;
    int64_t n[3];
    int64_t max_vol;       // largest staged region (box + halo) over all boxes, in cells
    const int4 *taps;      // non-zero taps: {dx, dy, dz, index into weights}
    int ntaps;
    int *status;
    int warp_rows;         // 2-D 3 x 3 box: most staged widths are multiples of 32, step by warp rows
};
cudaError_t prepare_band(size_t max_smem);

// Autotuner utilities: a seeded uniform [0, 1) fill, and out[0] = max |y - r|,
// out[1] = max |r| as ordered bit patterns (out zeroed by the caller).
cudaError_t launch_fill_uniform(double *d, size_t n, uint64_t seed, cudaStream_t s);
cudaError_t launch_max_diff(const double *y, const double *r, size_t n, unsigned long long *out, cudaStream_t s);
cudaError_t launch_band(const BandWork &w, size_t smem_bytes, cudaStream_t s);
size_t band_smem_bytes(int64_t max_vol, int ntaps);

// One (problem, pass) of a batch: its tile work and band boxes, plus the stage
// of the same problem's previous pass that must finish first.
struct BatchStage {
    TileWork tw;
    BandWork bw;
    int dim;
    int dep;           // index of the previous pass's stage, -1 for the first pass
    int64_t dep_count; // items of that stage
};
size_t batch_tile_smem_bytes();
cudaError_t prepare_batch(size_t max_smem);
// Polls (128 ns apart) a batch item waits for its problem's previous pass before it
// records kDevTimeoutDep and goes on: seconds, far above any real wait.
constexpr uint32_t kDepSpinLimit = 1u << 24;
cudaError_t launch_batch(const BatchStage *stages, const int64_t *start, int nstages, int64_t total, int *done,
                         unsigned long long *head, int *status, uint32_t dep_limit, size_t smem, int grid,
                         cudaStream_t s);

} // namespace ffst
