// Small device utilities of the autotuner: a seeded uniform fill of a scratch
// grid, and the max |y - r| / max |r| of two grids (the calibration of the Ozaki
// slice count against the FP64 form).
#include <cuda_runtime.h>
#include <stdint.h>

#include "ffs_kernels.h"

namespace ffst {
namespace util {

// splitmix64 of (seed, index) -> uniform [0, 1) with 53 random bits.
__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t i)
{
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void fill_uniform_kernel(double *d, size_t n, uint64_t seed)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        d[i] = uniform01(seed, i);
}

// out[0] = max |y - r|, out[1] = max |r|, as the bit patterns of non-negative
// doubles (which order like the doubles); out must start at zero.
__global__ void max_diff_kernel(const double *y, const double *r, size_t n, unsigned long long *out)
{
    double md = 0.0, mr = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        md = fmax(md, fabs(y[i] - r[i]));
        mr = fmax(mr, fabs(r[i]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        md = fmax(md, __shfl_xor_sync(0xffffffffu, md, o));
        mr = fmax(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(out, (unsigned long long)__double_as_longlong(md));
        atomicMax(out + 1, (unsigned long long)__double_as_longlong(mr));
    }
}

} // namespace util

cudaError_t launch_fill_uniform(double *d, size_t n, uint64_t seed, cudaStream_t s)
{
    util::fill_uniform_kernel<<<1184, 256, 0, s>>>(d, n, seed);
    return cudaGetLastError();
}

cudaError_t launch_max_diff(const double *y, const double *r, size_t n, unsigned long long *out, cudaStream_t s)
{
    util::max_diff_kernel<<<1184, 256, 0, s>>>(y, r, n, out);
    return cudaGetLastError();
}

} // namespace ffst
