// Pipe-peak microbenchmarks used as roofline denominators (libffs_peaks.so;
// benchmark infrastructure, not part of the solver ABI).
//   ffs_peak_dmma: FP64 mma.sync.m8n8k4 issue rate, 8 independent accumulator
//                  chains per warp, 4 warps per SM sub-partition.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

__global__ void __launch_bounds__(512) dmma_loop(double *sink, int iters)
{
    const int lane = threadIdx.x & 31;
    double a = 1.0 + lane * 1e-3, b = 1.0 - lane * 1e-3;
    double d[8][2];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        d[i][0] = d[i][1] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(d[i][0]), "+d"(d[i][1])
                         : "d"(a), "d"(b));
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        s += d[i][0] + d[i][1];
    if (s == 12345.678)
        sink[threadIdx.x] = s;
}

} // namespace

// Returns achieved FP64 TFLOP/s of back-to-back DMMA (best of `reps`), 0 on error.
extern "C" double ffs_peak_dmma(int iters, int reps)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return 0.0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    double *sink = nullptr;
    if (cudaMalloc(&sink, 512 * sizeof(double)) != cudaSuccess)
        return 0.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = sms * 2, threads = 512;
    dmma_loop<<<blocks, threads>>>(sink, iters / 10 + 1); // warm-up
    float best = 1e30f;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0);
        dmma_loop<<<blocks, threads>>>(sink, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best)
            best = ms;
    }
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess)
        return 0.0;
    const double flops = 2.0 * 8 * 8 * 4 * 8.0 * iters * (double)blocks * (threads / 32);
    return flops / (best * 1e-3) / 1e12;
}
