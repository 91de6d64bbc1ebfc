// Pipe-peak microbenchmarks used as roofline denominators (libffs_peaks.so;
// benchmark infrastructure, not part of the solver ABI).
//   ffs_peak_dmma: FP64 mma.sync.m8n8k4 issue rate, 8 independent accumulator
//                  chains per warp, 4 warps per SM sub-partition.
//   ffs_peak_dfma: FP64 fma.rn issue rate (no tensor core), 8 independent chains
//                  per thread, 32 warps per SM.
//   ffs_peak_smem: shared-memory load bandwidth, conflict-free 16-byte loads (each
//                  warp reads 512 contiguous bytes), 8 in flight per thread.
//   ffs_peak_tc:   tcgen05.mma issue rate (kind::i8 M128 N256 K32 or kind::f16
//                  bf16 M128 N256 K16), one issuing thread per SM, accumulating in TMEM.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ffs_tcgen05.cuh"

namespace {

constexpr int kPeakSmem = 120 * 1024; // one CTA per SM (it holds all 512 TMEM columns)

template <bool I8>
__global__ void __launch_bounds__(128, 1) tc_loop(int iters, int *status)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 64 * 1024);
    uint32_t *slot = reinterpret_cast<uint32_t *>(sm + 64 * 1024 + 8);
    const int tid = threadIdx.x;
    for (int i = tid; i < 16 * 1024; i += 128) // operands: small finite values
        reinterpret_cast<uint32_t *>(sm)[i] = I8 ? 0x01010101u : 0x3c003c00u;
    if (tid == 0) {
        ffst::mbar_init(bar, 1);
        ffst::fence_barrier_init();
    }
    if (tid < 32)
        ffst::tc::tmem_alloc(slot, 512);
    ffst::fence_proxy_async_shared();
    ffst::tc::fence_before_sync();
    __syncthreads();
    ffst::tc::fence_after_sync();
    const uint32_t tmem = *slot;
    if (tid == 0) {
        const uint32_t a = ffst::smem_u32(sm), b = a + 16 * 1024;
        const uint64_t ad = ffst::tc::smem_desc(a, 128, 8 * 32), bd = ffst::tc::smem_desc(b, 128, 8 * 32);
        for (int it = 0; it < iters; ++it) {
            const uint32_t d = tmem + 256 * (it & 1);
            if (I8)
                ffst::tc::mma_i8(d, ad, bd, ffst::tc::idesc_i8(128, 256), it > 1);
            else
                ffst::tc::mma_f16(d, ad, bd, ffst::tc::idesc_bf16(128, 256), it > 1);
        }
        ffst::tc::commit(bar);
    }
    const bool ok = ffst::mbar_wait_bounded(bar, 0);
    if (!ok && tid == 0)
        atomicExch(status, 1);
    ffst::tc::fence_after_sync();
    ffst::tc::fence_before_sync();
    __syncthreads();
    if (tid < 32)
        ffst::tc::tmem_dealloc(tmem, 512);
}


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

__global__ void __launch_bounds__(512) dfma_loop(double *sink, int iters)
{
    const double b = 1.0 - threadIdx.x * 1e-9, c = 1e-12;
    double d[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        d[i] = 1.0 + i * 1e-3;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile("fma.rn.f64 %0, %0, %1, %2;\n" : "+d"(d[i]) : "d"(b), "d"(c));
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        s += d[i];
    if (s == 12345.678)
        sink[threadIdx.x] = s;
}

constexpr int kSmemSlots = 4096; // 64 KiB of 16-byte slots per CTA

__global__ void __launch_bounds__(512) lds_loop(unsigned long long *sink, int iters)
{
    extern __shared__ __align__(16) uint4 buf[];
    const int tid = threadIdx.x;
    for (int i = tid; i < kSmemSlots; i += blockDim.x)
        buf[i] = make_uint4(i, i * 3u, i * 5u, i * 7u);
    __syncthreads();
    uint32_t acc = 0;
    int base = tid;
    for (int it = 0; it < iters; ++it) {
        uint4 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            v[k] = buf[(base + k * 512) & (kSmemSlots - 1)];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            acc ^= v[k].x ^ v[k].y ^ v[k].z ^ v[k].w;
        base = (base + 32) & (kSmemSlots - 1);
    }
    if (acc == 0x12345678u)
        sink[tid] = acc;
}

} // namespace

// Returns achieved shared-memory load bandwidth over all SMs in GB/s (best of `reps`), 0 on error.
extern "C" double ffs_peak_smem(int iters, int reps)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return 0.0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 2, threads = 512;
    const size_t smem = kSmemSlots * sizeof(uint4);
    if (cudaFuncSetAttribute(lds_loop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0.0;
    unsigned long long *sink = nullptr;
    if (cudaMalloc(&sink, 512 * sizeof(unsigned long long)) != cudaSuccess)
        return 0.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    lds_loop<<<blocks, threads, smem>>>(sink, iters / 10 + 1); // warm-up
    float best = 1e30f;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0);
        lds_loop<<<blocks, threads, smem>>>(sink, iters);
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
    const double bytes = 8.0 * 16.0 * iters * (double)blocks * threads;
    return bytes / (best * 1e-3) / 1e9;
}

// Returns achieved FP64 TFLOP/s of back-to-back fma.rn.f64 (best of `reps`), 0 on error.
extern "C" double ffs_peak_dfma(int iters, int reps)
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
    const int blocks = sms * 4, threads = 512;
    dfma_loop<<<blocks, threads>>>(sink, iters / 10 + 1); // warm-up
    float best = 1e30f;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0);
        dfma_loop<<<blocks, threads>>>(sink, iters);
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
    const double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
    return flops / (best * 1e-3) / 1e12;
}

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

// Returns achieved dense TOPS (i8) or TFLOP/s (bf16) of back-to-back tcgen05.mma, 0 on error.
extern "C" double ffs_peak_tc(int int8, int iters, int reps)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return 0.0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    auto kern = int8 ? tc_loop<true> : tc_loop<false>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kPeakSmem) != cudaSuccess)
        return 0.0;
    int *status = nullptr;
    if (cudaMalloc(&status, sizeof(int)) != cudaSuccess)
        return 0.0;
    cudaMemset(status, 0, sizeof(int));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    kern<<<sms, 128, kPeakSmem>>>(iters / 10 + 2, status);
    float best = 1e30f;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0);
        kern<<<sms, 128, kPeakSmem>>>(iters, status);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = ms < best ? ms : best;
    }
    int st = 0;
    cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost);
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(status);
    if (err != cudaSuccess || st != 0)
        return 0.0;
    const double macs = 128.0 * 256.0 * (int8 ? 32.0 : 16.0);
    return 2.0 * macs * iters * sms / (best * 1e-3) / 1e12;
}
