// Batched multi-problem execution: ONE persistent kernel for many independent
// FP64 stencil problems of mixed dimension, size, shape, boundary and T.
//
// The host lays out a "stage" per (problem, pass) -- the pass's tile work and,
// for a fixed boundary, its band boxes -- and orders all stages level by level
// (pass 0 of every problem, then pass 1, ...).  The work queue is the
// concatenation of every stage's items (tile pairs, then band boxes); one CTA
// per SM pops items with an atomic counter.  An item of pass p waits (bounded)
// until every item of pass p-1 of the same problem has finished: that stage was
// queued earlier, so its items are held by running CTAs that never wait on a
// later item, which guarantees progress.  Completion is published with a
// device-scope fence and an atomic per-stage counter; tile inputs are read with
// L1-bypassing loads so a CTA never sees a stale line of a buffer rewritten by
// another SM.  The persistent CUDA-graph launch replaces one launch per problem
// per pass (the reference launches one kernel per time step per problem,
// src/2D/2d_main.cu:150-170).
#include <cuda_runtime.h>

#include "ffs_band.cuh"
#include "ffs_dmma1d.cuh"
#include "ffs_dmma2d.cuh"
#include "ffs_dmma3d.cuh"

namespace ffst {
namespace batch {

constexpr int NT = 512;
constexpr size_t SPEC_OFF = 64 * 1024;
constexpr size_t TW_OFF = 128 * 1024;
constexpr size_t TILE_SMEM = TW_OFF + (dmma1d::T1N + dmma1d::T2N) * sizeof(double2);

__device__ __forceinline__ int find_stage(const int64_t *start, int nstages, int64_t item)
{
    int lo = 0, hi = nstages - 1; // largest s with start[s] <= item
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (start[mid] <= item)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(NT, 1) batch_kernel(const BatchStage *stages, const int64_t *start, int nstages,
                                                      int64_t total, int *done, unsigned long long *head, int *status,
                                                      uint32_t dep_limit)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ int64_t s_item;
    __shared__ int s_stage;
    double2 *work = reinterpret_cast<double2 *>(smem);
    double2 *spec = reinterpret_cast<double2 *>(smem + SPEC_OFF);
    double2 *tw = reinterpret_cast<double2 *>(smem + TW_OFF);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    const void *cached = nullptr; // spectrum currently in shared memory (block-uniform)

    for (;;) {
        if (tid == 0) {
            const int64_t item = (int64_t)atomicAdd(head, 1ull);
            s_item = item;
            if (item < total) {
                const int s = find_stage(start, nstages, item);
                s_stage = s;
                const int dep = stages[s].dep;
                if (dep >= 0) {
                    const int need = (int)stages[s].dep_count;
                    uint32_t spins = 0;
                    while (atomicAdd(done + dep, 0) < need) {
                        if (++spins > dep_limit) {
                            record_error(status, kDevTimeoutDep);
                            break;
                        }
                        __nanosleep(128);
                    }
                }
                __threadfence();
            }
        }
        __syncthreads();
        const int64_t item = s_item;
        if (item >= total)
            break;
        const BatchStage &S = stages[s_stage];
        const int64_t local = item - start[s_stage];
        if (local < S.tw.nitems) {
            const TileWork &p = S.tw;
            if (S.dim == 2) {
                if (cached != p.spec) {
                    for (int i = tid; i < 64 * 64; i += NT)
                        spec[i] = p.spec[i];
                    cached = p.spec;
                }
                const dmma2d::Item it = dmma2d::item_of(p, local);
                dmma2d::fill_plain(work, p, it, tid);
                __syncthreads();
                const r64::LaneConst c = r64::lane_consts(p.tables, p.tables + 8, g, t);
                dmma2d::compute_item(work, spec, c, p, it, warp, NT / 32, g, t);
            } else if (S.dim == 1) {
                if (cached != p.spec) {
                    for (int i = tid; i < 64 * 64; i += NT)
                        spec[i] = p.spec[i];
                    for (int i = tid; i < dmma1d::T1N + dmma1d::T2N; i += NT)
                        tw[i] = p.tables[8 + 64 + i];
                    cached = p.spec;
                }
                const dmma1d::Item it = dmma1d::item_of(p, local);
                dmma1d::fill_plain(work, p, it, tid);
                __syncthreads();
                const r64::LaneConst c = r64::lane_consts(p.tables, p.tables + 8, g, t);
                dmma1d::compute_item(work, spec, tw, tw + dmma1d::T1N, c, p, it, tid, NT, warp, NT / 32, g, t);
            } else {
                if (cached != p.spec) {
                    for (int i = tid; i < 16 * 16 * 16; i += NT)
                        spec[dmma3d::sw3(i)] = p.spec[i];
                    cached = p.spec;
                }
                const dmma3d::Item it = dmma3d::item_of(p, local);
                dmma3d::fill_plain(work, p, it, tid);
                __syncthreads();
                const dmma3d::Consts c = dmma3d::make_consts(p.tables, g, t);
                dmma3d::compute_item<dmma3d::kFromWork>(work, nullptr, spec, c, p, it, warp, g, t);
            }
        } else {
            const int box = (int)(local - S.tw.nitems);
            if (S.dim == 1)
                band::process_box<1>(S.bw, box, smem, NT);
            else if (S.dim == 2)
                band::process_box<2>(S.bw, box, smem, NT);
            else
                band::process_box<3>(S.bw, box, smem, NT);
            cached = nullptr; // shared memory was reused
        }
        __threadfence();
        __syncthreads();
        if (tid == 0)
            atomicAdd(done + s_stage, 1);
    }
}

} // namespace batch

size_t batch_tile_smem_bytes() { return batch::TILE_SMEM; }

cudaError_t prepare_batch(size_t max_smem)
{
    return cudaFuncSetAttribute(batch::batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_smem);
}

cudaError_t launch_batch(const BatchStage *stages, const int64_t *start, int nstages, int64_t total, int *done,
                         unsigned long long *head, int *status, uint32_t dep_limit, size_t smem, int grid,
                         cudaStream_t s)
{
    if (total <= 0)
        return cudaSuccess;
    batch::batch_kernel<<<grid, batch::NT, smem, s>>>(stages, start, nstages, total, done, head, status,
                                                      dep_limit);
    return cudaGetLastError();
}

} // namespace ffst
