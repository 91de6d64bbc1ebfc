// ffs_execute_noalloc: the 2-D FP64 solve for callers that must not allocate
// device memory.
//
// Who needs it: code that runs where cudaMalloc is off limits -- inside a
// framework that owns every device allocation through its own pool, in a
// real-time loop that may not block on the allocator, or in a host library
// whose policy forbids device allocations after start-up.  ffs_plan_create
// allocates the plan's spectra, tables and ping-pong workspace; this entry
// point instead keeps all of them in file-scope static __device__ arrays that
// the CUDA module reserves when the library is loaded on a GPU (the arrays stay
// resident on every GPU that loads libffs.so until the process exits).
//
// Limits: 2-D grids, FP64 form, at most kMaxCells cells (the ping-pong scratch
// is one grid), at most kMaxBoxes fixed-boundary band boxes per pass kind, and
// radius <= 4.  Every call shares the static arrays and they keep the previous
// call's contents: the device status word is cleared on each call, the
// spectra/tables/boxes are rewritten on each call, and two calls whose work
// overlaps on the GPU (different streams, or graph replays) race on them.
//
// The per-call constants (spectra, tables, taps, band boxes) reach the static
// arrays as the by-value parameters of small store kernels, at most
// kParamChunk bytes per launch: the launch copies its parameters, so no host
// buffer has to outlive the call and no pageable-memory copy (which would
// synchronise the stream with the host) is issued.
//
// The first call on a device resolves the arrays' device addresses with
// cudaGetSymbolAddress and sets the kernels' shared-memory limits, with that
// device current; make that first call before any stream capture.
// ffs_noalloc_status reads the shared status word back (synchronously).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ffs.h"
#include "ffs_kernels.h"
#include "ffs_plan.h"

using namespace ffst;

namespace {

constexpr int64_t kMaxCells = 1 << 20; // 8 MiB of FP64 scratch: e.g. a 1024 x 1024 grid
constexpr int kMaxBoxes = 1024;
constexpr int kSpecLen = 64 * 64; // the 2-D tile kernel's spectrum (DFT-64 x DFT-64)
constexpr int kTables = 8 + 64;
constexpr int kMaxTaps = 81; // 9 x 9

static __device__ __align__(256) double g_scratch[kMaxCells];
static __device__ __align__(256) double2 g_spec[2][kSpecLen];
static __device__ __align__(256) double2 g_tables[kTables];
static __device__ __align__(256) double g_weights[kMaxTaps];
static __device__ __align__(256) int4 g_taps[kMaxTaps];
static __device__ __align__(256) BandBox g_boxes[2][kMaxBoxes];
static __device__ __align__(256) int g_status;

// Kernel parameters hold at most 32,764 bytes; one store launch carries this many.
constexpr int kParamChunk = 31 * 1024;

struct StoreChunk {
    uint32_t *dst;   // 4-byte aligned destination inside one of the static arrays
    int nwords;      // 32-bit words to store
    uint32_t data[kParamChunk / 4];
};

__global__ void store_chunk_kernel(const __grid_constant__ StoreChunk c)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c.nwords; i += gridDim.x * blockDim.x)
        c.dst[i] = c.data[i];
}

struct StaticPtrs {
    int device = -1;
    int sms = 0;
    double *scratch = nullptr;
    double2 *spec = nullptr;
    double2 *tables = nullptr;
    double *weights = nullptr;
    int4 *taps = nullptr;
    BandBox *boxes = nullptr;
    int *status = nullptr;
};

std::mutex g_mu;
std::vector<StaticPtrs> g_devs;

template <typename T, typename S>
cudaError_t symbol_addr(T **dst, const S &sym)
{
    return cudaGetSymbolAddress(reinterpret_cast<void **>(dst), sym);
}

// Once per device, with that device current: device addresses of the static
// arrays (a kernel given the host-side symbol would read the wrong memory).
ffs_status setup(int dev, StaticPtrs *out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (const StaticPtrs &p : g_devs)
        if (p.device == dev) {
            *out = p;
            return FFS_OK;
        }
    StaticPtrs p;
    p.device = dev;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess)
        e = symbol_addr(&p.scratch, g_scratch);
    if (e == cudaSuccess)
        e = symbol_addr(&p.spec, g_spec);
    if (e == cudaSuccess)
        e = symbol_addr(&p.tables, g_tables);
    if (e == cudaSuccess)
        e = symbol_addr(&p.weights, g_weights);
    if (e == cudaSuccess)
        e = symbol_addr(&p.taps, g_taps);
    if (e == cudaSuccess)
        e = symbol_addr(&p.boxes, g_boxes);
    if (e == cudaSuccess)
        e = symbol_addr(&p.status, g_status);
    if (e == cudaSuccess)
        e = prepare_dmma2d();
    if (e == cudaSuccess)
        e = prepare_band(kBandSmemLimit);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&p.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) {
        (void)cudaGetLastError(); // a handled failure is not reported again by a later launch check
        return set_error(FFS_ERR_CUDA, std::string("ffs_execute_noalloc set-up: ") + cudaGetErrorString(e));
    }
    g_devs.push_back(p);
    *out = p;
    return FFS_OK;
}

PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    }();
    return fn;
}

bool tensor_map(CUtensorMap *m, const double *base, int64_t nx, int64_t ny)
{
    auto enc = encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(base) & 15) || ((nx * 8) & 15))
        return false;
    const int box = dmma2d_tile();
    cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
    cuuint64_t strides[1] = {(cuuint64_t)(nx * 8)};
    cuuint32_t boxd[2] = {(cuuint32_t)box, (cuuint32_t)box};
    cuuint32_t es[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims, strides, boxd, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Store `src` at `dst` (device) through the parameters of store_chunk_kernel
// launches on `s`.  Every type stored here is a whole number of 32-bit words.
template <typename T>
cudaError_t put(T *dst, const std::vector<T> &src, cudaStream_t s)
{
    static_assert(sizeof(T) % 4 == 0, "stored types are whole 32-bit words");
    const size_t words = src.size() * sizeof(T) / 4;
    const uint32_t *from = reinterpret_cast<const uint32_t *>(src.data());
    uint32_t *to = reinterpret_cast<uint32_t *>(dst);
    StoreChunk c; // ~31 KiB on the host stack; copied into the launch's parameter buffer
    for (size_t w0 = 0; w0 < words; w0 += kParamChunk / 4) {
        const int n = (int)std::min<size_t>(kParamChunk / 4, words - w0);
        c.dst = to + w0;
        c.nwords = n;
        std::memcpy(c.data, from + w0, (size_t)n * 4);
        store_chunk_kernel<<<(n + 255) / 256 < 16 ? (n + 255) / 256 : 16, 256, 0, s>>>(c);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

} // namespace

extern "C" ffs_status ffs_execute_noalloc(const ffs_problem *problem, const double *d_in, double *d_out,
                                          void *stream)
{
    if (!problem || !d_in || !d_out)
        return set_error(FFS_ERR_INVALID_ARGUMENT, "ffs_execute_noalloc: null argument");
    PlanSpec sp;
    std::string why;
    ffs_problem pr = *problem;
    if (pr.form == FFS_FORM_AUTO) // the one form this entry point has
        pr.form = FFS_FORM_FP64_DMMA;
    ffs_status st = build_plan_spec(pr, &sp, &why);
    if (st != FFS_OK)
        return set_error(st, "ffs_execute_noalloc: " + why);
    if (sp.dim != 2 || sp.form != FFS_FORM_FP64_DMMA)
        return set_error(FFS_ERR_UNSUPPORTED, "ffs_execute_noalloc: only 2-D grids with the FP64-DMMA form");
    if ((int64_t)sp.cells > kMaxCells)
        return set_error(FFS_ERR_UNSUPPORTED, "ffs_execute_noalloc: grid of " + std::to_string(sp.cells) +
                                                  " cells exceeds the static scratch limit of " +
                                                  std::to_string(kMaxCells) + " cells");
    if ((int)sp.taps.size() > kMaxTaps || (int)sp.weights.size() > kMaxTaps)
        return set_error(FFS_ERR_UNSUPPORTED, "ffs_execute_noalloc: stencil radius above 4");
    for (int k = 0; k < sp.npass_kinds; ++k)
        if ((int)sp.pass[k].boxes.size() > kMaxBoxes)
            return set_error(FFS_ERR_UNSUPPORTED, "ffs_execute_noalloc: too many band boxes");
    int dev = 0;
    (void)cudaGetLastError(); // launches below are checked with cudaGetLastError: no stale error
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return set_error(FFS_ERR_CUDA, std::string("ffs_execute_noalloc: ") + cudaGetErrorString(e));
    }
    StaticPtrs P;
    st = setup(dev, &P);
    if (st != FFS_OK)
        return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t bytes = sp.cells * sizeof(double);
    auto cuda_fail = [](cudaError_t err) {
        (void)cudaGetLastError(); // a handled failure is not reported again by a later launch check
        return set_error(FFS_ERR_CUDA, std::string("ffs_execute_noalloc: ") + cudaGetErrorString(err));
    };
    const int P_ = sp.passes;
    if (P_ == 0) {
        if (d_in != d_out && (e = cudaMemcpyAsync(d_out, d_in, bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
            return cuda_fail(e);
        return FFS_OK;
    }
    // this call's constants into the shared static arrays; clear the status word
    if ((e = cudaMemsetAsync(P.status, 0, sizeof(int), s)) != cudaSuccess)
        return cuda_fail(e);
    if ((e = put(P.tables, sp.tables, s)) != cudaSuccess || (e = put(P.weights, sp.weights, s)) != cudaSuccess ||
        (e = put(P.taps, sp.taps, s)) != cudaSuccess)
        return cuda_fail(e);
    for (int k = 0; k < sp.npass_kinds; ++k)
        if ((e = put(P.spec + (size_t)k * kSpecLen, sp.pass[k].spectrum, s)) != cudaSuccess ||
            (e = put(P.boxes + (size_t)k * kMaxBoxes, sp.pass[k].boxes, s)) != cudaSuccess)
            return cuda_fail(e);

    const double *src = d_in;
    if (d_in == d_out && (P_ % 2 == 1)) {
        if ((e = cudaMemcpyAsync(P.scratch, d_in, bytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
            return cuda_fail(e);
        src = P.scratch;
    }
    for (int i = 0; i < P_; ++i) {
        double *dst = ((P_ - 1 - i) % 2 == 0) ? d_out : P.scratch;
        const int kind = (i == P_ - 1) ? sp.last_kind : 0;
        const PassSpec &ps = sp.pass[kind];
        if (ps.nitems > 0) {
            TileWork w{};
            w.in = src;
            w.out = dst;
            w.spec = P.spec + (size_t)kind * kSpecLen;
            w.tables = P.tables;
            w.status = P.status;
            w.nx = sp.n[0];
            w.ny = sp.n[1];
            w.nz = sp.n[2];
            w.halo = ps.halo;
            w.useful = ps.useful;
            for (int d = 0; d < 3; ++d) {
                w.t0[d] = ps.t0[d];
                w.nt[d] = ps.nt[d];
                w.vlo[d] = ps.vlo[d];
                w.vhi[d] = ps.vhi[d];
            }
            w.npx = ps.npx;
            w.nitems = ps.nitems;
            w.periodic = sp.boundary == FFS_BOUNDARY_PERIODIC;
            CUtensorMap tm;
            w.use_tma = tensor_map(&tm, src, sp.n[0], sp.n[1]);
            e = launch_dmma2d(w.use_tma ? &tm : nullptr, w, (int)std::min<int64_t>(ps.nitems, P.sms), s);
            if (e != cudaSuccess)
                return cuda_fail(e);
        }
        if (!ps.boxes.empty()) {
            BandWork b{};
            b.in = src;
            b.out = dst;
            b.weights = P.weights;
            b.boxes = P.boxes + (size_t)kind * kMaxBoxes;
            b.nboxes = (int)ps.boxes.size();
            b.dim = sp.dim;
            b.r = sp.radius;
            b.tau = ps.tau;
            for (int d = 0; d < 3; ++d)
                b.n[d] = sp.n[d];
            b.max_vol = ps.band_max_vol;
            b.taps = P.taps;
            b.ntaps = (int)sp.taps.size();
            b.status = P.status;
            e = launch_band(b, band_smem_bytes(ps.band_max_vol, b.ntaps), s);
            if (e != cudaSuccess)
                return cuda_fail(e);
        }
        src = dst;
    }
    return FFS_OK;
}

extern "C" ffs_status ffs_noalloc_status(int *device_status)
{
    if (!device_status)
        return set_error(FFS_ERR_INVALID_ARGUMENT, "ffs_noalloc_status: null argument");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    StaticPtrs P;
    if (e == cudaSuccess) {
        const ffs_status st = setup(dev, &P);
        if (st != FFS_OK)
            return st;
        e = cudaDeviceSynchronize(); // the word is written by kernels on whatever stream the calls used
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(device_status, P.status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return set_error(FFS_ERR_CUDA, std::string("ffs_noalloc_status: ") + cudaGetErrorString(e));
    }
    return FFS_OK;
}
