// C ABI of libffs.so: plan building (shape table, FP64 spectra, tile geometry,
// autotuning, fixed-boundary band boxes) and execution (pass loop over the
// sm_100a kernels).  See include/ffs.h for the contract and the reference
// interfaces each entry point replaces.
#include "ffs.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "ffs_kernels.h"
#include "ffs_plan.h"

using namespace ffst;

namespace {

thread_local std::string g_err;

ffs_status fail(ffs_status st, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return st;
}

// On failure the runtime's per-thread last error is cleared too, so a handled
// failure (an allocation that did not fit) is not reported again by the error
// check after a later kernel launch.
#define CUDA_TRY(expr)                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            (void)cudaGetLastError();                                                                     \
            if (e_ == cudaErrorMemoryAllocation)                                                          \
                return fail(FFS_ERR_OUT_OF_MEMORY, "%s: %s", #expr, cudaGetErrorString(e_));             \
            return fail(FFS_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));                           \
        }                                                                                                 \
    } while (0)

// ---- tensor maps (driver entry point fetched through the runtime, so the
// library loads on machines without a GPU driver) ----
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    std::call_once(g_encode_once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    return g_encode;
}

// 2D FP64 tensor map over a natural row-major grid with a box x box tile.
bool make_tmap_2d(CUtensorMap *m, const double *base, int64_t nx, int64_t ny, int box)
{
    auto enc = encode_fn();
    if (!enc || (reinterpret_cast<uintptr_t>(base) & 15) || ((nx * 8) & 15) || nx >= (1ll << 31) ||
        ny >= (1ll << 31))
        return false;
    cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
    cuuint64_t strides[1] = {(cuuint64_t)(nx * 8)};
    cuuint32_t boxd[2] = {(cuuint32_t)box, (cuuint32_t)box};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims, strides, boxd, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 2D FP64 tensor map with 16 x 64 boxes (one 128-byte line per row) and the 128-byte
// swizzle: a 64 x 64 tile is four boxes, which the butterfly kernel reads with that swizzle.
bool make_tmap_2d_boxes(CUtensorMap *m, const double *base, int64_t nx, int64_t ny)
{
    auto enc = encode_fn();
    if (!enc || (reinterpret_cast<uintptr_t>(base) & 15) || ((nx * 8) & 15) || nx >= (1ll << 31) ||
        ny >= (1ll << 31))
        return false;
    cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
    cuuint64_t strides[1] = {(cuuint64_t)(nx * 8)};
    cuuint32_t boxd[2] = {16, 64};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims, strides, boxd, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 3D FP64 tensor map (x fastest) with a box^3 tile of 16-double (128-byte) rows,
// 128-byte swizzle: the kernel reads the staged tile with that swizzle.
bool make_tmap_3d(CUtensorMap *m, const double *base, int64_t nx, int64_t ny, int64_t nz, int box)
{
    auto enc = encode_fn();
    if (!enc || (reinterpret_cast<uintptr_t>(base) & 15) || ((nx * 8) & 15) || nx >= (1ll << 31) ||
        ny >= (1ll << 31) || nz >= (1ll << 31))
        return false;
    cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz};
    cuuint64_t strides[2] = {(cuuint64_t)(nx * 8), (cuuint64_t)(nx * ny * 8)};
    cuuint32_t boxd[3] = {(cuuint32_t)box, (cuuint32_t)box, (cuuint32_t)box};
    cuuint32_t es[3] = {1, 1, 1};
    if (box * 8 != 128)
        return false;
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(base), dims, strides, boxd, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

std::mutex g_prep_mu;
std::vector<int> g_prepared; // devices whose kernel attributes are set

ffs_status prepare_device(int dev)
{
    std::lock_guard<std::mutex> lk(g_prep_mu);
    if (std::find(g_prepared.begin(), g_prepared.end(), dev) != g_prepared.end())
        return FFS_OK;
    CUDA_TRY(prepare_dmma2d());
    CUDA_TRY(prepare_fft2d());
    CUDA_TRY(prepare_fft3d());
    CUDA_TRY(prepare_fft3d32());
    CUDA_TRY(prepare_fft2d128());
    CUDA_TRY(prepare_fft1d());
    CUDA_TRY(prepare_dmma1d());
    CUDA_TRY(prepare_dmma3d());
    CUDA_TRY(prepare_tc2d());
    CUDA_TRY(prepare_tc3d());
    CUDA_TRY(prepare_batch(std::max(kBandSmemLimit, batch_tile_smem_bytes())));
    CUDA_TRY(prepare_band(kBandSmemLimit));
    g_prepared.push_back(dev);
    return FFS_OK;
}

} // namespace

ffs_status ffst::set_error(ffs_status st, const std::string &msg)
{
    g_err = msg;
    return st;
}

// ------------------------------------------------------------------------------------------
struct ffs_plan {
    PlanSpec spec;            // host description (geometry, spectra, boxes)
    int device = 0;
    int num_sms = 148;
    double2 *d_tables = nullptr;
    unsigned char *d_aslices = nullptr;
    double *d_weights = nullptr;
    int4 *d_taps = nullptr;
    int *d_status = nullptr;
    double *d_work = nullptr;
    struct Dev {
        double2 *spec = nullptr;
        BandBox *boxes = nullptr;
    } dev[2];
    // tracing (ffs_plan_profile): events bracketing each launch, kind 0 = tile, 1 = band
    struct Mark {
        cudaEvent_t a, b;
        int kind;
    };
    mutable bool profiling = false;
    mutable std::vector<Mark> marks;
    // the band kernel runs beside the tile kernel on a side stream (fork/join events)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // executions of one plan share its workspace and side stream: each waits for the
    // previous one (on whatever stream that ran) through this event
    cudaEvent_t ev_last = nullptr;
    mutable bool ran = false;
    mutable std::mutex run_mu;
    // an ffs_execute call that repeats the previous call (same plan and buffers) replays a
    // CUDA graph of the pass sequence, captured on a private stream at the first repeat:
    // fewer launch and fork/join gaps between the passes.  Up to kGraphs buffer pairs per
    // plan, least recently used out.
    static constexpr int kGraphs = 4;
    struct GraphEntry {
        const double *in = nullptr;
        double *out = nullptr;
        cudaGraphExec_t exec = nullptr; // null: the pair was seen once, no graph yet
        uint64_t used = 0;
    };
    mutable GraphEntry graphs[kGraphs];
    mutable uint64_t graph_clock = 0;
    mutable cudaStream_t graph_stream = nullptr;
    // host-buffer path, set up on its first call: two device (input, output)
    // slots, a copy-in and a copy-out stream, and per-slot events, so the
    // copy-out of one grid, the compute of the next and the copy-in of the one
    // after that overlap (PCIe is full duplex)
    struct HostPipe {
        double *in[2] = {nullptr, nullptr}, *out[2] = {nullptr, nullptr};
        cudaStream_t s_in = nullptr, s_out = nullptr;
        cudaEvent_t start = nullptr, in_ready[2] = {}, comp_done[2] = {}, out_done[2] = {};
        // Slabs along the slowest axis, so one grid's copy-in, compute and
        // copy-out overlap each other.  Slab j's interior is rows [a[j], a[j+1]);
        // its sub-plan steps rows [lo[j], hi[j]) -- the interior plus g = r*T
        // ghost rows on each cut face (rows outside [0, n) wrap for periodic
        // grids) -- and only the interior is copied out.
        struct Slabs {
            bool decided = false;
            SlabModel model;
            int count = 1; // slabs built (1 = whole-grid pipeline only)
            int axis = 0;
            int64_t row = 0, ghost = 0;
            std::vector<int64_t> a, lo, hi;
            std::vector<int> sub, last_chunk, order;
            std::vector<ffs_plan *> plans; // distinct sub-plans (by rows and cut faces)
            int64_t max_rows = 0;
            double *ring[3] = {nullptr, nullptr, nullptr}; // sub-plan outputs
            cudaEvent_t comp_done[3] = {}, out_done[3] = {};
            bool ring_used[3] = {false, false, false};
            double *wrap = nullptr; // assembled input of a slab that wraps
            std::vector<cudaEvent_t> chunk[2];
            cudaEvent_t grid_done[2] = {};
        } slabs;
    };
    mutable HostPipe host;
    mutable std::mutex host_mu;
};

static void clear_marks(const ffs_plan *p)
{
    for (auto &m : p->marks) {
        cudaEventDestroy(m.a);
        cudaEventDestroy(m.b);
    }
    p->marks.clear();
}

// Brackets one launch with events when profiling is on.
struct LaunchMark {
    const ffs_plan *p;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    int kind;
    LaunchMark(const ffs_plan *p_, cudaStream_t s_, int kind_) : p(p_), s(s_), kind(kind_)
    {
        if (!p->profiling)
            return;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, s);
    }
    ~LaunchMark()
    {
        if (!a)
            return;
        cudaEventRecord(b, s);
        p->marks.push_back({a, b, kind});
    }
};

struct ffs_batch {
    std::vector<const ffs_plan *> plans;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<const double *> ins;
    std::vector<double *> outs;
    cudaStream_t stream = nullptr;
    int device = 0;
    int num_sms = 148;
    // persistent-kernel queue for the FP64 plans (rebuilt when buffers change)
    BatchStage *d_stages = nullptr;
    int64_t *d_start = nullptr;
    int *d_done = nullptr;
    unsigned long long *d_head = nullptr;
    int *d_status = nullptr;
    int nstages = 0;
    int64_t total = 0;
    size_t smem = 0;
    uint32_t dep_limit = kDepSpinLimit; // FFS_BATCH_WAIT_POLLS overrides it at creation
    // plans outside the persistent kernel (the butterfly and tensor-core forms) run as
    // their own launches on parallel branches of the graph (created on first capture)
    static constexpr int kBranches = 8;
    cudaStream_t branch[kBranches] = {};
    cudaEvent_t bfork = nullptr, bjoin[kBranches] = {};
};

static cudaError_t ensure_branches(ffs_batch *b)
{
    if (b->bfork)
        return cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int k = 0; k < ffs_batch::kBranches && e == cudaSuccess; ++k) {
        e = cudaStreamCreateWithFlags(&b->branch[k], cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&b->bjoin[k], cudaEventDisableTiming);
    }
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&b->bfork, cudaEventDisableTiming);
    return e;
}

static void release_batch_queue(ffs_batch *b)
{
    cudaFree(b->d_stages);
    cudaFree(b->d_start);
    cudaFree(b->d_done);
    b->d_stages = nullptr;
    b->d_start = nullptr;
    b->d_done = nullptr;
    b->nstages = 0;
    b->total = 0;
}

static void release(ffs_plan *p);

// Frees the slab pipeline's sub-plans, buffers and events and resets it to the
// whole-grid pipeline (count 1; the decision stays made).
static void release_slabs(ffs_plan::HostPipe::Slabs &sl)
{
    for (int r = 0; r < 3; ++r) {
        cudaFree(sl.ring[r]);
        for (cudaEvent_t e : {sl.comp_done[r], sl.out_done[r]})
            if (e)
                cudaEventDestroy(e);
        sl.ring[r] = nullptr;
        sl.comp_done[r] = sl.out_done[r] = nullptr;
    }
    cudaFree(sl.wrap);
    sl.wrap = nullptr;
    for (int k = 0; k < 2; ++k) {
        for (cudaEvent_t e : sl.chunk[k])
            if (e)
                cudaEventDestroy(e);
        sl.chunk[k].clear();
        if (sl.grid_done[k])
            cudaEventDestroy(sl.grid_done[k]);
        sl.grid_done[k] = nullptr;
    }
    for (ffs_plan *sp : sl.plans)
        release(sp);
    sl.plans.clear();
    sl.count = 1;
}

static void release(ffs_plan *p)
{
    if (!p)
        return;
    clear_marks(p);
    for (ffs_plan::GraphEntry &g : p->graphs)
        if (g.exec)
            cudaGraphExecDestroy(g.exec);
    if (p->graph_stream)
        cudaStreamDestroy(p->graph_stream);
    if (p->side)
        cudaStreamDestroy(p->side);
    if (p->ev_fork)
        cudaEventDestroy(p->ev_fork);
    if (p->ev_join)
        cudaEventDestroy(p->ev_join);
    if (p->ev_last)
        cudaEventDestroy(p->ev_last);
    {
        auto &h = p->host;
        for (int k = 0; k < 2; ++k) {
            cudaFree(h.in[k]);
            cudaFree(h.out[k]);
            for (cudaEvent_t e : {h.in_ready[k], h.comp_done[k], h.out_done[k]})
                if (e)
                    cudaEventDestroy(e);
        }
        if (h.start)
            cudaEventDestroy(h.start);
        if (h.s_in)
            cudaStreamDestroy(h.s_in);
        if (h.s_out)
            cudaStreamDestroy(h.s_out);
        release_slabs(h.slabs);
    }
    cudaFree(p->d_tables);
    cudaFree(p->d_aslices);
    cudaFree(p->d_weights);
    cudaFree(p->d_taps);
    cudaFree(p->d_status);
    cudaFree(p->d_work);
    for (auto &d : p->dev) {
        cudaFree(d.spec);
        cudaFree(d.boxes);
    }
    delete p;
}

template <typename T>
static cudaError_t upload(T **dst, const std::vector<T> &src)
{
    *dst = nullptr;
    if (src.empty())
        return cudaSuccess;
    cudaError_t e = cudaMalloc(dst, src.size() * sizeof(T));
    if (e != cudaSuccess)
        return e;
    return cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
}

extern "C" ffs_status ffs_plan_create(ffs_plan **out, const ffs_problem *problem)
{
    if (!out || !problem)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_plan_create: null argument");
    *out = nullptr;
    PlanSpec spec;
    std::string why;
    ffs_status st = build_plan_spec(*problem, &spec, &why);
    if (st != FFS_OK)
        return fail(st, "%s", why.c_str());

    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    st = prepare_device(dev);
    if (st != FFS_OK)
        return st;
    ffs_plan *p = new ffs_plan();
    p->spec = std::move(spec);
    p->device = dev;
    cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, dev);
    auto bail = [&](cudaError_t e, const char *what) {
        (void)cudaGetLastError(); // handled here: not to be seen by a later launch check
        release(p);
        return fail(e == cudaErrorMemoryAllocation ? FFS_ERR_OUT_OF_MEMORY : FFS_ERR_CUDA, "%s: %s", what,
                    cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = upload(&p->d_tables, p->spec.tables)) != cudaSuccess)
        return bail(e, "tables");
    if ((e = upload(&p->d_aslices, p->spec.a_slices)) != cudaSuccess)
        return bail(e, "tensor-core operand slices");
    if ((e = upload(&p->d_weights, p->spec.weights)) != cudaSuccess)
        return bail(e, "weights");
    if ((e = upload(&p->d_taps, p->spec.taps)) != cudaSuccess)
        return bail(e, "taps");
    for (int i = 0; i < p->spec.npass_kinds; ++i) {
        if ((e = upload(&p->dev[i].spec, p->spec.pass[i].spectrum)) != cudaSuccess)
            return bail(e, "spectrum");
        if ((e = upload(&p->dev[i].boxes, p->spec.pass[i].boxes)) != cudaSuccess)
            return bail(e, "band boxes");
    }
    if ((e = cudaMalloc(&p->d_status, sizeof(int))) != cudaSuccess)
        return bail(e, "status word");
    if ((e = cudaMemset(p->d_status, 0, sizeof(int))) != cudaSuccess)
        return bail(e, "status word");
    if (p->spec.passes >= 1) {
        if ((e = cudaMalloc(&p->d_work, p->spec.cells * sizeof(double))) != cudaSuccess)
            return bail(e, "workspace");
    }
    if ((e = cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&p->ev_last, cudaEventDisableTiming)) != cudaSuccess)
        return bail(e, "side stream");
    *out = p;
    return FFS_OK;
}

extern "C" ffs_status ffs_plan_destroy(ffs_plan *plan)
{
    release(plan);
    return FFS_OK;
}

static TileWork tile_work(const ffs_plan *p, int kind, const double *src, double *dst)
{
    const PlanSpec &sp = p->spec;
    const PassSpec &ps = sp.pass[kind];
    TileWork w{};
    w.in = src;
    w.out = dst;
    w.spec = p->dev[kind].spec;
    w.tables = p->d_tables;
    w.status = p->d_status;
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
    return w;
}

static BandWork band_work(const ffs_plan *p, int kind, const double *src, double *dst)
{
    const PlanSpec &sp = p->spec;
    const PassSpec &ps = sp.pass[kind];
    BandWork b{};
    b.in = src;
    b.out = dst;
    b.weights = p->d_weights;
    b.boxes = p->dev[kind].boxes;
    b.nboxes = (int)ps.boxes.size();
    b.dim = sp.dim;
    b.r = sp.radius;
    b.tau = ps.tau;
    for (int d = 0; d < 3; ++d)
        b.n[d] = sp.n[d];
    b.max_vol = ps.band_max_vol;
    b.taps = p->d_taps;
    b.ntaps = (int)sp.taps.size();
    b.status = p->d_status;
    // 3 x 3 boxes: the warp-row path pays when most staged regions are whole warps wide
    if (sp.dim == 2 && sp.radius == 1 && sp.taps.size() == 9) {
        const int64_t rt = (int64_t)sp.radius * ps.tau;
        size_t wide = 0;
        for (const BandBox &bx : ps.boxes) {
            const int64_t lo = std::max<int64_t>(bx.lo[0] - rt, 0), hi = std::min<int64_t>(bx.lo[0] + bx.ext[0] + rt, sp.n[0]);
            wide += ((hi - lo) & 31) == 0;
        }
        b.warp_rows = 2 * wide >= ps.boxes.size();
    }
    return b;
}

// Which kernel of a pass is launched first.  The butterfly forms' tile kernels (2D, and
// 3D on 16^3 tiles) fill whole SMs with their CTAs (every register), so a band CTA never
// shares an SM with them.  Launched first, the band's CTAs spread over all SMs and every
// tile CTA starts one box's duration late.  Launched after the tile kernel, they run on
// the SMs that its last, partial wave leaves idle (Box2D9P 4096^2: 1849 tiles on 148
// CTAs, 73 in the last wave; 947.7-961.4 -> 967.4-985.2 GStencil/s.  Box3D27P 512^3:
// 40678 pairs on 444 CTAs; 172.5-173.2 -> 180.4-181.3).  With the last wave (nearly)
// full there is no such room (Box2D9P 8192^2: 7396 tiles, 144 in the last wave;
// 1117.6-1126.5 band first, 1110.8-1114.1 after), so the band goes first.
static bool band_goes_first(const ffs_plan *p, const PassSpec &ps)
{
    const PlanSpec &sp = p->spec;
    if (sp.form != FFS_FORM_FP64_FFT || sp.dim == 1 || (sp.dim == 3 && sp.tile == 32))
        return true;
    const int64_t slots = sp.dim == 2 ? std::min<int64_t>(ps.nitems, p->num_sms) : fft3d_grid(ps.nitems, p->num_sms);
    const int64_t tail = ps.nitems % slots;
    return tail == 0 || tail * 10 >= slots * 9;
}

// One fused pass src -> dst with the pass kind's tau.
// The band kernel (when there is one) is forked onto the plan's side stream so it
// runs beside the tile kernel: both read `src` and write disjoint cells of `dst`.
static ffs_status run_pass(const ffs_plan *p, int kind, const double *src, double *dst, cudaStream_t s)
{
    const PlanSpec &sp = p->spec;
    const PassSpec &ps = sp.pass[kind];
    const bool fork = ps.nitems > 0 && !ps.boxes.empty();
    if (fork) {
        CUDA_TRY(cudaEventRecord(p->ev_fork, s));
        CUDA_TRY(cudaStreamWaitEvent(p->side, p->ev_fork, 0));
    }
    auto band = [&]() -> ffs_status {
        if (ps.boxes.empty())
            return FFS_OK;
        BandWork b = band_work(p, kind, src, dst);
        cudaStream_t bs = fork ? p->side : s;
        {
            LaunchMark mark(p, bs, 1);
            cudaError_t e = launch_band(b, band_smem_bytes(ps.band_max_vol, b.ntaps), bs);
            if (e != cudaSuccess)
                return fail(FFS_ERR_CUDA, "band kernel launch: %s", cudaGetErrorString(e));
        }
        if (fork)
            CUDA_TRY(cudaEventRecord(p->ev_join, p->side));
        return FFS_OK;
    };
    const bool band_first = ps.nitems == 0 || band_goes_first(p, ps);
    if (band_first) {
        const ffs_status st = band();
        if (st != FFS_OK)
            return st;
    }
    if (ps.nitems > 0) {
        TileWork w = tile_work(p, kind, src, dst);
        const int grid = (int)std::min<int64_t>(ps.nitems, p->num_sms);
        cudaError_t e = cudaSuccess;
        LaunchMark mark(p, s, 0);
        if (sp.dim == 2 && sp.form == FFS_FORM_FP64_DMMA) {
            CUtensorMap tm;
            w.use_tma = make_tmap_2d(&tm, src, sp.n[0], sp.n[1], dmma2d_tile());
            e = launch_dmma2d(w.use_tma ? &tm : nullptr, w, grid, s);
        } else if (sp.dim == 2 && sp.form == FFS_FORM_FP64_FFT && sp.tile == 128) {
            e = launch_fft2d128(w, grid, s);
        } else if (sp.dim == 2 && sp.form == FFS_FORM_FP64_FFT) {
            CUtensorMap tm;
            w.use_tma = make_tmap_2d_boxes(&tm, src, sp.n[0], sp.n[1]);
            e = launch_fft2d(w.use_tma ? &tm : nullptr, w, grid, s);
        } else if (sp.dim == 2 && (sp.form == FFS_FORM_OZAKI_I8 || sp.form == FFS_FORM_BF16X3)) {
            w.use_tma = 0;
            e = launch_tc2d(sp.form == FFS_FORM_OZAKI_I8 ? kFormOzaki : kFormBf16, sp.slices, w, p->d_aslices, grid,
                            s);
        } else if (sp.dim == 3 && (sp.form == FFS_FORM_OZAKI_I8 || sp.form == FFS_FORM_BF16X3)) {
            e = launch_tc3d(sp.form == FFS_FORM_OZAKI_I8 ? kFormOzaki : kFormBf16, sp.slices, w, p->d_aslices, grid,
                            s);
        } else if (sp.dim == 3 && sp.form == FFS_FORM_FP64_FFT) {
            e = sp.tile == 32 ? launch_fft3d32(w, p->num_sms, s) : launch_fft3d(w, p->num_sms, s);
        } else if (sp.dim == 3 && sp.form == FFS_FORM_FP64_DMMA) {
            CUtensorMap tm;
            w.use_tma = make_tmap_3d(&tm, src, sp.n[0], sp.n[1], sp.n[2], dmma3d_tile());
            e = launch_dmma3d(w.use_tma ? &tm : nullptr, w, grid, s);
        } else if (sp.dim == 1 && sp.form == FFS_FORM_FP64_FFT) {
            w.use_tma = (reinterpret_cast<uintptr_t>(src) & 15) == 0; // bulk copies need 16-B alignment
            e = launch_fft1d(w, grid, s);
        } else if (sp.dim == 1 && sp.form == FFS_FORM_FP64_DMMA) {
            w.use_tma = (reinterpret_cast<uintptr_t>(src) & 15) == 0; // bulk copies need 16-B alignment
            e = launch_dmma1d(w, grid, s);
        } else {
            return fail(FFS_ERR_UNSUPPORTED, "no kernel for dim %d form %d", sp.dim, (int)sp.form);
        }
        if (e != cudaSuccess)
            return fail(FFS_ERR_CUDA, "fused tile kernel launch: %s", cudaGetErrorString(e));
    }
    if (!band_first) {
        const ffs_status st = band();
        if (st != FFS_OK)
            return st;
    }
    if (fork)
        CUDA_TRY(cudaStreamWaitEvent(s, p->ev_join, 0));
    return FFS_OK;
}

// The copy (odd pass count in place) and the passes of one execution on `s`.
static ffs_status launch_passes(const ffs_plan *plan, const double *d_in, double *d_out, cudaStream_t s)
{
    const PlanSpec &sp = plan->spec;
    const int P = sp.passes;
    const double *src = d_in;
    if (d_in == d_out && (P % 2 == 1)) { // the first pass must not write its own input
        CUDA_TRY(cudaMemcpyAsync(plan->d_work, d_in, sp.cells * sizeof(double), cudaMemcpyDeviceToDevice, s));
        src = plan->d_work;
    }
    for (int i = 0; i < P; ++i) {
        double *dst = ((P - 1 - i) % 2 == 0) ? d_out : plan->d_work;
        const int kind = (i == P - 1) ? sp.last_kind : 0;
        ffs_status st = run_pass(plan, kind, src, dst, s);
        if (st != FFS_OK)
            return st;
        src = dst;
    }
    return FFS_OK;
}

// Whether this call repeats the process's previous ffs_execute call (same plan and buffers):
// the tight loop in which a captured graph pays.  Replaying graphs of many different plans
// in turn measured slower than launching them (512 small problems in sequence: 70-74 against
// 62.7 ms), so a graph is used only for such repeats.
static bool repeats_last_call(const ffs_plan *plan, const double *d_in, double *d_out)
{
    static std::mutex mu;
    static const ffs_plan *last_plan = nullptr;
    static const double *last_in = nullptr;
    static double *last_out = nullptr;
    std::lock_guard<std::mutex> lk(mu);
    const bool same = last_plan == plan && last_in == d_in && last_out == d_out;
    last_plan = plan;
    last_in = d_in;
    last_out = d_out;
    return same;
}

// The plan's graph of (d_in, d_out): found, or captured now on the plan's private stream.
// Called with run_mu held.
static ffs_status cached_graph(const ffs_plan *plan, const double *d_in, double *d_out, cudaGraphExec_t *out)
{
    *out = nullptr;
    ffs_plan::GraphEntry *hit = nullptr, *victim = &plan->graphs[0];
    for (ffs_plan::GraphEntry &g : plan->graphs) {
        if (g.in == d_in && g.out == d_out)
            hit = &g;
        if (g.used < victim->used)
            victim = &g;
    }
    const uint64_t now = ++plan->graph_clock;
    if (!hit) { // a new pair: the least recently used graph makes room
        if (victim->exec)
            cudaGraphExecDestroy(victim->exec);
        *victim = ffs_plan::GraphEntry{d_in, d_out, nullptr, now};
        hit = victim;
    }
    hit->used = now;
    if (!hit->exec) {
        if (!plan->graph_stream)
            CUDA_TRY(cudaStreamCreateWithFlags(&plan->graph_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamBeginCapture(plan->graph_stream, cudaStreamCaptureModeThreadLocal));
        const ffs_status st = launch_passes(plan, d_in, d_out, plan->graph_stream);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(plan->graph_stream, &g);
        if (st != FFS_OK || e != cudaSuccess) {
            if (g)
                cudaGraphDestroy(g);
            (void)cudaGetLastError();
            return st != FFS_OK ? st : fail(FFS_ERR_CUDA, "ffs_execute capture: %s", cudaGetErrorString(e));
        }
        const cudaError_t ei = cudaGraphInstantiate(&hit->exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            (void)cudaGetLastError();
            hit->exec = nullptr;
            return fail(FFS_ERR_CUDA, "ffs_execute graph instantiation: %s", cudaGetErrorString(ei));
        }
    }
    *out = hit->exec;
    return FFS_OK;
}

// One execution.  `graphs`: the public entry point, which replays cached graphs for
// repeated buffer pairs; the library's own pipelines (host buffers, slabs, autotuner,
// batch capture) cycle through many buffer pairs and launch directly.
static ffs_status execute_impl(const ffs_plan *plan, const double *d_in, double *d_out, void *stream, bool graphs)
{
    if (!plan || !d_in || !d_out)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_execute: null argument");
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != plan->device)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_execute: plan was created on device %d, current is %d",
                    plan->device, dev);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const PlanSpec &sp = plan->spec;
    const size_t bytes = sp.cells * sizeof(double);
    const int P = sp.passes;
    // the launches below are checked with cudaGetLastError: start from a clean slate, so an
    // earlier failed runtime call (handled by its caller) is not reported as a launch failure
    (void)cudaGetLastError();
    if (P == 0) {
        if (d_in != d_out)
            CUDA_TRY(cudaMemcpyAsync(d_out, d_in, bytes, cudaMemcpyDeviceToDevice, s));
        return FFS_OK;
    }
    std::lock_guard<std::mutex> lk(plan->run_mu); // side stream and fork/join events are per plan
    // the workspace may still be in use by the previous execution on another stream; inside
    // a graph capture (a batch) the graph's own edges order the work instead
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(s, &cap));
    const bool capturing = cap != cudaStreamCaptureStatusNone;
    cudaGraphExec_t gexec = nullptr;
    if (graphs && !capturing && !plan->profiling && repeats_last_call(plan, d_in, d_out)) {
        const ffs_status st = cached_graph(plan, d_in, d_out, &gexec);
        if (st != FFS_OK)
            return st;
    }
    if (plan->ran && !capturing)
        CUDA_TRY(cudaStreamWaitEvent(s, plan->ev_last, 0));
    if (gexec) {
        CUDA_TRY(cudaGraphLaunch(gexec, s));
    } else {
        const ffs_status st = launch_passes(plan, d_in, d_out, s);
        if (st != FFS_OK)
            return st;
    }
    if (!capturing) {
        CUDA_TRY(cudaEventRecord(plan->ev_last, s));
        plan->ran = true;
    }
    return FFS_OK;
}

extern "C" ffs_status ffs_execute(const ffs_plan *plan, const double *d_in, double *d_out, void *stream)
{
    return execute_impl(plan, d_in, d_out, stream, true);
}

// Creates the host-buffer pipeline's streams, events and input slots on first
// use; the whole-grid output slots only when `whole` (the slab path has its own).
static ffs_status host_pipe_setup(const ffs_plan *plan, size_t bytes, bool whole)
{
    auto &h = plan->host;
    for (int k = 0; k < 2; ++k) {
        if (!h.in[k])
            CUDA_TRY(cudaMalloc(&h.in[k], bytes));
        if (whole && !h.out[k])
            CUDA_TRY(cudaMalloc(&h.out[k], bytes));
        for (cudaEvent_t *e : {&h.in_ready[k], &h.comp_done[k], &h.out_done[k]})
            if (!*e)
                CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    if (!h.start)
        CUDA_TRY(cudaEventCreateWithFlags(&h.start, cudaEventDisableTiming));
    if (!h.s_in)
        CUDA_TRY(cudaStreamCreateWithFlags(&h.s_in, cudaStreamNonBlocking));
    if (!h.s_out)
        CUDA_TRY(cudaStreamCreateWithFlags(&h.s_out, cudaStreamNonBlocking));
    return FFS_OK;
}

// ---- slab pipeline for host buffers ----

// Builds the slab layout, its sub-plans, buffers and events (first slab call).
// Leaves count = 1 when a sub-plan cannot be built, so the caller falls back to
// the whole-grid pipeline.
static ffs_status slab_setup(const ffs_plan *plan, const SlabModel &m)
{
    auto &sl = plan->host.slabs;
    const PlanSpec &sp = plan->spec;
    const int axis = sp.dim - 1;
    const int64_t n = sp.n[axis];
    const int64_t h = (n + m.count - 1) / m.count;
    const int K = (int)((n + h - 1) / h);
    const bool periodic = sp.boundary == FFS_BOUNDARY_PERIODIC;
    sl.axis = axis;
    sl.row = (int64_t)sp.cells / n;
    sl.ghost = (int64_t)sp.radius * sp.T;
    sl.a.assign(K + 1, 0);
    for (int j = 0; j <= K; ++j)
        sl.a[j] = std::min<int64_t>((int64_t)j * h, n);
    sl.lo.assign(K, 0);
    sl.hi.assign(K, 0);
    sl.sub.assign(K, 0);
    sl.last_chunk.assign(K, 0);
    std::vector<int64_t> key_rows;
    std::vector<int> key_open;
    int64_t wrap_rows = 0;
    for (int j = 0; j < K; ++j) {
        int64_t lo = sl.a[j] - sl.ghost, hi = sl.a[j + 1] + sl.ghost;
        int open = 0;
        if (!periodic) {
            lo = std::max<int64_t>(lo, 0);
            hi = std::min<int64_t>(hi, n);
            open = (lo > 0 ? 1 << (2 * axis) : 0) | (hi < n ? 2 << (2 * axis) : 0); // a clipped face is real
        }
        sl.lo[j] = lo;
        sl.hi[j] = hi;
        const bool wraps = lo < 0 || hi > n;
        if (wraps)
            wrap_rows = std::max(wrap_rows, hi - lo);
        sl.last_chunk[j] = wraps ? K - 1 : (int)((hi - 1) / h);
        int idx = -1;
        for (size_t u = 0; u < key_rows.size(); ++u)
            if (key_rows[u] == hi - lo && key_open[u] == open)
                idx = (int)u;
        if (idx < 0) {
            ffs_problem q = slab_problem(sp, hi - lo, open);
            ffs_plan *sub = nullptr;
            if (ffs_plan_create(&sub, &q) != FFS_OK) {
                release_slabs(sl);
                return FFS_OK;
            }
            idx = (int)sl.plans.size();
            sl.plans.push_back(sub);
            key_rows.push_back(hi - lo);
            key_open.push_back(open);
        }
        sl.sub[j] = idx;
        sl.max_rows = std::max(sl.max_rows, hi - lo);
    }
    // slabs in the order their last input chunk arrives (chunks arrive in row order)
    sl.order.resize(K);
    for (int j = 0; j < K; ++j)
        sl.order[j] = j;
    std::stable_sort(sl.order.begin(), sl.order.end(),
                     [&](int x, int y) { return sl.last_chunk[x] < sl.last_chunk[y]; });
    const size_t slab_bytes = (size_t)(sl.max_rows * sl.row) * sizeof(double);
    for (int r = 0; r < 3; ++r) {
        CUDA_TRY(cudaMalloc(&sl.ring[r], slab_bytes));
        CUDA_TRY(cudaEventCreateWithFlags(&sl.comp_done[r], cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&sl.out_done[r], cudaEventDisableTiming));
    }
    if (wrap_rows > 0)
        CUDA_TRY(cudaMalloc(&sl.wrap, (size_t)(wrap_rows * sl.row) * sizeof(double)));
    for (int k = 0; k < 2; ++k) {
        sl.chunk[k].assign(K, nullptr);
        for (cudaEvent_t &e : sl.chunk[k])
            CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&sl.grid_done[k], cudaEventDisableTiming));
    }
    sl.count = K;
    return FFS_OK;
}

// The slab pipeline over `count` grids.  Per grid (input slot k = i % 2): the
// copy-in stream copies the slabs' interiors in row order, one event per chunk;
// slab j's compute (on `stream`) waits for the last chunk it reads and for its
// output ring slot's previous copy-out, runs its sub-plan on a view of the slot
// (or, for a periodic slab that wraps, on rows assembled modulo n), and the
// copy-out stream then copies its interior rows to the host.  Grid i + 2's
// copy-in waits until grid i's last slab has read the slot.
static cudaError_t slab_enqueue(const ffs_plan *plan, int count, const double *const *h_in, double *const *h_out,
                                cudaStream_t s, ffs_status *st)
{
    auto &h = plan->host;
    auto &sl = h.slabs;
    const int K = sl.count;
    const int64_t n = plan->spec.n[sl.axis];
    const size_t rb = (size_t)sl.row * sizeof(double);
    int slot = 0;
    for (int r = 0; r < 3; ++r)
        sl.ring_used[r] = false;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < count; ++i) {
        const int k = i & 1;
        double *in = h.in[k];
        if (i >= 2 && (e = cudaStreamWaitEvent(h.s_in, sl.grid_done[k], 0)) != cudaSuccess)
            return e;
        size_t next = 0; // position in sl.order
        for (int c = 0; c < K; ++c) {
            const int64_t off = sl.a[c] * sl.row;
            if ((e = cudaMemcpyAsync(in + off, h_in[i] + off, (size_t)(sl.a[c + 1] - sl.a[c]) * rb,
                                     cudaMemcpyHostToDevice, h.s_in)) != cudaSuccess ||
                (e = cudaEventRecord(sl.chunk[k][c], h.s_in)) != cudaSuccess)
                return e;
            for (; next < sl.order.size() && sl.last_chunk[sl.order[next]] == c; ++next) {
                const int j = sl.order[next];
                const int r = slot++ % 3;
                if ((e = cudaStreamWaitEvent(s, sl.chunk[k][c], 0)) != cudaSuccess)
                    return e;
                if (sl.ring_used[r] && (e = cudaStreamWaitEvent(s, sl.out_done[r], 0)) != cudaSuccess)
                    return e;
                const double *src = in + sl.lo[j] * sl.row;
                if (sl.lo[j] < 0 || sl.hi[j] > n) { // periodic wrap: rows lo..hi modulo n
                    for (int64_t y = sl.lo[j]; y < sl.hi[j];) {
                        const int64_t m = ((y % n) + n) % n, len = std::min(sl.hi[j] - y, n - m);
                        if ((e = cudaMemcpyAsync(sl.wrap + (y - sl.lo[j]) * sl.row, in + m * sl.row, (size_t)len * rb,
                                                 cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
                            return e;
                        y += len;
                    }
                    src = sl.wrap;
                }
                *st = execute_impl(sl.plans[sl.sub[j]], src, sl.ring[r], s, false);
                if (*st != FFS_OK)
                    return cudaSuccess;
                const int64_t skip = sl.a[j] - sl.lo[j], rows = sl.a[j + 1] - sl.a[j];
                if ((e = cudaEventRecord(sl.comp_done[r], s)) != cudaSuccess ||
                    (e = cudaStreamWaitEvent(h.s_out, sl.comp_done[r], 0)) != cudaSuccess ||
                    (e = cudaMemcpyAsync(h_out[i] + sl.a[j] * sl.row, sl.ring[r] + skip * sl.row, (size_t)rows * rb,
                                         cudaMemcpyDeviceToHost, h.s_out)) != cudaSuccess ||
                    (e = cudaEventRecord(sl.out_done[r], h.s_out)) != cudaSuccess)
                    return e;
                sl.ring_used[r] = true;
            }
        }
        if ((e = cudaEventRecord(sl.grid_done[k], s)) != cudaSuccess)
            return e;
    }
    // `stream` completes only after the last copy-out
    for (int r = 0; r < 3; ++r)
        if (sl.ring_used[r] && (e = cudaStreamWaitEvent(s, sl.out_done[r], 0)) != cudaSuccess)
            return e;
    return cudaSuccess;
}

// Whole-grid pipeline: grid i uses slot i % 2.  Copy-in of grid i waits until
// the compute of grid i - 2 has read the slot's input; its compute (on
// `stream`) waits for the copy-in and for the copy-out of grid i - 2 to have
// read the slot's output; its copy-out waits for its compute.
static cudaError_t whole_enqueue(const ffs_plan *plan, int count, const double *const *h_in, double *const *h_out,
                                 cudaStream_t s, ffs_status *st)
{
    auto &h = plan->host;
    const size_t bytes = plan->spec.cells * sizeof(double);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < count; ++i) {
        const int k = i & 1;
        if ((i >= 2 && (e = cudaStreamWaitEvent(h.s_in, h.comp_done[k], 0)) != cudaSuccess) ||
            (e = cudaMemcpyAsync(h.in[k], h_in[i], bytes, cudaMemcpyHostToDevice, h.s_in)) != cudaSuccess ||
            (e = cudaEventRecord(h.in_ready[k], h.s_in)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(s, h.in_ready[k], 0)) != cudaSuccess ||
            (i >= 2 && (e = cudaStreamWaitEvent(s, h.out_done[k], 0)) != cudaSuccess))
            return e;
        *st = execute_impl(plan, h.in[k], h.out[k], s, false);
        if (*st != FFS_OK)
            return cudaSuccess;
        if ((e = cudaEventRecord(h.comp_done[k], s)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(h.s_out, h.comp_done[k], 0)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h_out[i], h.out[k], bytes, cudaMemcpyDeviceToHost, h.s_out)) != cudaSuccess ||
            (e = cudaEventRecord(h.out_done[k], h.s_out)) != cudaSuccess)
            return e;
    }
    // `stream` completes only after the last copy-out
    if (count > 0 && (e = cudaStreamWaitEvent(s, h.out_done[(count - 1) & 1], 0)) != cudaSuccess)
        return e;
    if (count > 1 && (e = cudaStreamWaitEvent(s, h.out_done[count & 1], 0)) != cudaSuccess)
        return e;
    return cudaSuccess;
}

// Host-buffer execution of `count` grids.  The slab pipeline (built on the
// first call when the model prefers it for one grid) is used when its modelled
// time for `count` grids beats the whole-grid pipeline's by 10 %, or always
// when FFS_HOST_SLABS forces it.
static ffs_status host_pipeline(const ffs_plan *plan, int count, const double *const *h_in, double *const *h_out,
                                cudaStream_t s, const char *who)
{
    const size_t bytes = plan->spec.cells * sizeof(double);
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != plan->device) // the pipeline's buffers and slab sub-plans live on the plan's device
        return fail(FFS_ERR_INVALID_ARGUMENT, "%s: plan was created on device %d, current is %d", who, plan->device,
                    dev);
    std::lock_guard<std::mutex> lk(plan->host_mu);
    auto &h = plan->host;
    auto &sl = h.slabs;
    ffs_status st = FFS_OK;
    if (!sl.decided) {
        sl.decided = true;
        sl.model = slab_model(plan->spec);
        // a slab layout that cannot be built (device memory for the sub-plans and slab
        // buffers) leaves the whole-grid pipeline, which needs less memory
        if (sl.model.count > 1 && slab_setup(plan, sl.model) != FFS_OK)
            release_slabs(sl);
    }
    // many grids keep the whole-grid pipeline unless the slabs win clearly: with both at the copy
    // bound, the slabs' shorter copies measured about 5 % slower per grid
    const bool slabs = sl.count > 1 && (sl.model.forced || sl.model.slabs(count) < 0.9 * sl.model.whole(count));
    if ((st = host_pipe_setup(plan, bytes, !slabs)) != FFS_OK)
        return st;
    std::vector<const ffs_plan *> status_of{plan};
    if (slabs)
        status_of.insert(status_of.end(), sl.plans.begin(), sl.plans.end());
    cudaError_t e = cudaSuccess;
    for (const ffs_plan *q : status_of)
        if (e == cudaSuccess)
            e = cudaMemsetAsync(q->d_status, 0, sizeof(int), s);
    if (e == cudaSuccess)
        e = cudaEventRecord(h.start, s); // the pipeline starts after prior work on `stream`
    if (e == cudaSuccess)
        e = cudaStreamWaitEvent(h.s_in, h.start, 0);
    if (e == cudaSuccess)
        e = slabs ? slab_enqueue(plan, count, h_in, h_out, s, &st) : whole_enqueue(plan, count, h_in, h_out, s, &st);
    std::vector<int> dstatus(status_of.size(), 0);
    for (size_t u = 0; u < status_of.size() && e == cudaSuccess && st == FFS_OK; ++u)
        e = cudaMemcpyAsync(&dstatus[u], status_of[u]->d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
    // drain all three streams whatever happened, so no copy outlives the call
    cudaError_t se = cudaStreamSynchronize(s);
    cudaError_t si = cudaStreamSynchronize(h.s_in);
    cudaError_t so = cudaStreamSynchronize(h.s_out);
    if (st != FFS_OK)
        return st;
    for (cudaError_t x : {se, si, so})
        if (e == cudaSuccess)
            e = x;
    if (e != cudaSuccess)
        return fail(FFS_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
    for (int d : dstatus) {
        if (d == kDevTimeoutTma || d == kDevTimeoutMma)
            return fail(FFS_ERR_TIMEOUT, "device wait timed out (code %d)", d);
        if (d != 0)
            return fail(FFS_ERR_INTERNAL, "device reported error code %d", d);
    }
    return FFS_OK;
}

extern "C" ffs_status ffs_execute_host(const ffs_plan *plan, const double *h_in, double *h_out, void *stream)
{
    if (!plan || !h_in || !h_out)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_execute_host: null argument");
    return host_pipeline(plan, 1, &h_in, &h_out, reinterpret_cast<cudaStream_t>(stream), "ffs_execute_host");
}

extern "C" ffs_status ffs_execute_host_many(const ffs_plan *plan, int count, const double *const *h_in,
                                            double *const *h_out, void *stream)
{
    if (!plan || count < 0 || (count > 0 && (!h_in || !h_out)))
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_execute_host_many: null argument or negative count");
    for (int i = 0; i < count; ++i)
        if (!h_in[i] || !h_out[i])
            return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_execute_host_many: null buffer for grid %d", i);
    if (count == 0)
        return FFS_OK;
    return host_pipeline(plan, count, h_in, h_out, reinterpret_cast<cudaStream_t>(stream), "ffs_execute_host_many");
}

extern "C" ffs_status ffs_plan_get_info(const ffs_plan *plan, ffs_plan_info *info)
{
    if (!plan || !info)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_plan_get_info: null argument");
    fill_plan_info(plan->spec, info);
    info->work_bytes = plan->d_work ? (int64_t)(plan->spec.cells * sizeof(double)) : 0;
    return FFS_OK;
}

// Max |y - r| / max |r| over n cells, on the device (synchronises `s`); -1 on failure.
static double device_rel_diff(const double *y, const double *r, size_t n, unsigned long long *d_acc, cudaStream_t s)
{
    unsigned long long h[2] = {0, 0};
    if (cudaMemsetAsync(d_acc, 0, 2 * sizeof(unsigned long long), s) != cudaSuccess ||
        launch_max_diff(y, r, n, d_acc, s) != cudaSuccess ||
        cudaMemcpyAsync(h, d_acc, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        (void)cudaGetLastError();
        return -1.0;
    }
    double md, mr;
    memcpy(&md, &h[0], 8);
    memcpy(&mr, &h[1], 8);
    return mr > 0.0 ? md / mr : md;
}

// Ozaki slice count of `problem`'s class: the smallest s in [4, 8] whose solve of a
// seeded uniform [0, 1) grid differs from the FP64 butterfly form's solve by at most
// kSliceCalibrationTol (max relative difference); 8 if none does.  Recorded in the
// tuning table under slice_key.
static ffs_status calibrate_slices(const ffs_problem &problem, const PlanSpec &spec, double *din, double *dout,
                                   cudaStream_t s, int *chosen)
{
    const size_t bytes = spec.cells * sizeof(double);
    double *dref = nullptr;
    unsigned long long *acc = nullptr;
    if (cudaMalloc(&dref, bytes) != cudaSuccess || cudaMalloc(&acc, 2 * sizeof(unsigned long long)) != cudaSuccess) {
        (void)cudaGetLastError();
        cudaFree(dref);
        return fail(FFS_ERR_OUT_OF_MEMORY, "ffs_autotune: calibration scratch allocation failed");
    }
    ffs_status st = FFS_OK;
    *chosen = 0;
    if (launch_fill_uniform(din, spec.cells, 0x5eed5eedull, s) != cudaSuccess) {
        (void)cudaGetLastError();
        st = fail(FFS_ERR_CUDA, "ffs_autotune: calibration fill failed");
    }
    ffs_problem qref = problem;
    qref.form = FFS_FORM_FP64_FFT;
    qref.slices = 0;
    ffs_plan *ref = nullptr;
    if (st == FFS_OK && (st = ffs_plan_create(&ref, &qref)) == FFS_OK) {
        st = execute_impl(ref, din, dref, s, false);
        ffs_plan_destroy(ref);
    }
    for (int sl = 4; sl <= 8 && st == FFS_OK && !*chosen; ++sl) {
        ffs_problem q = problem;
        q.slices = sl;
        ffs_plan *p = nullptr;
        if ((st = ffs_plan_create(&p, &q)) != FFS_OK)
            break;
        st = execute_impl(p, din, dout, s, false);
        ffs_plan_destroy(p);
        if (st != FFS_OK)
            break;
        const double err = device_rel_diff(dout, dref, spec.cells, acc, s);
        if (err < 0.0)
            st = fail(FFS_ERR_CUDA, "ffs_autotune: calibration comparison failed");
        else if (err <= kSliceCalibrationTol || sl == 8)
            *chosen = sl;
    }
    cudaFree(dref);
    cudaFree(acc);
    if (st == FFS_OK)
        tune_record(slice_key(spec), *chosen);
    return st;
}

// Measured autotuning of the fused step count, and of the Ozaki slice count when
// the problem leaves it open (see include/ffs.h).
extern "C" ffs_status ffs_autotune(const ffs_problem *problem, int candidates, int *best_tau, double *best_ms,
                                   void *stream)
{
    if (!problem || !best_tau)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_autotune: null argument");
    PlanSpec spec;
    std::string why;
    ffs_status st = build_plan_spec(*problem, &spec, &why, false);
    if (st != FFS_OK)
        return fail(st, "%s", why.c_str());
    *best_tau = 0;
    if (spec.T == 0)
        return FFS_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t bytes = spec.cells * sizeof(double);
    double *din = nullptr, *dout = nullptr;
    CUDA_TRY(cudaMalloc(&din, bytes));
    if (cudaMalloc(&dout, bytes) != cudaSuccess) {
        (void)cudaGetLastError(); // handled here: not to be seen by a later launch check
        cudaFree(din);
        return fail(FFS_ERR_OUT_OF_MEMORY, "ffs_autotune: scratch allocation failed");
    }
    // the 3D butterfly form has two tile edges: the model's candidates of each are timed
    std::vector<int> tiles = {problem->tile};
    if (spec.form == FFS_FORM_FP64_FFT && (spec.dim == 2 || spec.dim == 3) && problem->tile == 0)
        tiles = spec.dim == 2 ? std::vector<int>{64, 128} : std::vector<int>{16, 32};
    cudaMemsetAsync(din, 0x3f, bytes, s); // finite FP64 pattern (0x3f3f... ~ 4.8e-4)
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int arg = 0, arg_tile = 0;
    for (int tile : tiles) {
        ffs_problem base = *problem;
        base.tile = tile;
        double tile_best = 1e300;
        int tile_arg = 0;
        for (int tau : tau_candidates(base, candidates > 0 ? candidates : 6)) {
            ffs_problem q = base;
            q.tau = tau;
            ffs_plan *p = nullptr;
            if (ffs_plan_create(&p, &q) != FFS_OK)
                continue;
            execute_impl(p, din, dout, stream, false); // warm-up
            float ms = 0.f, mn = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                cudaEventRecord(e0, s);
                execute_impl(p, din, dout, stream, false);
                cudaEventRecord(e1, s);
                cudaEventSynchronize(e1);
                cudaEventElapsedTime(&ms, e0, e1);
                mn = std::min(mn, ms);
            }
            ffs_plan_destroy(p);
            if (mn < tile_best) {
                tile_best = mn;
                tile_arg = tau;
            }
        }
        PlanSpec at;
        if (tile_arg && build_plan_spec(base, &at, &why, false) == FFS_OK)
            tune_record(tune_key(at), tile_arg); // this edge's best step count
        if (tile_arg && tile_best < best) {
            best = tile_best;
            arg = tile_arg;
            arg_tile = at.tile;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!arg) {
        cudaFree(din);
        cudaFree(dout);
        return fail(FFS_ERR_INTERNAL, "ffs_autotune: no candidate could run");
    }
    if (tiles.size() > 1)
        tune_record(tile_key(spec), arg_tile);
    if (spec.form == FFS_FORM_OZAKI_I8 && problem->slices == 0) {
        // the slice count at the chosen fused step count, recorded with that count
        ffs_problem q = *problem;
        q.tau = arg;
        int sl = 0;
        st = calibrate_slices(q, spec, din, dout, s, &sl);
        if (st == FFS_OK) {
            q.slices = sl;
            PlanSpec at;
            if (build_plan_spec(q, &at, &why, false) == FFS_OK) {
                at.tau = arg;
                tune_record(tune_key(at), arg);
            }
        }
    }
    cudaFree(din);
    cudaFree(dout);
    if (st != FFS_OK)
        return st;
    *best_tau = arg;
    if (best_ms)
        *best_ms = best;
    return FFS_OK;
}

extern "C" ffs_status ffs_plan_profile(ffs_plan *plan, int enable)
{
    if (!plan)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_plan_profile: null plan");
    plan->profiling = enable != 0;
    return FFS_OK;
}

extern "C" ffs_status ffs_plan_profile_read(ffs_plan *plan, ffs_profile *out, int reset)
{
    if (!plan || !out)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_plan_profile_read: null argument");
    memset(out, 0, sizeof(*out));
    if (!plan->marks.empty())
        CUDA_TRY(cudaEventSynchronize(plan->marks.back().b));
    for (auto &m : plan->marks) {
        float ms = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&ms, m.a, m.b));
        if (m.kind == 0) {
            out->tile_ms += ms;
            out->tile_launches++;
        } else {
            out->band_ms += ms;
            out->band_launches++;
        }
    }
    if (reset)
        clear_marks(plan);
    return FFS_OK;
}

extern "C" ffs_status ffs_shape_lookup(const char *name, ffs_shape *shape, int *dim, int *radius,
                                       const char **label, double *weights, int weights_len)
{
    const ShapeDef *sd = find_shape(name);
    if (!sd)
        return fail(FFS_ERR_INVALID_ARGUMENT, "unknown stencil shape '%s'", name ? name : "(null)");
    if (shape)
        *shape = sd->id;
    if (dim)
        *dim = sd->dim;
    if (radius)
        *radius = sd->radius;
    if (label)
        *label = sd->label;
    if (weights) {
        const std::vector<double> w = shape_weights(*sd);
        if (weights_len < (int)w.size())
            return fail(FFS_ERR_INVALID_ARGUMENT, "weights buffer too small: need %d", (int)w.size());
        std::copy(w.begin(), w.end(), weights);
    }
    return FFS_OK;
}

// ---- batches: one captured CUDA graph replaying every plan's passes ----
extern "C" ffs_status ffs_batch_create(ffs_batch **out, ffs_plan *const *plans, int count)
{
    if (!out || (!plans && count > 0) || count < 0)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_batch_create: bad arguments");
    *out = nullptr;
    ffs_batch *b = new ffs_batch();
    if (const char *polls = std::getenv("FFS_BATCH_WAIT_POLLS")) { // bound of the dependency waits
        char *end = nullptr;
        const unsigned long v = std::strtoul(polls, &end, 10);
        if (end != polls && *end == '\0' && v <= kDepSpinLimit)
            b->dep_limit = (uint32_t)v;
    }
    cudaGetDevice(&b->device);
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device);
    if (cudaMalloc(&b->d_head, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&b->d_status, sizeof(int)) != cudaSuccess || cudaMemset(b->d_status, 0, sizeof(int)) != cudaSuccess) {
        (void)cudaGetLastError(); // handled here: not to be seen by a later launch check
        cudaFree(b->d_head);
        cudaFree(b->d_status);
        delete b;
        return fail(FFS_ERR_OUT_OF_MEMORY, "ffs_batch_create: device allocation failed");
    }
    for (int i = 0; i < count; ++i) {
        if (!plans[i]) {
            cudaFree(b->d_head);
            cudaFree(b->d_status);
            delete b;
            return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_batch_create: plan %d is null", i);
        }
        b->plans.push_back(plans[i]);
    }
    *out = b;
    return FFS_OK;
}

// Level-ordered stage list of every FP64 plan's passes (the persistent kernel's
// queue); pre-copies for in-place odd-pass problems and T = 0 copies go to `copies`.
struct CopyOp {
    double *dst;
    const double *src;
    size_t bytes;
};

static ffs_status build_queue(ffs_batch *b, const double *const *ins, double *const *outs, std::vector<CopyOp> *copies,
                              std::vector<size_t> *others)
{
    release_batch_queue(b);
    std::vector<BatchStage> stages;
    std::vector<int64_t> start;
    struct Seq {
        std::vector<const double *> src;
        std::vector<double *> dst;
        std::vector<int> kind;
        int last_stage = -1;
    };
    const size_t n = b->plans.size();
    std::vector<Seq> seq(n);
    int max_passes = 0;
    size_t smem = batch_tile_smem_bytes();
    for (size_t i = 0; i < n; ++i) {
        const ffs_plan *p = b->plans[i];
        const PlanSpec &sp = p->spec;
        const size_t bytes = sp.cells * sizeof(double);
        if (sp.form != FFS_FORM_FP64_DMMA) {
            others->push_back(i);
            continue;
        }
        const int P = sp.passes;
        if (P == 0) {
            if (ins[i] != outs[i])
                copies->push_back({outs[i], ins[i], bytes});
            continue;
        }
        const double *src = ins[i];
        if (ins[i] == outs[i] && (P % 2 == 1)) {
            copies->push_back({p->d_work, ins[i], bytes});
            src = p->d_work;
        }
        for (int k = 0; k < P; ++k) {
            double *dst = ((P - 1 - k) % 2 == 0) ? outs[i] : p->d_work;
            seq[i].src.push_back(src);
            seq[i].dst.push_back(dst);
            seq[i].kind.push_back(k == P - 1 ? sp.last_kind : 0);
            src = dst;
        }
        max_passes = std::max(max_passes, P);
    }
    int64_t total = 0;
    for (int lvl = 0; lvl < max_passes; ++lvl)
        for (size_t i = 0; i < n; ++i) {
            if ((int)seq[i].src.size() <= lvl)
                continue;
            const ffs_plan *p = b->plans[i];
            const int kind = seq[i].kind[lvl];
            BatchStage st{};
            st.tw = tile_work(p, kind, seq[i].src[lvl], seq[i].dst[lvl]);
            st.tw.use_tma = 0;
            st.bw = band_work(p, kind, seq[i].src[lvl], seq[i].dst[lvl]);
            st.dim = p->spec.dim;
            st.dep = seq[i].last_stage;
            st.dep_count = st.dep >= 0 ? stages[st.dep].tw.nitems + stages[st.dep].bw.nboxes : 0;
            if (st.bw.nboxes > 0)
                smem = std::max(smem, band_smem_bytes(st.bw.max_vol, st.bw.ntaps));
            seq[i].last_stage = (int)stages.size();
            start.push_back(total);
            total += st.tw.nitems + st.bw.nboxes;
            stages.push_back(st);
        }
    b->nstages = (int)stages.size();
    b->total = total;
    b->smem = smem;
    if (stages.empty())
        return FFS_OK;
    CUDA_TRY(cudaMalloc(&b->d_stages, stages.size() * sizeof(BatchStage)));
    CUDA_TRY(cudaMalloc(&b->d_start, start.size() * sizeof(int64_t)));
    CUDA_TRY(cudaMalloc(&b->d_done, stages.size() * sizeof(int)));
    CUDA_TRY(cudaMemcpy(b->d_stages, stages.data(), stages.size() * sizeof(BatchStage), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(b->d_start, start.data(), start.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
    return FFS_OK;
}

extern "C" ffs_status ffs_batch_execute(ffs_batch *b, const double *const *ins, double *const *outs, void *stream)
{
    if (!b || (!b->plans.empty() && (!ins || !outs)))
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_batch_execute: bad arguments");
    const size_t n = b->plans.size();
    for (size_t i = 0; i < n; ++i)
        if (!ins[i] || !outs[i])
            return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_batch_execute: null buffer for problem %zu", i);
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != b->device)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_batch_execute: batch was created on device %d", b->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    (void)cudaGetLastError(); // launches below are checked with cudaGetLastError (see ffs_execute)
    bool same = b->exec && b->stream == s && b->ins.size() == n;
    for (size_t i = 0; same && i < n; ++i)
        same = b->ins[i] == ins[i] && b->outs[i] == outs[i];
    if (!same) {
        if (b->exec)
            cudaGraphExecDestroy(b->exec);
        if (b->graph)
            cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
        std::vector<CopyOp> copies;
        std::vector<size_t> others;
        ffs_status st = build_queue(b, ins, outs, &copies, &others);
        if (st != FFS_OK)
            return st;
        cudaStream_t cap = s;
        bool own = false;
        if (!cap) { // the legacy stream cannot be captured; capture on a private stream
            CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            own = true;
        }
        CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaSuccess;
        for (const CopyOp &c : copies)
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToDevice, cap);
        if (e == cudaSuccess) // every replay starts with a clear status word
            e = cudaMemsetAsync(b->d_status, 0, sizeof(int), cap);
        if (e == cudaSuccess && b->nstages > 0) {
            e = cudaMemsetAsync(b->d_done, 0, b->nstages * sizeof(int), cap);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(b->d_head, 0, sizeof(unsigned long long), cap);
            if (e == cudaSuccess)
                e = launch_batch(b->d_stages, b->d_start, b->nstages, b->total, b->d_done, b->d_head, b->d_status,
                                 b->dep_limit, b->smem, (int)std::min<int64_t>(b->total, b->num_sms), cap);
        }
        if (e == cudaSuccess && !others.empty()) {
            // fork the branches off the capture stream.  Longest first onto the least loaded
            // branch, by the plan builder's modelled time: the branches run side by side, so the
            // batch ends with its longest branch.  Every execution of one plan stays on one
            // branch, since they share the plan's workspace.
            e = ensure_branches(b);
            if (e == cudaSuccess)
                e = cudaEventRecord(b->bfork, cap);
            for (int k = 0; k < ffs_batch::kBranches && e == cudaSuccess; ++k)
                e = cudaStreamWaitEvent(b->branch[k], b->bfork, 0);
            std::stable_sort(others.begin(), others.end(), [&](size_t x, size_t y) {
                return b->plans[x]->spec.est_seconds > b->plans[y]->spec.est_seconds;
            });
            std::map<const ffs_plan *, int> branch_of;
            double load[ffs_batch::kBranches] = {};
            for (size_t k = 0; k < others.size() && e == cudaSuccess && st == FFS_OK; ++k) {
                const ffs_plan *pl = b->plans[others[k]];
                auto it = branch_of.find(pl);
                if (it == branch_of.end())
                    it = branch_of.emplace(pl, (int)(std::min_element(load, load + ffs_batch::kBranches) - load)).first;
                load[it->second] += pl->spec.est_seconds;
                st = execute_impl(pl, ins[others[k]], outs[others[k]], b->branch[it->second], false);
            }
            for (int k = 0; k < ffs_batch::kBranches && b->bjoin[k]; ++k) { // join even after an error
                cudaError_t ej = cudaEventRecord(b->bjoin[k], b->branch[k]);
                if (ej == cudaSuccess)
                    ej = cudaStreamWaitEvent(cap, b->bjoin[k], 0);
                if (e == cudaSuccess)
                    e = ej;
            }
        }
        cudaGraph_t g = nullptr;
        cudaError_t ee = cudaStreamEndCapture(cap, &g);
        if (own)
            cudaStreamDestroy(cap);
        if (st != FFS_OK || e != cudaSuccess || ee != cudaSuccess) {
            if (g)
                cudaGraphDestroy(g);
            if (st != FFS_OK)
                return st;
            return fail(FFS_ERR_CUDA, "batch capture: %s", cudaGetErrorString(e != cudaSuccess ? e : ee));
        }
        b->graph = g;
        CUDA_TRY(cudaGraphInstantiate(&b->exec, g, 0));
        b->ins.assign(ins, ins + n);
        b->outs.assign(outs, outs + n);
        b->stream = s;
    }
    CUDA_TRY(cudaGraphLaunch(b->exec, s));
    return FFS_OK;
}

// Device status of the last batch run (0 = ok); synchronises the batch's stream.
extern "C" ffs_status ffs_batch_status(ffs_batch *b, int *device_status)
{
    if (!b || !device_status)
        return fail(FFS_ERR_INVALID_ARGUMENT, "ffs_batch_status: null argument");
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    CUDA_TRY(cudaMemcpy(device_status, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (*device_status != 0)
        return fail(FFS_ERR_TIMEOUT, "ffs_batch_status: a bounded device wait gave up (code %d)", *device_status);
    return FFS_OK;
}

extern "C" ffs_status ffs_batch_destroy(ffs_batch *b)
{
    if (!b)
        return FFS_OK;
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    if (b->graph)
        cudaGraphDestroy(b->graph);
    release_batch_queue(b);
    cudaFree(b->d_head);
    cudaFree(b->d_status);
    for (int k = 0; k < ffs_batch::kBranches; ++k) {
        if (b->branch[k])
            cudaStreamDestroy(b->branch[k]);
        if (b->bjoin[k])
            cudaEventDestroy(b->bjoin[k]);
    }
    if (b->bfork)
        cudaEventDestroy(b->bfork);
    delete b;
    return FFS_OK;
}

extern "C" const char *ffs_last_error_string(void) { return g_err.c_str(); }
extern "C" int ffs_abi_version(void) { return FFS_ABI_VERSION; }
