/*
 * ffs.h - C ABI of the B200 fused DFT-tile stencil solver (libffs.so).
 *
 * The reference (FlashFFTStencil) has no library: its surface is three CLI
 * programs, a host function that fills __constant__ memory, and a fused tile
 * kernel launched T times on caller-owned buffers.  Each entry point below
 * replaces one piece of that surface:
 *
 *   ffs_plan_create    <- void CreatePlan(double* k, int K, bool print)
 *                         src/1D/create_fft_pfa_plan.cu:19, src/2D/create_fft_pfa_plan.cu:17,
 *                         src/3D/create_fft_pfa_plan.cu:17 (DFT matrices + cuFFT kernel
 *                         spectrum uploaded to __constant__); here a plan object owns
 *                         its spectra and tables, so plans are re-entrant.
 *   ffs_execute        <- the launch loops src/1D/1d_main.cu:164-177,
 *                         src/2D/2d_main.cu:150-170, src/3D/3d_main.cu:147-170 around
 *                         rfft_pfa_stencil_8_nwarp / rfft_2d_8_nwarp / rfft_3d_8_nwarp
 *                         (src/1D/rfftstencil_pfa/rfft_8_pfa_fastcomplex.cu:17,
 *                         src/2D/rfft_2d/2d_rfft_1_async.cu:17, src/3D/rfft_3d/3d_rfft_N.cu:17).
 *                         Inputs are natural row-major device buffers (no host re-tiling,
 *                         cf. src/2D/2d_main.cu:96-112) and T means T true time steps.
 *   ffs_plan_destroy   <- the (commented-out) frees of src/1D/create_fft_pfa_plan.cu:217-227.
 *   ffs_shape_lookup   <- the shape tables src/1D/1d_main.cu:45-65,187-193,
 *                         src/2D/2d_main.cu:179-183, src/3D/3d_main.cu:179-183.
 *   ffs_last_error_string <- checkCudaErrors' exit(EXIT_FAILURE)
 *                         (src/1D/helper_cuda/helper_cuda.h:169-182); nothing here exits.
 *   ffs_batch_*        <- no counterpart: many problems in one CUDA graph (FP64-DMMA plans in
 *                         one persistent kernel, the other forms' launches on parallel branches).
 *
 * Conventions: every call returns an ffs_status and never exits or aborts.
 * Plans are immutable after creation and any thread may execute them; the
 * executions of one plan share its workspace, so each waits on the device for
 * the previous one (whatever stream it ran on) -- use one plan per stream to run
 * problems concurrently.  Grids are FP64, row-major with x fastest:
 *   idx = (z * ny + y) * nx + x.
 * Weights are a dense (2r+1)^dim FP64 array with dx fastest
 *   w[((dz + r) * K + (dy + r)) * K + (dx + r)],  K = 2r + 1,
 * applied as a centred correlation: out[i] = sum_d w[d] * in[i + d].
 */
#ifndef FFS_H
#define FFS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFS_ABI_VERSION 4

typedef enum {
    FFS_OK = 0,
    FFS_ERR_INVALID_ARGUMENT = 1,
    FFS_ERR_UNSUPPORTED = 2,
    FFS_ERR_CUDA = 3,
    FFS_ERR_OUT_OF_MEMORY = 4,
    FFS_ERR_TIMEOUT = 5,
    FFS_ERR_INTERNAL = 6
} ffs_status;

typedef enum {
    FFS_BOUNDARY_PERIODIC = 0, /* reference semantics (src/2D/check_correct.hpp:53-61) */
    FFS_BOUNDARY_FIXED = 1     /* ring/shell of width r held at its initial value */
} ffs_boundary;

typedef enum {
    FFS_FORM_AUTO = 0,      /* fastest FP64-exact form (FP64_FFT) */
    FFS_FORM_FP64_DMMA = 1, /* FP64 mma.sync m8n8k4 DFT GEMMs */
    FFS_FORM_OZAKI_I8 = 2,  /* Ozaki split products on INT8 tcgen05/TMEM */
    FFS_FORM_BF16X3 = 3,    /* 3-way BF16 split, FP32 accumulate (~1e-7 work) */
    FFS_FORM_FP64_FFT = 4   /* FP64 butterflies on the FP64 pipe (every dimension) */
} ffs_form;

typedef enum {
    FFS_SHAPE_CUSTOM = 0,
    FFS_SHAPE_HEAT_1D = 1,
    FFS_SHAPE_1D5P = 2,
    FFS_SHAPE_1D7P = 3,
    FFS_SHAPE_HEAT_2D = 4,
    FFS_SHAPE_BOX2D9P = 5,
    FFS_SHAPE_STAR2D9P = 6,
    FFS_SHAPE_BOX2D25P = 7,
    FFS_SHAPE_HEAT_3D = 8,
    FFS_SHAPE_BOX3D27P = 9
} ffs_shape;

typedef struct {
    int dim;               /* 1, 2 or 3 */
    ffs_shape shape;       /* named shape, or FFS_SHAPE_CUSTOM */
    int radius;            /* stencil radius r; only read for FFS_SHAPE_CUSTOM */
    int64_t extents[3];    /* {nx, ny, nz}; unused dims must be 1 */
    const double *weights; /* dense (2r+1)^dim, host memory; NULL = shape default */
    int T;                 /* time steps, >= 0 */
    ffs_boundary boundary;
    ffs_form form;
    int slices;            /* Ozaki INT8 slice count (0 = auto); 2..3 for BF16X3 */
    int tau;               /* fused steps per pass (0 = autotuned) */
    int open_faces;        /* bit 2d / 2d+1: the low / high face of axis d is a cut through a
                              larger grid (domain decomposition), not a boundary: no boundary
                              handling there, and cells within r*T of it are not meaningful
                              (the caller supplies ghost cells and discards them); 0 = none */
    int tile;              /* DFT tile edge: 0 = the plan builder's choice (the autotuner's
                              measured one for the problem class when it has timed both, else
                              its cost model); the FP64 butterfly form takes 64 (a pair of real
                              tiles per CTA) or 128 (one real tile per CTA) in 2D and 16 (one CTA
                              per tile pair) or 32 (a four-CTA cluster per pair) in 3D; every other
                              form has one edge (1D 4096, 2D 64, 3D 16) and accepts only that */
    int reserved[6];       /* must be zero */
} ffs_problem;

typedef struct {
    int dim;
    int radius;
    ffs_form form;       /* resolved form */
    int tile;            /* DFT tile edge n (per dim) */
    int halo;            /* halo per side, >= r * tau, even */
    int useful;          /* cropped output edge u = n - 2 * halo */
    int tau;             /* fused steps per full pass */
    int tau_last;        /* fused steps in the last pass */
    int passes;          /* number of passes (ceil(T / tau)) */
    int slices;          /* resolved slice count (Ozaki / BF16 forms) */
    int64_t tiles;       /* tiles per pass */
    int64_t work_bytes;  /* device workspace owned by the plan */
    double flops_per_pass;   /* algorithmic DFT-GEMM flops per pass (dense count) */
    double exec_flops_per_pass; /* flops the chosen factorisation executes per pass */
    double hbm_bytes_per_pass;  /* algorithmic HBM bytes per pass (16 B per cell) */
    int host_slabs;      /* slabs per grid of ffs_execute_host (1 = whole grid; FFS_HOST_SLABS
                            forces a count) */
    double model_ms;     /* the plan builder's cost-model estimate of one ffs_execute on a
                            148-SM B200 (all passes; the model that ranks fused step counts) */
} ffs_plan_info;

typedef struct {
    double tile_ms;        /* summed device time of the fused tile kernel launches */
    int64_t tile_launches;
    double band_ms;        /* summed device time of the fixed-boundary band launches */
    int64_t band_launches;
} ffs_profile;

typedef struct ffs_plan ffs_plan;
typedef struct ffs_batch ffs_batch;

/* Build a plan: spectra (FP64 direct DFT, raised to tau by repeated squaring),
 * DFT/twiddle tables and tile geometry; allocates the plan's device memory on
 * the current device.  Replaces CreatePlan (src/2D/create_fft_pfa_plan.cu:17). */
ffs_status ffs_plan_create(ffs_plan **out, const ffs_problem *problem);

/* Run T steps: d_out = S^T(d_in).  Asynchronous on `stream` (a cudaStream_t,
 * NULL = legacy default stream).  d_in is never written; d_in == d_out is
 * allowed.  Replaces the launch loop of src/2D/2d_main.cu:150-170.  Launches are
 * checked through the CUDA runtime's per-thread last error, which this call
 * (like ffs_batch_execute and ffs_execute_noalloc) clears first, so a failure an
 * earlier call already returned is not reported as a launch failure.  A call
 * that repeats the process's previous ffs_execute call (same plan, same buffers)
 * replays a CUDA graph of the pass sequence, captured on a private stream at the
 * first repeat (not while the plan is traced, nor inside a caller's stream
 * capture); the plan keeps the graphs of up to four buffer pairs. */
ffs_status ffs_execute(const ffs_plan *plan, const double *d_in, double *d_out, void *stream);

/* Same as ffs_execute with host buffers: copies in, runs, copies out and
 * synchronises `stream` (the CLI's and the end-to-end benchmark's path). */
ffs_status ffs_execute_host(const ffs_plan *plan, const double *h_in, double *h_out, void *stream);

/* `count` independent grids through the same plan, host buffers in and out
 * (an ensemble of runs; the reference solves one grid per process,
 * src/2D/2d_main.cu:135-187).  Grid i's copy-in, compute and copy-out are
 * pipelined against grids i-1 and i+1 on two device slots, so with pinned host
 * buffers the copy-out of one grid overlaps the copy-in of the next.  Returns
 * after every h_out[i] is written; `stream` orders the start after its prior
 * work and carries the compute. */
ffs_status ffs_execute_host_many(const ffs_plan *plan, int count, const double *const *h_in,
                                 double *const *h_out, void *stream);

ffs_status ffs_plan_get_info(const ffs_plan *plan, ffs_plan_info *info);

/* Plan geometry (form, tile, tau, passes, tiles) without touching the GPU;
 * validates `problem` exactly as ffs_plan_create does. */
ffs_status ffs_plan_describe(const ffs_problem *problem, ffs_plan_info *info);
ffs_status ffs_plan_destroy(ffs_plan *plan);

/* Measured autotuning (no counterpart in the reference, whose fused sizes are
 * compile-time constants, src/1D/1d_main.cu:45-65).  It ranks the fused step
 * counts with the plan builder's cost model, times the best `candidates`
 * (0 = 6) on the current device with scratch grids and keeps the fastest; for
 * the FP64 butterfly form in 2D and 3D with problem->tile == 0 it does so for
 * both tile edges (64 and 128, 16 and 32) and keeps the faster edge as well.  For
 * an Ozaki problem with slices == 0 it then calibrates the slice count at that
 * step count: it solves a seeded uniform [0, 1) grid of the problem's geometry
 * with the FP64 butterfly form and with 4 .. 8 slices, and keeps the smallest
 * count whose max relative difference is at most 1e-12 / 1.5 (8 if none is).
 * The choices go into the process-wide tuning table -- also appended to the
 * file named by FFS_TUNE_CACHE, read back on first use -- keyed by problem class
 * (form, slice count, tile edge, dim, taps, boundary, T, log2 extents);
 * ffs_plan_create consults it when problem->tau == 0 (fused steps), when
 * problem->tile == 0 (tile edge) and, for the Ozaki form, when
 * problem->slices == 0 (slice count; 7 when the class was never calibrated). */
ffs_status ffs_autotune(const ffs_problem *problem, int candidates, int *best_tau, double *best_ms, void *stream);

/* Tracing aid: with profiling enabled, every kernel launch of ffs_execute on
 * this plan is bracketed by CUDA events on the execute stream; read sums them
 * (synchronising on the last event) and optionally resets.  Not thread-safe.
 * The slab sub-plans of ffs_execute_host are not traced. */
ffs_status ffs_plan_profile(ffs_plan *plan, int enable);
ffs_status ffs_plan_profile_read(ffs_plan *plan, ffs_profile *out, int reset);

/* Shape table: dim, radius, label ("box_2d1r" ...) and default weights
 * ((2r+1)^dim doubles; pass NULL to query the size only).  Names accepted:
 * Heat-1D 1D5P 1D7P Heat-2D Box2D9P Star2D9P Box2D25P Heat-3D Box3D27P. */
ffs_status ffs_shape_lookup(const char *name, ffs_shape *shape, int *dim, int *radius,
                            const char **label, double *weights, int weights_len);

/* Batched execution: many independent plans (mixed dims, sizes, shapes,
 * boundaries and T).  Every FP64 plan's passes go into ONE persistent kernel
 * launch (a level-ordered work queue of tile pairs and band boxes with
 * per-pass dependency counters); plans of the tensor-core forms run after it
 * with their own kernels.  The launch sequence is captured in a CUDA graph on
 * the first execute and replayed while the buffer pointers match.  A batch uses
 * its plans' workspaces: do not run one of its plans on its own while the batch
 * may still be running. */
ffs_status ffs_batch_create(ffs_batch **out, ffs_plan *const *plans, int count);
ffs_status ffs_batch_execute(ffs_batch *batch, const double *const *d_ins, double *const *d_outs,
                             void *stream);
ffs_status ffs_batch_destroy(ffs_batch *batch);
/* Device status word of the batch's last run after a synchronise (0 = ok,
 * non-zero = a bounded device wait gave up, and the call returns
 * FFS_ERR_TIMEOUT).  Each run starts with a clear word.  A batch item waits at
 * most 2^24 polls (about 2 s) for its problem's previous pass; the environment
 * variable FFS_BATCH_WAIT_POLLS, read by ffs_batch_create, lowers that bound
 * (a diagnostic for exercising the timeout path). */
ffs_status ffs_batch_status(ffs_batch *batch, int *device_status);

/* No counterpart in the reference.  The 2-D FP64 solve for callers that may
 * not allocate device memory (a framework that owns every device allocation
 * through its own pool, a loop that must not block on the allocator), on the
 * FP64-DMMA form (FFS_FORM_AUTO means that form here; the others are
 * unsupported): no cudaMalloc, cudaFree or allocating library call.  Spectra,
 * tables and the ping-pong workspace live in static __device__ arrays of the
 * library, which limit the grid to 1,048,576 cells (8 MiB of scratch held on
 * every GPU that loads the library) and the radius to 4; larger problems get
 * FFS_ERR_UNSUPPORTED.  The per-call constants reach those arrays as kernel
 * parameters, so the call issues no host-to-device copy and returns without
 * waiting for the stream.  The first call on a device resolves the arrays'
 * addresses (make it before any stream capture).  All calls share the arrays:
 * calls that overlap on the GPU race.  Asynchronous on `stream`; a device-side
 * wait that gives up is recorded in the shared status word, which each call
 * clears and ffs_noalloc_status reads back. */
ffs_status ffs_execute_noalloc(const ffs_problem *problem, const double *d_in, double *d_out, void *stream);

/* The shared status word of ffs_execute_noalloc on the current device, after a
 * device synchronise (0 = ok, non-zero = a bounded device wait of the last call
 * gave up and its output is not valid).  Synchronous; allocates nothing. */
ffs_status ffs_noalloc_status(int *device_status);

/* Message of the last failing call on this thread ("" if none). */
const char *ffs_last_error_string(void);
int ffs_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FFS_H */
