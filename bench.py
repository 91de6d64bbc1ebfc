#!/usr/bin/env python
"""Benchmark of the fused DFT-tile stencil path on B200.

Workload (default): Box2D9P on a 4096 x 4096 FP64 grid, uniform[0,1) inputs and
3x3 weights uniform(0,1) normalised to sum 1 (both from a seeded mt19937-style
generator), fixed boundary ring of width 1, T = 32 true time steps.  One bench
"step" is one full T-step solve (ffs_execute).  Metric: GStencil/s =
interior cells x T / s / 1e9, at <= 1e-12 max relative error against the FP64
oracle (checked in the same run).  The headline form is fp64_fft (radix-8
butterflies on the FP64 pipe, the fastest FP64-exact form on B200); FP64-DMMA,
Ozaki INT8 and 3-way BF16 are measured beside it under "forms".

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--form fp64_fft|fp64|ozaki|bf16x3]

With N > 1 (torchrun, one rank per GPU) every rank solves its own grid
(replicas: the grids are independent, no collective on the data path), the
timed region is bracketed by barriers and the max time over ranks is used.
`--impl reference` times the reference's own CPU stencil (stencil2D from
src/2D/check_correct.hpp, built into oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20251203 + 1
# name -> (shape, dims (x fastest), T, boundary, input range, weights kind, seed offset) (the benchmark configurations)
WORKLOADS = {
    "box2d9p": ("Box2D9P", (4096, 4096), 32, "fixed", (0.0, 1.0), "uniform", 1),
    "heat1d": ("Heat-1D", (1 << 20,), 64, "fixed", (0.0, 1.0), "default", 0),
    "box3d27p": ("Box3D27P", (512, 512, 512), 16, "fixed", (0.0, 1.0), "uniform", 2),
    "box2d25p": ("Box2D25P", (8192, 8192), 128, "periodic", (-1.0, 1.0), "normal_rho1", 3),
    "box2d9p_8192": ("Box2D9P", (8192, 8192), 32, "fixed", (0.0, 1.0), "uniform", 1),
    "box3d27p_256": ("Box3D27P", (256, 256, 256), 16, "fixed", (0.0, 1.0), "uniform", 2),  # profiling size
}
WORKLOAD = dict(shape="Box2D9P", n=4096, T=32, boundary="fixed")
METRIC = "GStencil/s (cells x steps / s) at <=1e-12 max rel err vs FP64 oracle"
UNIT = "GStencil/s"


def seeded_inputs(n, r, seed):
    rng = np.random.Generator(np.random.MT19937(seed))
    x = rng.random((n, n))
    w = rng.random((2 * r + 1, 2 * r + 1))
    w /= w.sum()
    return x, w


def workload_inputs(name, seed_base):
    """Seeded grid and weights of a named workload (mt19937; input drawn first, then weights)."""
    shape, ext, T, bnd, (lo, hi), wkind, off = WORKLOADS[name]
    import flashfftstencil_b200 as ffs
    si = ffs.shape_info(shape)
    rng = np.random.Generator(np.random.MT19937(seed_base + off))
    x = lo + (hi - lo) * rng.random(tuple(reversed(ext)))
    if wkind == "default":
        w = si.weights.copy()
    elif wkind == "uniform":
        w = rng.random(si.weights.shape) * (si.weights != 0)
        w /= w.sum()
    else:  # N(0,1) taps scaled so that max |S(w)| over the grid's periodic frequencies is 1
        K = 2 * si.radius + 1
        w = rng.standard_normal((K,) * si.dim)
        ker = np.zeros(tuple(reversed(ext)))
        for idx in np.ndindex(*w.shape):
            ker[tuple((-(i - si.radius)) % n for i, n in zip(idx, ker.shape))] += w[idx]
        w = (w / np.abs(np.fft.fftn(ker)).max()).ravel()
    return si, x, np.asarray(w, dtype=np.float64).ravel(), T, bnd


# Reference GPU programs and the only arguments they are run with: each was checked by reading
# for in-bounds loads and stores (complete tile pairs; 1D7P is excluded, its last block writes
# past the output).  The 3D program allocates ~15 GB of host memory and only runs with room.
REFERENCE_GPU_RUNS = [
    ("ref_1d.out", ["Heat-1D", "1048572", "64"], ("Heat-1D", (1048572,), 64)),
    ("ref_2d.out", ["Box2D9P", "4104", "32"], ("Box2D9P", (4104, 4104), 32)),
    ("ref_2d.out", ["Box2D9P", "8196", "32"], ("Box2D9P", (8196, 8196), 32)),
    ("ref_3d.out", ["Box3D27P", "768", "16"], ("Box3D27P", (768, 768, 768), 16)),
]


def run_reference_gpu(args):
    """Context: the reference's own GPU programs (oracle/_ref/ref_{1,2,3}d.out, built from its
    unmodified mains for sm_100a) beside this solver on the same sizes.  The reference launches one
    fused kernel per time step (14 steps per launch in 1D) on a re-used, host-re-tiled input with a
    periodic wrap and random weights; its output is not parity-checked, so only throughput is
    compared, with its own GStencil/s formula (src/2D/2d_main.cu:185, src/1D/1d_main.cu:195)."""
    import torch
    import flashfftstencil_b200 as ffs
    torch.cuda.set_device(0)
    out = {"metric": "GStencil/s (each program's own count), periodic wrap", "runs": []}
    try:
        free_gb = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE") / 1e9
    except (ValueError, OSError):
        free_gb = 0.0
    for exe, argv, (shape, ext, T) in REFERENCE_GPU_RUNS:
        row = {"program": exe, "args": argv}
        path = os.path.join(ROOT, "oracle", "_ref", exe)
        if not os.path.exists(path):
            row["reference"] = "not built (make -C oracle refgpu where the reference sources exist)"
        elif exe == "ref_3d.out" and free_gb < 48:
            row["reference"] = f"skipped: {free_gb:.0f} GB host memory available, the program needs ~15 GB"
        else:
            try:
                r = subprocess.run([path] + argv, capture_output=True, text=True, timeout=600)
                line = [ln for ln in r.stdout.splitlines() if ln.startswith("FlashFFTStencil")]
                if r.returncode == 0 and line:
                    f = [t.strip() for t in line[-1].split(",")]
                    row["reference"] = {"ms": float(f[-2]), "gstencil_s": float(f[-1]), "line": line[-1]}
                else:
                    row["reference"] = f"exit {r.returncode}: {(r.stderr or r.stdout)[-300:]}"
            except subprocess.TimeoutExpired:
                row["reference"] = "timed out"
        si = ffs.shape_info(shape)
        plan = ffs.Plan(si.dim, shape, ext, T, boundary="periodic", form="auto")  # fastest FP64-exact form
        x = torch.rand(tuple(reversed(ext)), dtype=torch.float64, device="cuda",
                       generator=torch.Generator("cuda").manual_seed(2))
        y = torch.empty_like(x)
        for _ in range(3):
            plan.run(x, y)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 20
        e0.record()
        for _ in range(reps):
            plan.run(x, y)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        row["ours"] = {"shape": shape, "extents": ext, "T": T, "boundary": "periodic", "ms": ms,
                       "gstencil_s": float(np.prod(ext)) * T / (ms * 1e-3) / 1e9, "plan": plan.info}
        plan.close()
        if isinstance(row.get("reference"), dict):
            row["speedup"] = row["ours"]["gstencil_s"] / row["reference"]["gstencil_s"]
        out["runs"].append(row)
        print(json.dumps(row), file=sys.stderr, flush=True)
    print(json.dumps(out), flush=True)
    return 0


COMPETITOR_CASES = (("Box2D9P", (8192, 8192), 32), ("Box3D27P", (512, 512, 512), 16))


def measure_competitors(cases=COMPETITOR_CASES, reps=5):
    """Context, not the product: library (cuFFT / cuDNN through torch) ways to advance the same
    periodic grids by T steps, next to the fused tile path.  Mirrors the reference's comparison
    scripts (benchmarks/cufft-by-pytorch/rfft2D.py: one full-domain rfft2 / multiply / irfft2 per
    step; benchmarks/cudnn/cudnn-test.cpp: direct FP64 convolution).  Each library result is
    compared with the fused tile path's."""
    import torch
    import flashfftstencil_b200 as ffs
    from tests.helpers import rel_errors
    out = {"metric": "GStencil/s, periodic boundary (library baselines for context)", "cases": []}
    for shape, ext, T in cases:
        si = ffs.shape_info(shape)
        rng = np.random.Generator(np.random.MT19937(SEED + 9))
        w = rng.random(si.weights.shape)
        w /= w.sum()
        dims = tuple(reversed(ext))
        x = torch.rand(dims, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
        K = 2 * si.radius + 1
        wk = torch.from_numpy(w.reshape((K,) * si.dim)).cuda()
        ker = torch.zeros(dims, dtype=torch.float64, device="cuda")
        for idx in np.ndindex(*wk.shape):  # correlation taps placed at -d (periodic)
            ker[tuple((-(i - si.radius)) % n for i, n in zip(idx, dims))] += wk[idx]
        axes = tuple(range(-si.dim, 0))
        S = torch.fft.rfftn(ker, dim=axes)
        cells = float(np.prod(ext)) * T
        ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

        def timed(fn, n):
            fn()
            torch.cuda.synchronize()
            e0, e1 = ev(), ev()
            e0.record()
            for _ in range(n):
                fn()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / n

        # ours
        plan = ffs.Plan(si.dim, None, ext, T, weights=w, radius=si.radius, boundary="periodic", form="auto")
        y_ours = plan.run(x)
        ms_ours = timed(lambda: plan.run(x, y_ours), reps)
        # cuFFT, S^T in one round trip (periodic only; independent of T)
        ST = S ** T
        f_pow = lambda: torch.fft.irfftn(torch.fft.rfftn(x, dim=axes) * ST, s=dims, dim=axes)  # noqa: E731
        y_fft = f_pow()
        ms_pow = timed(f_pow, reps)
        # cuFFT, one round trip per time step (the reference's script, timed per step)
        f_step = lambda: torch.fft.irfftn(torch.fft.rfftn(x, dim=axes) * S, s=dims, dim=axes)  # noqa: E731
        ms_step = timed(f_step, 3) * T
        # cuDNN direct FP64 convolution, T launches (circular padding)
        import torch.nn.functional as F
        conv = F.conv2d if si.dim == 2 else F.conv3d
        wc = wk.reshape((1, 1) + (K,) * si.dim)

        def f_conv():
            y = x.reshape((1, 1) + dims)
            for _ in range(T):
                y = conv(F.pad(y, (si.radius,) * (2 * si.dim), mode="circular"), wc)
            return y

        y_conv = f_conv().reshape(dims)
        ms_conv = timed(f_conv, 1)
        ours = y_ours.cpu().numpy()
        out["cases"].append({"shape": shape, "extents": ext, "T": T,
                             "fused_tile_fp64": cells / (ms_ours * 1e-3) / 1e9,
                             "cufft_spectrum_power": cells / (ms_pow * 1e-3) / 1e9,
                             "cufft_per_step": cells / (ms_step * 1e-3) / 1e9,
                             "cudnn_direct_fp64": cells / (ms_conv * 1e-3) / 1e9,
                             "fused_vs_cufft_power_max_rel_diff": rel_errors(ours, y_fft.cpu().numpy())[0],
                             "fused_vs_cudnn_max_rel_diff": rel_errors(ours, y_conv.cpu().numpy())[0]})
        plan.close()
        del ker, S, ST, y_fft, y_conv
        torch.cuda.empty_cache()
    return out


def run_competitors(args):
    import torch
    torch.cuda.set_device(0)
    print(json.dumps(measure_competitors()), flush=True)
    return 0


def run_host_slabs(args):
    """Host-buffer calls (pinned memory, copies inside the timed region) by slab count:
    ffs_execute_host on one grid and ffs_execute_host_many on --steps grids, with
    FFS_HOST_SLABS forcing 1 (whole grid), 2, 4, 8, 16 slabs and unset (the plan's model).
    Box2D9P 4096^2 fixed T=32 and Box3D27P 512^3 fixed T=16, butterfly form."""
    import torch
    import flashfftstencil_b200 as ffs
    torch.cuda.set_device(0)
    out = {"metric": "GStencil/s end to end with host buffers, by host slab count", "cases": []}
    # the link itself: pinned copies of one 4096^2 FP64 grid (134 MB), each direction alone and
    # both at once, the copy split over 1 or 2 streams per direction (wall clock, 10 repetitions)
    n = 4096 * 4096
    h_in, h_out = torch.rand(n, dtype=torch.float64).pin_memory(), torch.empty(n, dtype=torch.float64).pin_memory()
    d_in, d_out = torch.empty(n, dtype=torch.float64, device="cuda"), torch.rand(n, dtype=torch.float64, device="cuda")
    cs = [torch.cuda.Stream() for _ in range(4)]
    link = {}
    for mode in ["h2d", "d2h", "both"]:
        for parts in [1, 2]:
            k = n // parts
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(10):
                for i in range(parts):
                    if mode != "d2h":
                        with torch.cuda.stream(cs[i]):
                            d_in[i * k:(i + 1) * k].copy_(h_in[i * k:(i + 1) * k], non_blocking=True)
                    if mode != "h2d":
                        with torch.cuda.stream(cs[2 + i]):
                            h_out[i * k:(i + 1) * k].copy_(d_out[i * k:(i + 1) * k], non_blocking=True)
                torch.cuda.synchronize()
            link[f"{mode}_{parts}_streams_gbs_per_direction"] = n * 8 * 10 / (time.perf_counter() - t0) / 1e9
    out["link"] = link
    del h_in, h_out, d_in, d_out
    for shape, ext, T in [("Box2D9P", (4096, 4096), 32), ("Box3D27P", (512, 512, 512), 16)]:
        dim = len(ext)
        dims = tuple(reversed(ext))
        cells = float(np.prod(ext)) * T
        rng = np.random.Generator(np.random.MT19937(SEED))
        x = torch.from_numpy(rng.random(dims)).pin_memory()
        y = torch.empty_like(x).pin_memory()
        many = max(2, min(args.steps, 20 if dim == 2 else 4))
        case = {"shape": shape, "extents": list(ext), "T": T, "grids_many": many, "by_slabs": []}
        ref = None
        for k in ["1", "2", "4", "8", "16", None]:
            if k is None:
                os.environ.pop("FFS_HOST_SLABS", None)
            else:
                os.environ["FFS_HOST_SLABS"] = k
            plan = ffs.Plan(dim, shape, ext, T, boundary="fixed", form="fp64_fft")
            plan.run_host(x.numpy(), y.numpy())  # warm-up: sub-plans, buffers
            if ref is None:
                ref = y.numpy().copy()
            err = float(np.abs(y.numpy() - ref).max() / np.abs(ref).max())
            reps = 5 if dim == 2 else 2
            t0 = time.perf_counter()
            for _ in range(reps):
                plan.run_host(x.numpy(), y.numpy())
            single = (time.perf_counter() - t0) / reps * 1e3
            xs, ys = [x.numpy()] * many, [y.numpy()] * many
            plan.run_host_many(xs, ys)  # warm-up with the same count: the same pipeline and buffers
            t0 = time.perf_counter()
            plan.run_host_many(xs, ys)
            per_grid = (time.perf_counter() - t0) / many * 1e3
            case["by_slabs"].append({"FFS_HOST_SLABS": k, "host_slabs": plan.info["host_slabs"],
                                     "single_ms": single, "single_gstencil_s": cells / (single * 1e-3) / 1e9,
                                     "many_ms_per_grid": per_grid,
                                     "many_gstencil_s": cells / (per_grid * 1e-3) / 1e9,
                                     "max_rel_diff_vs_whole_grid": err})
            plan.close()
        os.environ.pop("FFS_HOST_SLABS", None)
        out["cases"].append(case)
    print(json.dumps(out), flush=True)
    return 0


def run_named_workload(args):
    """A named benchmark configuration on one GPU: each available form, accuracy vs the oracle."""
    import torch
    import flashfftstencil_b200 as ffs
    from tests.helpers import rel_errors
    torch.cuda.set_device(0)
    si, x_np, w, T, bnd = workload_inputs(args.workload, 20251203)
    ext = tuple(reversed(x_np.shape))
    if args.kernel_only:
        plan = ffs.Plan(si.dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form=args.form,
                        slices=FORMS[args.form][1], tile=args.tile)
        d_in = torch.from_numpy(x_np).cuda()
        d_out = torch.empty_like(d_in)
        for _ in range(args.warmup + args.steps):
            plan.run(d_in, d_out)
        torch.cuda.synchronize()
        plan.close()
        return 0
    forms = ["fp64", "fp64_fft"] if si.dim == 1 else ["fp64", "fp64_fft", "ozaki", "bf16x3"]
    ref, cpu_s = None, None
    if not args.no_cpu:
        import oracle
        t0 = time.perf_counter()
        ref = oracle.run(x_np, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
        cpu_s = time.perf_counter() - t0
    d_in = torch.from_numpy(x_np).cuda()
    cells = float(np.prod(ext)) * T
    out = {"workload": args.workload, "shape": si.name, "extents": ext, "T": T, "boundary": bnd,
           "cpu_oracle_s": cpu_s, "forms": {}}
    stream = torch.cuda.current_stream()
    tuned = {}
    for form in forms:
        # the measured autotuner (ffs_autotune) picks the fused step count for this problem;
        # the plan then takes it from the tuning table (tau = 0)
        tuned[form] = ffs.autotune(si.dim, None, ext, T, candidates=6, weights=w, radius=si.radius, boundary=bnd,
                                   form=form, slices=FORMS[form][1])[0]
        plan = ffs.Plan(si.dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form=form,
                        slices=FORMS[form][1])
        d_out = plan.run(d_in)
        torch.cuda.synchronize()
        acc = rel_errors(d_out.cpu().numpy(), ref) if ref is not None else None
        for _ in range(3):
            plan.run(d_in, d_out)

        def timed(steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                plan.run(d_in, d_out)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / steps

        # solve rate without per-launch events; launch durations from a shorter run with them
        ms = timed(args.steps)
        plan.profile(True)
        plan.profile_read(reset=True)
        timed(max(args.steps // 5, 3))
        prof = plan.profile_read(reset=True)
        plan.profile(False)
        out["forms"][FORMS[form][0]] = {
            "gstencil_s": cells / (ms * 1e-3) / 1e9, "ms_per_solve": ms, "info": plan.info,
            "autotuned_tau": tuned[form],
            "max_rel_err": acc[0] if acc else None, "l2_rel_err": acc[1] if acc else None,
            "tile_ms_per_launch": prof["tile_ms"] / max(prof["tile_launches"], 1),
            "band_ms_per_launch": prof["band_ms"] / max(prof["band_launches"], 1)}
        plan.close()
    if si.dim >= 2 and args.sweep:  # Ozaki slice-count sweep: error and speed per slice count
        out["ozaki_sweep"] = {}
        for sl in range(4, 9):
            plan = ffs.Plan(si.dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form="ozaki",
                            slices=sl)
            d_out = plan.run(d_in)
            torch.cuda.synchronize()
            acc = rel_errors(d_out.cpu().numpy(), ref) if ref is not None else (None, None)
            for _ in range(2):
                plan.run(d_in, d_out)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(max(args.steps // 2, 1)):
                plan.run(d_in, d_out)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / max(args.steps // 2, 1)
            out["ozaki_sweep"][sl] = {"gstencil_s": cells / (ms * 1e-3) / 1e9, "max_rel_err": acc[0],
                                      "l2_rel_err": acc[1]}
            plan.close()
    if si.dim >= 2 and args.sweep and not args.no_cpu:
        # 3xBF16 error against the number of fused passes at a fixed step count per pass: the
        # error each pass of four (2-D) or six (3-D) GEMM stages adds
        import oracle
        tau = tuned["bf16x3"]
        mode = oracle.FIXED if bnd == "fixed" else oracle.PERIODIC
        out["bf16x3_by_passes"] = {}
        for npass in range(1, 5):
            Tp = min(T, npass * tau)
            plan = ffs.Plan(si.dim, None, ext, Tp, weights=w, radius=si.radius, boundary=bnd, form="bf16x3",
                            slices=3, tau=tau)
            y = plan.run(d_in)
            torch.cuda.synchronize()
            acc = rel_errors(y.cpu().numpy(), oracle.run(x_np, w, si.radius, Tp, mode))
            out["bf16x3_by_passes"][npass] = {"T": Tp, "passes": plan.info["passes"], "max_rel_err": acc[0],
                                              "l2_rel_err": acc[1]}
            plan.close()
            if Tp == T:
                break
    if cpu_s:
        out["cpu_oracle_gstencil_s"] = cells / cpu_s / 1e9
    print(json.dumps(out), flush=True)
    return 0


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"ffs_bench_clocks_{os.getpid()}_rank{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [s.strip() for s in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        under = [s for s in sm if mx and s > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(under) if under else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


TRAFFIC_FILES = {("fp64", 64): "dmma2d_box2d9p_4096_traffic.json", ("fp64_fft", 64): "fft2d_box2d9p_4096_traffic.json",
                 ("fp64_fft", 128): "fft2d128_box2d9p_4096_traffic.json"}


def fft2d_smem_bytes_per_pair(useful):
    """Shared-memory bytes the butterfly kernel moves per tile pair, from its design: per thread of
    the 512, pass A reads 8 staged points of both tiles (128 B) and moves 8 complex values three
    times (transpose out, transpose in, row out: 384 B); pass B loads 8, passes two transposes,
    reads 8 spectrum values and stores 8 (896 B); pass C (8 threads per wanted row) loads 8 and
    passes one transpose (384 B); the TMA writes the two 32 KiB staged tiles."""
    return 512 * (128 + 384) + 512 * 896 + 8 * useful * 384 + 2 * 64 * 64 * 8


def fft2d128_smem_bytes_per_tile(useful):
    """Shared-memory bytes the 128 x 128 butterfly kernel moves per tile, from its design (16-byte
    accesses): pass A, per thread of the 512, an exchange put and get and the row's output write
    (48 accesses); pass B, per thread, the two-load gather of 16 points, two exchanges and the
    scatter (112); pass C, 8 threads for each of the u/2 wanted row pairs, the two-load gather and
    one exchange (64); and the twiddle-table reads, 15 per thread and line transform
    (64 + 128 + u/2 line transforms)."""
    lines = 64 + 128 + useful // 2
    return 16 * (512 * 48 + 512 * 112 + 8 * (useful // 2) * 64 + 8 * lines * 15)


def read_traffic(form, tile=64):
    if (form, tile) not in TRAFFIC_FILES:
        return None
    path = os.path.join(ROOT, "profiles", TRAFFIC_FILES[(form, tile)])
    try:
        return json.load(open(path))
    except Exception:
        return None


def cpu_oracle_baseline(x, w, T, steps_cap=None):
    """FP64 oracle (OpenMP over all host threads) on the workload; returns result and timing."""
    import oracle
    t0 = time.perf_counter()
    ref = oracle.run(x, w, 1, T, oracle.FIXED)
    dt = time.perf_counter() - t0
    return ref, dt, oracle.max_threads()


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    import oracle
    n = WORKLOAD["n"]
    x, w = seeded_inputs(n, 1, SEED)
    if oracle.ref_lib() is not None:
        kind = "reference"
        fn = lambda a: oracle.ref_stencil2d(a, w)  # noqa: E731
        what = "reference stencil2D (src/2D/check_correct.hpp:64-100, periodic wrap, OpenMP)"
    else:
        kind = "port"
        fn = lambda a: oracle.run(a, w, 1, 1, oracle.FIXED)  # noqa: E731
        what = "oracle port (direct FP64 stepping, fixed ring, OpenMP)"
    # size each bench step so that the whole timed run stays near a minute
    t0 = time.perf_counter()
    fn(x)
    t_full = time.perf_counter() - t0
    budget = 60.0 / max(args.steps, 1)
    side = n if t_full <= budget else max(64, int(n * (budget / t_full) ** 0.5))
    xs = np.ascontiguousarray(x[:side, :side])
    y = xs
    for _ in range(args.warmup):
        y = fn(y)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        y = fn(y)
    dt = time.perf_counter() - t0
    value = side * side * args.steps / dt / 1e9
    cores = oracle.max_threads()
    sample = (f"{what}: one time step of a {side}x{side} corner of the {n}x{n} grid per bench step "
              f"(full-grid step took {t_full:.3f} s)")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{WORKLOAD['shape']} {n}x{n} FP64, fixed ring width 1, T={WORKLOAD['T']}"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "vs_baseline": None}
    print(json.dumps(line), flush=True)
    return 0


FORMS = {"fp64": ("fp64_dmma", 0), "fp64_fft": ("fp64_fft", 0), "ozaki": ("ozaki_i8", 7), "bf16x3": ("bf16x3", 3)}


def c5_specs(count, seed):
    """The batched mixed workload: 60 % 2D (Heat-2D/Star2D9P/Box2D9P, sides log-uniform
    64-2048), 30 % 1D (1D5P/1D7P, N log-uniform 2^12-2^20), 10 % 3D (Heat-3D/Box3D27P,
    sides log-uniform 32-256); T uniform in 1..64; boundary fixed or periodic at random."""
    rng = np.random.Generator(np.random.MT19937(seed))
    lu = lambda lo, hi: int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))  # noqa: E731
    specs = []
    for _ in range(count):
        u = rng.random()
        if u < 0.6:
            shape, dim, ext = ["Heat-2D", "Star2D9P", "Box2D9P"][int(rng.integers(0, 3))], 2, (lu(64, 2048), lu(64, 2048))
        elif u < 0.9:
            shape, dim, ext = ["1D5P", "1D7P"][int(rng.integers(0, 2))], 1, (lu(2 ** 12, 2 ** 20),)
        else:
            shape, dim, ext = ["Heat-3D", "Box3D27P"][int(rng.integers(0, 2))], 3, (lu(32, 256), lu(32, 256), lu(32, 256))
        T = int(rng.integers(1, 65))
        bnd = "fixed" if rng.random() < 0.5 else "periodic"
        specs.append((shape, dim, ext, T, bnd))
    return specs


def run_batch_workload(args):
    """512 independent problems as one CUDA graph replay (`ffs_batch_*`: the FP64-DMMA plans in one
    persistent kernel, plans of the other forms as their own launches on parallel graph branches)
    vs per-problem launches."""
    import torch
    import flashfftstencil_b200 as ffs
    from tests.helpers import rel_errors
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    specs = c5_specs(args.problems, SEED + 4 + rank)
    # fp64_fft: each problem takes the fastest FP64-exact form (butterflies in 2-D/3-D, whose plans
    # run as captured per-plan launches beside the persistent kernel); fp64: every problem on DMMA
    # in the one persistent kernel
    form = "auto" if args.form == "fp64_fft" else args.form
    rng = np.random.Generator(np.random.MT19937(SEED + 40 + rank))
    plans, ins, outs, cells = [], [], [], 0.0
    for shape, dim, ext, T, bnd in specs:
        si = ffs.shape_info(shape)
        w = rng.random(si.weights.shape) * (si.weights != 0)
        w /= w.sum()
        plans.append(ffs.Plan(dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form=form,
                              slices=FORMS[args.form][1] if dim > 1 else 0))
        x = torch.rand(tuple(reversed(ext)), dtype=torch.float64, device="cuda")
        ins.append(x)
        outs.append(torch.empty_like(x))
        cells += float(np.prod(ext)) * T
    stream = torch.cuda.current_stream()
    batch = ffs.Batch(plans)
    iptr, optr = [t.data_ptr() for t in ins], [t.data_ptr() for t in outs]
    if args.kernel_only:  # warm-up + timed launches only (profiler captures)
        for _ in range(args.warmup + args.steps):
            batch.execute(iptr, optr, stream.cuda_stream)
        torch.cuda.synchronize()
        return 0 if batch.status() == 0 else 1
    # parity of the persistent launch against the per-problem path
    batch.execute(iptr, optr, stream.cuda_stream)
    torch.cuda.synchronize()
    assert batch.status() == 0
    worst = 0.0
    for p, x, o in zip(plans, ins, outs):
        worst = max(worst, rel_errors(o.cpu().numpy(), p.run(x).cpu().numpy())[0])
    for _ in range(max(args.warmup, 3)):
        batch.execute(iptr, optr, stream.cuda_stream)
    torch.cuda.synchronize()
    reps = max(1, args.steps // 50)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        batch.execute(iptr, optr, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_batch = e0.elapsed_time(e1) / reps
    for _ in range(2):
        for p, x, o in zip(plans, ins, outs):
            p.execute(x.data_ptr(), o.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        for p, x, o in zip(plans, ins, outs):
            p.execute(x.data_ptr(), o.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_plain = e0.elapsed_time(e1) / reps
    line = {"metric": f"GStencil/s, {len(specs)}-problem batched mixed workload (one CUDA graph replay)",
            "value": cells / (ms_batch * 1e-3) / 1e9, "unit": UNIT, "n_gpus": 1, "steps": reps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_batch, "higher_is_better": True, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"{len(specs)} problems: 60% 2D (Heat-2D/Star2D9P/Box2D9P, sides log-uniform 64-2048), "
                                   "30% 1D (1D5P/1D7P, N log-uniform 2^12-2^20), 10% 3D (Heat-3D/Box3D27P, sides "
                                   "32-256), T uniform 1..64, boundary fixed/periodic at random",
                       "form": form,
                       "execution": "one CUDA graph per replay: FP64-DMMA plans in one persistent kernel, plans "
                                    "of the other forms as their own launches on 8 parallel graph branches",
                       "cell_steps": cells, "problems": len(specs)},
            "per_problem_launches": {"value": cells / (ms_plain * 1e-3) / 1e9, "ms_per_step": ms_plain},
            "speedup_vs_per_problem": ms_plain / ms_batch,
            "max_rel_err_vs_per_problem": worst}
    print(json.dumps(line), flush=True)
    batch.close()
    return 0


def measure_form(ffs, torch, form, n, T, w, d_in, steps, warmup, ref, clocks=None, barrier=None, tile=0):
    """One form on the workload: accuracy vs the oracle result, then `steps` timed solves."""
    from tests.helpers import rel_errors
    slices = FORMS[form][1]
    plan = ffs.Plan(2, None, (n, n), T, weights=w, radius=1, boundary=WORKLOAD["boundary"], form=form,
                    slices=slices, tile=tile)
    d_out = torch.empty_like(d_in)
    stream = torch.cuda.current_stream()
    plan.run(d_in, d_out)
    torch.cuda.synchronize()
    acc = None
    if ref is not None:
        mx, l2 = rel_errors(d_out.cpu().numpy(), ref)
        acc = {"max_rel_err": mx, "l2_rel_err": l2}
    for _ in range(max(warmup, 3)):
        plan.run(d_in, d_out)
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        time.sleep(0.3)

    def timed_region():
        if barrier:
            barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            plan.run(d_in, d_out)
        e1.record(stream)
        torch.cuda.synchronize()
        if barrier:
            barrier()
        return e0.elapsed_time(e1)

    # the solve rate is timed without per-launch events (recording them around every
    # launch slows a 4096^2 solve by about 6 %); the same K steps then run again with
    # the events on, which give each kernel's average launch duration for the roofline
    ms = timed_region()
    plan.profile(True)
    plan.profile_read(reset=True)
    ms_profiled = timed_region()
    prof = plan.profile_read(reset=True)
    plan.profile(False)
    ck = clocks.stop() if clocks else None
    return plan, {"ms_total": ms, "ms_total_profiled": ms_profiled, "accuracy": acc, "profile": prof,
                  "info": plan.info, "clocks": ck}


# The north-star target configurations (Ozaki-INT8 against FP64-DMMA at <= 1e-12), measured in the
# default run beside the headline: each form's autotuned solve rate and its error against the oracle.
TARGETS = ("box2d9p_8192", "box3d27p")
TARGET_FORMS = (("fp64_fft", 0), ("fp64", 0), ("ozaki", 0), ("ozaki", 6), ("ozaki", 7), ("bf16x3", 3))


def measure_targets(ffs, torch, steps, warmup, with_oracle):
    """Box2D9P 8192^2 T=32 and Box3D27P 512^3 T=16 (fixed boundary, seeded inputs): per form the
    solve rate over `steps` solves (inputs larger than L2), max/L2 error against the oracle, and
    Ozaki-INT8 over FP64-DMMA at each slice count and at the fastest count meeting 1e-12."""
    from tests.helpers import rel_errors
    out = {}
    stream = torch.cuda.current_stream()
    for name in TARGETS:
        si, x_np, w, T, bnd = workload_inputs(name, 20251203)
        ext = tuple(reversed(x_np.shape))
        ref = None
        t_cpu = None
        if with_oracle:
            import oracle
            t0 = time.perf_counter()
            ref = oracle.run(x_np, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
            t_cpu = time.perf_counter() - t0
        d_in = torch.from_numpy(x_np).cuda()
        cells = float(np.prod(ext)) * T
        rec = {"workload": f"{si.name} {'x'.join(map(str, ext))} FP64, {bnd} boundary, T={T}, U[0,1) inputs, "
                           "U(0,1) weights normalised to 1",
               "cpu_oracle_s": t_cpu, "forms": {}}
        for form, sl in TARGET_FORMS:
            # Ozaki with slices 0: the autotuner calibrates the slice count against the FP64 form
            key = FORMS[form][0] + ((f"_s{sl}" if sl else "_auto") if form == "ozaki" else "")
            tau = ffs.autotune(si.dim, None, ext, T, candidates=4, weights=w, radius=si.radius, boundary=bnd,
                               form=form, slices=sl)[0]
            plan = ffs.Plan(si.dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form=form,
                            slices=sl, tau=tau)
            d_out = plan.run(d_in)
            torch.cuda.synchronize()
            acc = rel_errors(d_out.cpu().numpy(), ref) if ref is not None else (None, None)
            for _ in range(max(warmup, 3)):
                plan.run(d_in, d_out)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                plan.run(d_in, d_out)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            rec["forms"][key] = {"value": cells / (ms * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms,
                                 "tau": plan.info["tau"], "passes": plan.info["passes"],
                                 "slices": plan.info["slices"] or None,
                                 "max_rel_err": acc[0], "l2_rel_err": acc[1],
                                 "meets_1e-12": None if acc[0] is None else bool(acc[0] <= 1e-12)}
            plan.close()
            del d_out
        f = rec["forms"]
        base = f["fp64_dmma"]["value"]
        for sl in (6, 7):
            f[f"ozaki_i8_s{sl}_vs_fp64_dmma"] = f[f"ozaki_i8_s{sl}"]["value"] / base
        f["ozaki_i8_auto_vs_fp64_dmma"] = f["ozaki_i8_auto"]["value"] / base
        ok = [f[k]["value"] for k in ("ozaki_i8_auto", "ozaki_i8_s6", "ozaki_i8_s7") if f[k]["meets_1e-12"]]
        rec["ozaki_vs_fp64"] = max(ok) / base if ok else None
        rec["ozaki_vs_fp64_note"] = ("fastest Ozaki-INT8 slice count (calibrated, 6 or 7) meeting 1e-12 against the "
                                     "oracle / FP64-DMMA")
        out[name] = rec
        del d_in
        torch.cuda.empty_cache()
    return out


def measure_decomposed(args, ws, rank, local, dist=None):
    """One headline grid split into slabs over the ws ranks (strong scaling): each rank
    solves its rows with a ghost exchange of r*tau rows per fused pass over NCCL
    (flashfftstencil_b200.slab).  Every rank calls it together; returns the line."""
    import torch
    from flashfftstencil_b200.slab import SlabPlan

    n, T = WORKLOAD["n"], WORKLOAD["T"]
    x_np, w = seeded_inputs(n, 1, SEED)  # the same global grid on every rank
    pl = SlabPlan(2, None, (n, n), T, weights=w, radius=1, boundary=WORKLOAD["boundary"], rank=rank, world=ws,
                  form=args.form)
    x = torch.from_numpy(np.ascontiguousarray(x_np[pl.lo:pl.hi])).cuda()
    bufs = pl.allocate(x)
    for _ in range(max(args.warmup, 3)):
        pl.run(x, bufs=bufs)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        y = pl.run(x, bufs=bufs)
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    err = None
    if not args.no_cpu:
        import oracle
        ref = oracle.run(x_np, w, 1, T, oracle.FIXED)
        err = float(np.abs(y.cpu().numpy() - ref[pl.lo:pl.hi]).max() / np.abs(ref).max())
    if dist:
        t = torch.tensor([ms, err if err is not None else -1.0], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, err = t[0].item(), (t[1].item() if err is not None else None)
        dist.barrier()
    return {"metric": METRIC, "value": float(n) * n * T * args.steps / (ms * 1e-3) / 1e9, "unit": UNIT,
            "n_gpus": ws, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"{WORKLOAD['shape']} {n}x{n} FP64, fixed ring width 1, T={T}, one grid",
                       "parallelism": f"slabs x{ws} along y, ghost exchange of r*tau rows per pass (NCCL)",
                       "form": args.form,
                       "passes": len(pl.passes), "tau": pl.passes[0].tau if pl.passes else 0,
                       "rows_per_rank": pl.rows, "split": bool(pl.passes and pl.passes[0].split)},
            "max_rel_err": err, "clocks": ck}


def run_decomposed(args):
    """The slab decomposition alone (``--decompose``); rank 0 prints one JSON line."""
    import datetime

    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    line = measure_decomposed(args, ws, rank, local, dist)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="fp64_fft", choices=list(FORMS),
                    help="form of the headline value (the others are reported under 'forms')")
    ap.add_argument("--only", action="store_true", help="measure the headline form only")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle check/baseline")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only warm-up + timed solves of --form (for profiler launch lists and captures)")
    ap.add_argument("--tile", type=int, default=0,
                    help="named workloads with --kernel-only: DFT tile edge (0 = the plan builder's choice; the "
                         "3D FP64 butterfly form takes 16 or 32)")
    ap.add_argument("--sweep", action="store_true", help="named 2-D/3-D workloads: Ozaki slice sweep 4..8")
    ap.add_argument("--no-targets", action="store_true",
                    help="skip the target configurations (Box2D9P 8192^2, Box3D27P 512^3) and the library "
                         "baselines of the default run")
    ap.add_argument("--workload", default="box2d9p",
                    choices=["batch", "competitors", "reference_gpu", "host_slabs"] + list(WORKLOADS),
                    help="box2d9p: the headline workload (full JSON contract); batch: the 512-problem mixed "
                         "batch; others: the other benchmark configurations, every available form")
    ap.add_argument("--problems", type=int, default=512, help="batch workload: number of problems (512 = C5)")
    ap.add_argument("--decompose", action="store_true",
                    help="headline grid split into slabs over the N ranks (strong scaling) instead of N replicas")
    args = ap.parse_args()
    if args.decompose and args.impl != "reference":
        return run_decomposed(args)
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batch":
        return run_batch_workload(args)
    if args.workload == "competitors":
        return run_competitors(args)
    if args.workload == "reference_gpu":
        return run_reference_gpu(args)
    if args.workload == "host_slabs":
        return run_host_slabs(args)
    if args.workload != "box2d9p":
        return run_named_workload(args)

    import torch
    import flashfftstencil_b200 as ffs

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist

    def barrier():
        if pg:
            pg.barrier()

    n, T = WORKLOAD["n"], WORKLOAD["T"]
    x_np, w = seeded_inputs(n, 1, SEED + rank)
    d_in = torch.from_numpy(x_np).cuda()

    if args.kernel_only:  # box2d9p
        plan = ffs.Plan(2, None, (n, n), T, weights=w, radius=1, boundary=WORKLOAD["boundary"], form=args.form,
                        slices=FORMS[args.form][1])
        d_out = torch.empty_like(d_in)
        for _ in range(args.warmup + args.steps):
            plan.run(d_in, d_out)
        torch.cuda.synchronize()
        plan.close()
        return 0

    # the oracle result of this exact workload (rank 0) checks every form and is the CPU baseline
    ref, cpu_baseline = None, None
    if rank == 0 and not args.no_cpu:
        ref, dt_cpu, cores = cpu_oracle_baseline(x_np, w, T)
        cpu_baseline = {"value": n * n * T / dt_cpu / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
                        "sample": f"oracle (direct FP64 stepping, fixed ring, OpenMP) full workload {n}x{n} T={T}"
                                  f" in {dt_cpu:.2f} s"}

    order = [args.form] + ([] if args.only else [f for f in FORMS if f != args.form])
    results = {}
    head_plan = None
    for form in order:
        clocks = Clocks(local) if form == args.form else None
        plan, r = measure_form(ffs, torch, form, n, T, w, d_in, args.steps, args.warmup, ref, clocks,
                               barrier if pg else None)
        ms = r["ms_total"]
        if pg:
            t = torch.tensor([ms], device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = t.item()
        r["ms_total"] = ms
        r["value"] = ws * float(n) * n * T * args.steps / (ms * 1e-3) / 1e9
        results[form] = r
        if form == args.form:
            head_plan = plan
        else:
            plan.close()
    # the butterfly form's other 2D tile edge (64 x 64 pairs or one real 128 x 128 tile per CTA),
    # beside the plan builder's choice for this grid
    other_edge = None
    if "fp64_fft" in results and not pg:
        edge = 64 if results["fp64_fft"]["info"]["tile"] == 128 else 128
        plan_o, r_o = measure_form(ffs, torch, "fp64_fft", n, T, w, d_in, args.steps, args.warmup, ref, tile=edge)
        plan_o.close()
        p_o = r_o["profile"]
        other_edge = {"value": float(n) * n * T * args.steps / (r_o["ms_total"] * 1e-3) / 1e9, "unit": UNIT,
                      "ms_per_step": r_o["ms_total"] / args.steps, "tile": r_o["info"]["tile"],
                      "tau": r_o["info"]["tau"], "passes": r_o["info"]["passes"], "accuracy": r_o["accuracy"],
                      "tile_kernel_ms": p_o["tile_ms"] / max(p_o["tile_launches"], 1)}
    head = results[args.form]
    info, prof, ms = head["info"], head["profile"], head["ms_total"]

    # end to end through the public API with host buffers (pinned): every step copies its own grid
    # in and its result out inside the timed region.  ffs_execute_host_many runs the K steps as K
    # grids and pipelines them on two device slots (copy-out of grid i beside the compute of grid
    # i+1 and the copy-in of grid i+2); the host buffers rotate over a ring of two inputs and two
    # outputs.  The single-grid call (ffs_execute_host, nothing to overlap) is timed beside it.
    stream = torch.cuda.current_stream()
    ring = 2
    pin_in = [torch.from_numpy(x_np).pin_memory() for _ in range(ring)]
    pin_out = [torch.empty_like(pin_in[0]).pin_memory() for _ in range(ring)]
    xs = [pin_in[i % ring].numpy() for i in range(args.steps)]
    ys = [pin_out[i % ring].numpy() for i in range(args.steps)]
    head_plan.run_host_many(xs[:max(args.warmup, 3)], ys[:max(args.warmup, 3)], stream=stream.cuda_stream)
    # three timed repetitions of the K-grid pipeline, the median reported: the PCIe link is
    # shared with the host's other GPUs, and single runs of it varied by up to 3x between boxes
    reps_e2e = []
    for _ in range(3):
        barrier()
        torch.cuda.synchronize()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        head_plan.run_host_many(xs, ys, stream=stream.cuda_stream)
        e3.record(stream)
        torch.cuda.synchronize()
        barrier()
        reps_e2e.append(e2.elapsed_time(e3))
    ms_e2e = statistics.median(reps_e2e)
    e2e_err = None
    if ref is not None:
        e2e_err = max(float(np.abs(y.numpy() - ref).max() / np.abs(ref).max()) for y in pin_out)
    # one grid through ffs_execute_host: on slabs when the plan's model prefers them
    # (host_slabs > 1), so its copy-in, compute and copy-out overlap within the grid
    single = 5
    head_plan.run_host(xs[0], ys[0], stream=stream.cuda_stream)  # warm-up: slab sub-plans, buffers
    single_err = None if ref is None else float(np.abs(ys[0] - ref).max() / np.abs(ref).max())
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    for i in range(single):
        head_plan.run_host(xs[i % len(xs)], ys[i % len(ys)], stream=stream.cuda_stream)
    e5.record(stream)
    torch.cuda.synchronize()
    ms_single = e4.elapsed_time(e5) / single
    # the link's rate with both directions busy (pinned copies of the grid's size, one stream per
    # direction, as the pipeline uses): the roofline of the end-to-end figure
    d_a = torch.empty_like(pin_in[0], device="cuda")
    d_b = torch.empty_like(pin_in[0], device="cuda")
    s_h2d, s_d2h = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    t_link = time.perf_counter()
    for _ in range(5):
        with torch.cuda.stream(s_h2d):
            d_a.copy_(pin_in[0], non_blocking=True)
        with torch.cuda.stream(s_d2h):
            pin_out[1].copy_(d_b, non_blocking=True)
        torch.cuda.synchronize()
    link_gbs = x_np.nbytes * 5 / (time.perf_counter() - t_link) / 1e9
    del d_a, d_b
    if pg:
        t = torch.tensor([ms_e2e, ms_single], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_e2e, ms_single = t.tolist()
    cell_steps = float(n) * n * T
    value = head["value"]
    e2e_value = ws * cell_steps * args.steps / (ms_e2e * 1e-3) / 1e9

    # pipe peaks measured in this run (MEASURED_PEAKS.json has HBM and cuBLAS BF16 only)
    peak_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks_file = json.load(open(peak_path)) if os.path.exists(peak_path) else {}
    hbm_peak = peaks_file.get("hbm_gbs", 6650.0)
    import ctypes
    plib = ctypes.CDLL(os.path.join(ROOT, "flashfftstencil_b200", "libffs_peaks.so"))
    plib.ffs_peak_dmma.restype = ctypes.c_double
    plib.ffs_peak_dmma.argtypes = [ctypes.c_int, ctypes.c_int]
    plib.ffs_peak_dfma.restype = ctypes.c_double
    plib.ffs_peak_dfma.argtypes = [ctypes.c_int, ctypes.c_int]
    plib.ffs_peak_tc.restype = ctypes.c_double
    plib.ffs_peak_tc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    plib.ffs_peak_smem.restype = ctypes.c_double
    plib.ffs_peak_smem.argtypes = [ctypes.c_int, ctypes.c_int]
    peaks = {"fp64_dmma_tflops": plib.ffs_peak_dmma(4000, 5), "fp64_fma_tflops": plib.ffs_peak_dfma(20000, 3),
             "smem_gbs": plib.ffs_peak_smem(20000, 3),
             "int8_tc_tops": plib.ffs_peak_tc(1, 20000, 3),
             "bf16_tc_tflops": plib.ffs_peak_tc(0, 20000, 3),
             "bf16_cublas_tflops_file": peaks_file.get("bf16_tflops"), "hbm_gbs_file": hbm_peak,
             "how": "issue loops in libffs_peaks.so on this GPU (mma.sync f64; fma.rn.f64; 16-byte shared loads; "
                    "tcgen05.mma i8 M128N256K32, "
                    "bf16 M128N256K16), best of reps"}
    pipe_peak = {"fp64": peaks["fp64_dmma_tflops"], "fp64_fft": peaks["fp64_fma_tflops"], "ozaki": peaks["int8_tc_tops"],
                 "bf16x3": peaks["bf16_tc_tflops"]}
    kern_name = {"fp64": "ffst::dmma2d::dmma2d_kernel", "fp64_fft": "ffst::fft2d::fft2d_kernel",
                 "ozaki": "ffst::tc2d::tc2d_kernel<2,7>",
                 "bf16x3": "ffst::tc2d::tc2d_kernel<3,3>"}

    forms_out = {}
    for form, r in results.items():
        p_ = r["profile"]
        avg = p_["tile_ms"] / max(p_["tile_launches"], 1)
        ach = r["info"]["exec_flops_per_pass"] / (avg * 1e-3) / 1e12
        forms_out[FORMS[form][0]] = {
            "value": r["value"], "unit": UNIT, "ms_per_step": r["ms_total"] / args.steps,
            "slices": r["info"]["slices"] or None, "tau": r["info"]["tau"], "passes": r["info"]["passes"],
            "accuracy": r["accuracy"], "tile_kernel_ms": avg,
            "pipe_achieved": ach, "pipe_peak": pipe_peak[form],
            "pipe_frac": ach / pipe_peak[form] if pipe_peak[form] else None,
            "pipe_unit": "TOPS (int8)" if form == "ozaki" else "TFLOP/s",
            "fp64_equiv_tflops": r["info"]["flops_per_pass"] / (avg * 1e-3) / 1e12}
    if "fp64" in results and "ozaki" in results:
        forms_out["ozaki_vs_fp64"] = results["ozaki"]["value"] / results["fp64"]["value"]
    if other_edge:
        forms_out[f"fp64_fft_tile{other_edge['tile']}"] = other_edge

    avg_tile_ms = prof["tile_ms"] / max(prof["tile_launches"], 1)
    achieved = info["exec_flops_per_pass"] / (avg_tile_ms * 1e-3) / 1e12
    hbm_achieved = info["hbm_bytes_per_pass"] / (avg_tile_ms * 1e-3) / 1e9
    tr = read_traffic(args.form, info["tile"])
    peak = pipe_peak[args.form]
    pipe = {"achieved": achieved, "peak": peak, "unit": "TOPS" if args.form == "ozaki" else "TFLOP/s",
            "frac": achieved / peak if peak else None}
    if args.form == "fp64_fft":
        # no tensor pipe: the binding roof is shared-memory bandwidth, the FP64 pipe is reported beside it
        if info["tile"] == 128:
            smem_bytes = fft2d128_smem_bytes_per_tile(info["useful"]) * info["tiles"]
            smem_how = "bench.fft2d128_smem_bytes_per_tile x tiles"
        else:
            smem_bytes = fft2d_smem_bytes_per_pair(info["useful"]) * info["tiles"] / 2
            smem_how = "bench.fft2d_smem_bytes_per_pair x tile pairs"
        smem_achieved = smem_bytes / (avg_tile_ms * 1e-3) / 1e9
        roofline = {"bound": "smem", "achieved": smem_achieved, "peak": peaks["smem_gbs"], "unit": "GB/s",
                    "frac": smem_achieved / peaks["smem_gbs"] if peaks["smem_gbs"] else None,
                    "smem_bytes_per_launch": smem_bytes,
                    "smem_note": f"algorithmic shared-memory bytes of the butterfly kernel's design per launch "
                                 f"({smem_how})",
                    "fp64_pipe": dict(pipe, peak_source="fma.rn.f64 loop")}
    else:
        roofline = dict({"bound": "tensor"}, **pipe)
    roofline.update({
                "traffic": tr.get("bytes_per_launch") if tr else None,
                "traffic_source": (f"{tr.get('source')} (profiles/{TRAFFIC_FILES[(args.form, info['tile'])]}, captured on "
                                   f"commit {tr.get('captured_on', 'unrecorded')}, not measured in this run)")
                                  if tr else None,
                "kernel": ("ffst::fft2d128::fft2d128_kernel" if args.form == "fp64_fft" and info["tile"] == 128
                           else kern_name[args.form]),
                "peak_source": "measured in this run: " + peaks["how"],
                "flops_per_launch": info["exec_flops_per_pass"],
                "flops_note": ("FP64 operations of the butterflies per launch (add = mul = 1, fma = 2)"
                               if args.form == "fp64_fft" else
                               "executed DFT-GEMM ops per launch (radix-8 8(d) count for fp64; dense DFT-64 x "
                               "slice products for the tensor-core forms)") +
                              f"; dense-DFT FP64 equivalent {info['flops_per_pass']:.4g} per launch",
                "avg_launch_ms": avg_tile_ms,
                "launch_timing": "CUDA events around every launch on its own stream, over a second run of "
                                 "the same K steps (value is timed without them: they slow the solve to "
                                 f"{head['ms_total_profiled'] / args.steps:.4f} ms per step)",
                "hbm": {"achieved_gbs": hbm_achieved, "peak_gbs": hbm_peak, "frac": hbm_achieved / hbm_peak,
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks_file else "fallback"}})
    launches = prof["tile_launches"] + prof["band_launches"]
    # on several GPUs the same headline grid is also solved split into slabs over the ranks
    # (strong scaling, NCCL ghost exchange per pass), reported beside the replicas value
    decomposed = None
    if pg:
        try:  # a failure here (it is the only cross-rank data exchange) must not cost the replicas line
            d = measure_decomposed(args, ws, rank, local, pg)
            decomposed = {k: d[k] for k in ("value", "unit", "ms_per_step", "scaling", "config", "max_rel_err",
                                            "clocks")}
        except Exception as exc:  # noqa: BLE001
            decomposed = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    targets = competitors = None
    if ws == 1 and not args.no_targets and not args.only:
        targets = measure_targets(ffs, torch, min(args.steps, 20), args.warmup, not args.no_cpu)
        competitors = measure_competitors()
    acc = head["accuracy"]
    if acc is not None:
        acc = dict(acc, tolerance=1e-12, **{"pass": bool(acc["max_rel_err"] <= 1e-12)})
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{WORKLOAD['shape']} {n}x{n} FP64, fixed ring width 1, T={T}, "
                                   "U[0,1) inputs, U(0,1) weights normalised to 1",
                       "form": info["form"], "tile": info["tile"], "tau": info["tau"], "passes": info["passes"],
                       "l2": "inputs larger than L2 (134 MB grid in + out + workspace)",
                       "parallelism": f"replicas x{ws} (independent grids)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(x_np.nbytes),
                    "d2h_bytes_per_step": int(x_np.nbytes), "ms_per_step": ms_e2e / args.steps,
                    "api": "ffs_execute_host_many (K grids, copies pipelined across grids)",
                    "repetitions_ms_per_step": [r / args.steps for r in reps_e2e],
                    "timing": "median of three timed runs of the K grids",
                    "max_rel_err": e2e_err,
                    "link": {"gbs_per_direction_both_busy": link_gbs,
                             "achieved_gbs_per_direction": x_np.nbytes / (ms_e2e / args.steps * 1e-3) / 1e9,
                             "frac": x_np.nbytes / (ms_e2e / args.steps * 1e-3) / 1e9 / link_gbs,
                             "note": "pinned copies of one grid each way at once, 5 repetitions, wall clock"},
                    "single_grid": {"api": "ffs_execute_host", "ms": ms_single,
                                    "value": ws * float(n) * n * T / (ms_single * 1e-3) / 1e9,
                                    "host_slabs": head_plan.info["host_slabs"], "max_rel_err": single_err}},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu_baseline,
            "accuracy": acc,
            "clocks": head["clocks"],
            "forms": forms_out,
            "decomposed": decomposed,
            "targets": targets,
            "competitors": competitors,
            "peaks": peaks,
            "kernel_ms": {"tile_total": prof["tile_ms"], "band_total": prof["band_ms"]}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    head_plan.close()
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
