#!/usr/bin/env python
"""Benchmark of the fused DFT-tile stencil path on B200.

Workload (default): Box2D9P on a 4096 x 4096 FP64 grid, uniform[0,1) inputs and
3x3 weights uniform(0,1) normalised to sum 1 (both from a seeded mt19937-style
generator), fixed boundary ring of width 1, T = 32 true time steps.  One bench
"step" is one full T-step solve (ffs_execute).  Metric: GStencil/s =
interior cells x T / s / 1e9, at <= 1e-12 max relative error against the FP64
oracle (checked in the same run).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form fp64|ozaki|bf16x3]

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
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20251203 + 1
WORKLOAD = dict(shape="Box2D9P", n=4096, T=32, boundary="fixed")
METRIC = "GStencil/s (cells x steps / s) at <=1e-12 max rel err vs FP64 oracle"
UNIT = "GStencil/s"


def seeded_inputs(n, r, seed):
    rng = np.random.Generator(np.random.MT19937(seed))
    x = rng.random((n, n))
    w = rng.random((2 * r + 1, 2 * r + 1))
    w /= w.sum()
    return x, w


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
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{index}.csv")

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


def read_traffic():
    path = os.path.join(ROOT, "profiles", "dmma2d_box2d9p_4096_traffic.json")
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="fp64", choices=["fp64", "ozaki", "bf16x3", "auto"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle check/baseline")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only warm-up + timed solves (for profiler launch lists and captures)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

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
    plan = ffs.Plan(2, None, (n, n), T, weights=w, radius=1, boundary=WORKLOAD["boundary"], form=args.form)
    info = plan.info
    stream = torch.cuda.current_stream()
    d_in = torch.from_numpy(x_np).cuda()
    d_out = torch.empty_like(d_in)

    if args.kernel_only:
        for _ in range(args.warmup + args.steps):
            plan.run(d_in, d_out)
        torch.cuda.synchronize()
        plan.close()
        return 0

    # correctness of this exact run against the oracle (rank 0), doubling as the CPU baseline
    accuracy = None
    cpu_baseline = None
    plan.run(d_in, d_out)
    torch.cuda.synchronize()
    if rank == 0 and not args.no_cpu:
        from tests.helpers import rel_errors
        ref, dt_cpu, cores = cpu_oracle_baseline(x_np, w, T)
        mx, l2 = rel_errors(d_out.cpu().numpy(), ref)
        accuracy = {"max_rel_err": mx, "l2_rel_err": l2, "tolerance": 1e-12, "pass": bool(mx <= 1e-12)}
        cpu_baseline = {"value": n * n * T / dt_cpu / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
                        "sample": f"oracle (direct FP64 stepping, fixed ring, OpenMP) full workload {n}x{n} T={T}"
                                  f" in {dt_cpu:.2f} s"}

    for _ in range(max(args.warmup, 3)):
        plan.run(d_in, d_out)
    torch.cuda.synchronize()

    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    plan.profile(True)
    plan.profile_read(reset=True)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        plan.run(d_in, d_out)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    prof = plan.profile_read(reset=True)
    plan.profile(False)
    ck = clocks.stop()
    if pg:
        t = torch.tensor([ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = t.item()

    # end to end through the public API with host buffers (pinned), copies inside the timed region
    h_in = torch.from_numpy(x_np).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    hi, ho = h_in.numpy(), h_out.numpy()
    for _ in range(2):
        plan.run_host(hi, ho)
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        plan.run_host(hi, ho, stream=stream.cuda_stream)
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = e2.elapsed_time(e3)
    if pg:
        t = torch.tensor([ms_e2e], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_e2e = t.item()

    cell_steps = float(n) * n * T
    value = ws * cell_steps * args.steps / (ms * 1e-3) / 1e9
    e2e_value = ws * cell_steps * args.steps / (ms_e2e * 1e-3) / 1e9

    # roofline of the dominant kernel (the fused tile kernel)
    peak_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peak_path)) if os.path.exists(peak_path) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    import ctypes
    plib = ctypes.CDLL(os.path.join(ROOT, "flashfftstencil_b200", "libffs_peaks.so"))
    plib.ffs_peak_dmma.restype = ctypes.c_double
    plib.ffs_peak_dmma.argtypes = [ctypes.c_int, ctypes.c_int]
    dmma_peak = plib.ffs_peak_dmma(4000, 5)
    avg_tile_ms = prof["tile_ms"] / max(prof["tile_launches"], 1)
    achieved = info["exec_flops_per_pass"] / (avg_tile_ms * 1e-3) / 1e12
    hbm_achieved = info["hbm_bytes_per_pass"] / (avg_tile_ms * 1e-3) / 1e9
    tr = read_traffic()
    roofline = {"bound": "tensor", "achieved": achieved, "peak": dmma_peak, "unit": "TFLOP/s",
                "frac": achieved / dmma_peak if dmma_peak > 0 else None,
                "traffic": tr.get("bytes_per_launch") if tr else None,
                "kernel": "ffst::dmma2d::dmma2d_kernel",
                "peak_source": "FP64 mma.sync.m8n8k4 issue loop (libffs_peaks.so), measured in this run",
                "flops_per_launch": info["exec_flops_per_pass"],
                "flops_note": "radix-8 DFT-GEMM flops (8(d) count with n -> n1+n2 = 16); dense-DFT equivalent "
                              f"{info['flops_per_pass']:.4g} per launch",
                "avg_launch_ms": avg_tile_ms,
                "hbm": {"achieved_gbs": hbm_achieved, "peak_gbs": hbm_peak, "frac": hbm_achieved / hbm_peak,
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback"}}
    launches = prof["tile_launches"] + prof["band_launches"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{WORKLOAD['shape']} {n}x{n} FP64, fixed ring width 1, T={T}, "
                                   "U[0,1) inputs, U(0,1) weights normalised to 1",
                       "form": info["form"], "tile": info["tile"], "tau": info["tau"], "passes": info["passes"],
                       "l2": "inputs larger than L2 (134 MB grid in + out + workspace)",
                       "parallelism": f"replicas x{ws} (independent grids)"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(x_np.nbytes),
                    "d2h_bytes_per_step": int(x_np.nbytes)},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu_baseline,
            "accuracy": accuracy,
            "clocks": ck,
            "kernel_ms": {"tile_total": prof["tile_ms"], "band_total": prof["band_ms"]}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
