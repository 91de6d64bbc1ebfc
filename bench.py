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


FORMS = {"fp64": ("fp64_dmma", 0), "ozaki": ("ozaki_i8", 7), "bf16x3": ("bf16x3", 3)}


def measure_form(ffs, torch, form, n, T, w, d_in, steps, warmup, ref, clocks=None, barrier=None):
    """One form on the workload: accuracy vs the oracle result, then `steps` timed solves."""
    from tests.helpers import rel_errors
    slices = FORMS[form][1]
    plan = ffs.Plan(2, None, (n, n), T, weights=w, radius=1, boundary=WORKLOAD["boundary"], form=form,
                    slices=slices)
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
    plan.profile(True)
    plan.profile_read(reset=True)
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
    ms = e0.elapsed_time(e1)
    prof = plan.profile_read(reset=True)
    plan.profile(False)
    ck = clocks.stop() if clocks else None
    return plan, {"ms_total": ms, "accuracy": acc, "profile": prof, "info": plan.info, "clocks": ck}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="fp64", choices=["fp64", "ozaki", "bf16x3"],
                    help="form of the headline value (the others are reported under 'forms')")
    ap.add_argument("--only", action="store_true", help="measure the headline form only")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle check/baseline")
    ap.add_argument("--kernel-only", action="store_true",
                    help="only warm-up + timed solves of --form (for profiler launch lists and captures)")
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
    d_in = torch.from_numpy(x_np).cuda()

    if args.kernel_only:
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
    head = results[args.form]
    info, prof, ms = head["info"], head["profile"], head["ms_total"]

    # end to end through the public API with host buffers (pinned), copies inside the timed region
    stream = torch.cuda.current_stream()
    h_in = torch.from_numpy(x_np).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    hi, ho = h_in.numpy(), h_out.numpy()
    for _ in range(2):
        head_plan.run_host(hi, ho, stream=stream.cuda_stream)
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        head_plan.run_host(hi, ho, stream=stream.cuda_stream)
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms_e2e = e2.elapsed_time(e3)
    if pg:
        t = torch.tensor([ms_e2e], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_e2e = t.item()
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
    plib.ffs_peak_tc.restype = ctypes.c_double
    plib.ffs_peak_tc.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    peaks = {"fp64_dmma_tflops": plib.ffs_peak_dmma(4000, 5), "int8_tc_tops": plib.ffs_peak_tc(1, 20000, 3),
             "bf16_tc_tflops": plib.ffs_peak_tc(0, 20000, 3),
             "bf16_cublas_tflops_file": peaks_file.get("bf16_tflops"), "hbm_gbs_file": hbm_peak,
             "how": "issue loops in libffs_peaks.so on this GPU (mma.sync f64; tcgen05.mma i8 M128N256K32, "
                    "bf16 M128N256K16), best of reps"}
    pipe_peak = {"fp64": peaks["fp64_dmma_tflops"], "ozaki": peaks["int8_tc_tops"],
                 "bf16x3": peaks["bf16_tc_tflops"]}
    kern_name = {"fp64": "ffst::dmma2d::dmma2d_kernel", "ozaki": "ffst::tc2d::tc2d_kernel<2,7>",
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

    avg_tile_ms = prof["tile_ms"] / max(prof["tile_launches"], 1)
    achieved = info["exec_flops_per_pass"] / (avg_tile_ms * 1e-3) / 1e12
    hbm_achieved = info["hbm_bytes_per_pass"] / (avg_tile_ms * 1e-3) / 1e9
    tr = read_traffic() if args.form == "fp64" else None
    peak = pipe_peak[args.form]
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak,
                "unit": "TOPS" if args.form == "ozaki" else "TFLOP/s",
                "frac": achieved / peak if peak else None,
                "traffic": tr.get("bytes_per_launch") if tr else None,
                "kernel": kern_name[args.form],
                "peak_source": "measured in this run: " + peaks["how"],
                "flops_per_launch": info["exec_flops_per_pass"],
                "flops_note": "executed DFT-GEMM ops per launch (radix-8 8(d) count for fp64; dense DFT-64 x "
                              "slice products for the tensor-core forms); dense-DFT FP64 equivalent "
                              f"{info['flops_per_pass']:.4g} per launch",
                "avg_launch_ms": avg_tile_ms,
                "hbm": {"achieved_gbs": hbm_achieved, "peak_gbs": hbm_peak, "frac": hbm_achieved / hbm_peak,
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks_file else "fallback"}}
    launches = prof["tile_launches"] + prof["band_launches"]
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
                    "d2h_bytes_per_step": int(x_np.nbytes)},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "cpu_baseline": cpu_baseline,
            "accuracy": acc,
            "clocks": head["clocks"],
            "forms": forms_out,
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
