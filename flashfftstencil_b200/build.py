"""Build libffs.so (the C-ABI library with the sm_100a kernels) and the CLI.

Compiles every CUDA/C++ source under csrc/ with nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) and links one shared library with a
static CUDA runtime, so it loads on hosts without a GPU driver (the driver is
reached lazily at the first CUDA call).  Objects go to _build/ (git-ignored).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libffs.so")
CLI = os.path.join(PKG, "ffs")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC]
LIB_SOURCES = ["ffs_api.cpp", "ffs_plan.cpp", "ffs_dmma2d.cu", "ffs_fft1d.cu", "ffs_fft2d.cu", "ffs_fft3d.cu", "ffs_fft3d32.cu", "ffs_fft2d128.cu", "ffs_dmma1d.cu", "ffs_dmma3d.cu", "ffs_tc2d.cu", "ffs_tc3d.cu", "ffs_band.cu", "ffs_batch.cu", "ffs_noalloc.cu", "ffs_util.cu"]
CLI_SOURCES = ["ffs_cli.cpp"]
PEAKS_SRC = "ffs_peaks.cu"
PEAKS_LIB = os.path.join(PKG, "libffs_peaks.so")


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_compiler_flags() -> list[str]:
    gxx = "/usr/bin/g++"
    return ["-ccbin", gxx] if os.path.exists(gxx) else []


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs + [os.path.join(INCLUDE, "ffs.h")]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    hdrs = _headers()
    objs = []
    for src in LIB_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + hdrs):
            cmd = [cc, *ARCH, *NVCC_FLAGS, *_host_compiler_flags(), "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    if force or _stale(LIB, objs):
        cmd = [cc, *ARCH, *_host_compiler_flags(), "-shared", "-cudart", "static", "-o", LIB, *objs]
        _run(cmd)
    psrc = os.path.join(CSRC, PEAKS_SRC)
    if force or _stale(PEAKS_LIB, [psrc]):
        _run([cc, *ARCH, *NVCC_FLAGS, *_host_compiler_flags(), "-shared", "-cudart", "static", psrc, "-o",
              PEAKS_LIB])
    cli_src = [os.path.join(CSRC, s) for s in CLI_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if cli_src and (force or _stale(CLI, cli_src + [LIB] + hdrs)):
        cmd = [cc, *_host_compiler_flags(), "-O2", "-std=c++17", "-I" + INCLUDE, "-I" + CSRC, *cli_src,
               "-o", CLI, "-L" + PKG, "-lffs", "-Xlinker", "-rpath=$ORIGIN", "-cudart", "static"]
        _run(cmd)
    for d in ("1d", "2d", "3d"):  # reference program names: the dimension comes from argv[0]
        link = os.path.join(PKG, f"{d}.out")
        if os.path.exists(CLI) and not os.path.islink(link):
            os.symlink("ffs", link)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
