"""CPU oracle for the fused DFT-tile stencil path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` /
``--impl reference`` legs may import this package, and only as the checker or
the timed CPU baseline.  The product (``flashfftstencil_b200``) never imports it.

``liboracle.so`` is the C restatement in ``stencil_oracle.c`` (it follows the
reference's ``src/1D/check_correct.hpp:15-38`` and ``src/2D/check_correct.hpp:53-100``,
extended to centred correlation, 3D, a fixed boundary and T steps).
``_ref/libffsref.so`` (optional) is the reference's own ``stencil1D``/``stencil2D``
compiled from the reference sources by ``oracle/Makefile``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PERIODIC = 0
FIXED = 1

_lib = None
_ref = None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        i64, dp = ctypes.c_int64, ctypes.POINTER(ctypes.c_double)
        L.ffs_oracle_step.argtypes = [ctypes.c_int, i64, i64, i64, ctypes.c_int, dp, ctypes.c_int, dp, dp]
        L.ffs_oracle_run.argtypes = [ctypes.c_int, i64, i64, i64, ctypes.c_int, dp, ctypes.c_int,
                                     ctypes.c_int, dp, dp]
        L.ffs_oracle_max_threads.restype = ctypes.c_int
        L.ffs_oracle_set_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own CPU stencils (None when oracle/_ref was not built)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libffsref.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        L.ffs_ref_stencil1d.argtypes = [dp, ctypes.c_int, dp, ctypes.c_int, dp]
        L.ffs_ref_stencil2d.argtypes = [dp, ctypes.c_int, dp, ctypes.c_int, dp]
        L.ffs_ref_rotate180.argtypes = [dp, ctypes.c_int, dp]
        _ref = L
    return _ref


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _extents(grid: np.ndarray, dim: int):
    shp = grid.shape
    if len(shp) != dim:
        raise ValueError(f"grid has {len(shp)} dims, expected {dim}")
    nx = shp[-1]
    ny = shp[-2] if dim >= 2 else 1
    nz = shp[-3] if dim >= 3 else 1
    return nx, ny, nz


def run(grid: np.ndarray, weights: np.ndarray, radius: int, T: int, boundary: int = PERIODIC,
        threads: int | None = None) -> np.ndarray:
    """T steps of the centred-correlation stencil on a 1/2/3-D FP64 grid."""
    grid = np.ascontiguousarray(grid, dtype=np.float64)
    dim = grid.ndim
    w = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
    if w.size != (2 * radius + 1) ** dim:
        raise ValueError("weights must be a dense (2r+1)^dim array")
    nx, ny, nz = _extents(grid, dim)
    out = np.empty_like(grid)
    L = lib()
    if threads:
        L.ffs_oracle_set_threads(int(threads))
    rc = L.ffs_oracle_run(dim, nx, ny, nz, radius, _dp(w), boundary, int(T), _dp(grid), _dp(out))
    if rc != 0:
        raise RuntimeError(f"ffs_oracle_run failed with code {rc}")
    return out


def max_threads() -> int:
    return int(lib().ffs_oracle_max_threads())


def ref_stencil1d(x: np.ndarray, k: np.ndarray) -> np.ndarray:
    L = ref_lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    k = np.ascontiguousarray(k, dtype=np.float64)
    out = np.empty_like(x)
    L.ffs_ref_stencil1d(_dp(x), x.size, _dp(k), k.size, _dp(out))
    return out


def ref_stencil2d(x: np.ndarray, k: np.ndarray) -> np.ndarray:
    L = ref_lib()
    x = np.ascontiguousarray(x, dtype=np.float64)
    k = np.ascontiguousarray(k, dtype=np.float64)
    out = np.empty_like(x)
    L.ffs_ref_stencil2d(_dp(x), x.shape[0], _dp(k), k.shape[0], _dp(out))
    return out


def ref_rotate180(k: np.ndarray) -> np.ndarray:
    L = ref_lib()
    k = np.ascontiguousarray(k, dtype=np.float64)
    out = np.empty_like(k)
    L.ffs_ref_rotate180(_dp(k), k.shape[0], _dp(out))
    return out


def spectral_periodic(grid: np.ndarray, weights: np.ndarray, radius: int, T: int) -> np.ndarray:
    """Independent periodic check via numpy.fft: out = IFFT(FFT(x) * S^T).

    S(k) = sum_d w[d] exp(+2 pi i d.k / n) is the correlation symbol.
    """
    grid = np.asarray(grid, dtype=np.float64)
    dim = grid.ndim
    K = 2 * radius + 1
    w = np.asarray(weights, dtype=np.float64).reshape((K,) * dim)
    ker = np.zeros(grid.shape)
    for idx in np.ndindex(*w.shape):
        d = tuple(i - radius for i in idx)
        pos = tuple((-dd) % n for dd, n in zip(d, grid.shape))
        ker[pos] += w[idx]
    # correlation with w == convolution with the flipped kernel placed at -d
    S = np.fft.fftn(ker)
    return np.real(np.fft.ifftn(np.fft.fftn(grid) * S ** T))
