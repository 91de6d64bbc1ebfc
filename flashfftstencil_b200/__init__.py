"""flashfftstencil_b200 -- B200 (sm_100a) fused DFT-tile stencil solver.

Python mirror of the C ABI in ``include/ffs.h`` (``libffs.so``).  The
reference's surface is ``CreatePlan(double* k, int K, bool print)`` plus a tile
kernel launched T times (``src/2D/create_fft_pfa_plan.cu:17``,
``src/2D/2d_main.cu:150-170``); here :class:`Plan` (alias :func:`CreatePlan`)
owns the spectra and tables and :meth:`Plan.execute` runs all T steps.

There is no CPU fallback: importing this package fails loudly when
``libffs.so`` has not been built (``python flashfftstencil_b200/build.py``).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libffs.so")

# ---- enums (mirror include/ffs.h) ----
OK, ERR_INVALID_ARGUMENT, ERR_UNSUPPORTED, ERR_CUDA, ERR_OUT_OF_MEMORY, ERR_TIMEOUT, ERR_INTERNAL = range(7)
BOUNDARY = {"periodic": 0, "fixed": 1}
FORM = {"auto": 0, "fp64": 1, "fp64_dmma": 1, "ozaki": 2, "ozaki_i8": 2, "bf16x3": 3, "fp64_fft": 4}
FORM_NAME = {0: "auto", 1: "fp64_dmma", 2: "ozaki_i8", 3: "bf16x3", 4: "fp64_fft"}
SHAPES = ("Heat-1D", "1D5P", "1D7P", "Heat-2D", "Box2D9P", "Star2D9P", "Box2D25P", "Heat-3D", "Box3D27P")


class FFSError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"ffs status {status}: {msg}")
        self.status = status


class _Problem(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("shape", ctypes.c_int),
        ("radius", ctypes.c_int),
        ("extents", ctypes.c_int64 * 3),
        ("weights", ctypes.POINTER(ctypes.c_double)),
        ("T", ctypes.c_int),
        ("boundary", ctypes.c_int),
        ("form", ctypes.c_int),
        ("slices", ctypes.c_int),
        ("tau", ctypes.c_int),
        ("open_faces", ctypes.c_int),
        ("tile", ctypes.c_int),
        ("reserved", ctypes.c_int * 6),
    ]


class _Info(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("radius", ctypes.c_int),
        ("form", ctypes.c_int),
        ("tile", ctypes.c_int),
        ("halo", ctypes.c_int),
        ("useful", ctypes.c_int),
        ("tau", ctypes.c_int),
        ("tau_last", ctypes.c_int),
        ("passes", ctypes.c_int),
        ("slices", ctypes.c_int),
        ("tiles", ctypes.c_int64),
        ("work_bytes", ctypes.c_int64),
        ("flops_per_pass", ctypes.c_double),
        ("exec_flops_per_pass", ctypes.c_double),
        ("hbm_bytes_per_pass", ctypes.c_double),
        ("host_slabs", ctypes.c_int),
        ("model_ms", ctypes.c_double),
    ]


class _Profile(ctypes.Structure):
    _fields_ = [("tile_ms", ctypes.c_double), ("tile_launches", ctypes.c_int64),
                ("band_ms", ctypes.c_double), ("band_launches", ctypes.c_int64)]


# every symbol include/ffs.h declares
EXPORTS = (
    "ffs_plan_create", "ffs_execute", "ffs_execute_host", "ffs_execute_host_many", "ffs_plan_get_info", "ffs_plan_describe",
    "ffs_plan_destroy", "ffs_autotune", "ffs_plan_profile", "ffs_plan_profile_read", "ffs_shape_lookup", "ffs_batch_create",
    "ffs_batch_execute", "ffs_batch_destroy", "ffs_batch_status", "ffs_execute_noalloc", "ffs_noalloc_status", "ffs_last_error_string", "ffs_abi_version",
)


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python flashfftstencil_b200/build.py` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip = ctypes.c_void_p, ctypes.c_int
    L.ffs_plan_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(_Problem)]
    L.ffs_execute.argtypes = [vp, vp, vp, vp]
    L.ffs_execute_host.argtypes = [vp, vp, vp, vp]
    L.ffs_execute_host_many.argtypes = [vp, ip, ctypes.POINTER(vp), ctypes.POINTER(vp), vp]
    L.ffs_plan_get_info.argtypes = [vp, ctypes.POINTER(_Info)]
    L.ffs_plan_describe.argtypes = [ctypes.POINTER(_Problem), ctypes.POINTER(_Info)]
    L.ffs_plan_destroy.argtypes = [vp]
    L.ffs_shape_lookup.argtypes = [ctypes.c_char_p, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip),
                                   ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_double), ip]
    L.ffs_autotune.argtypes = [ctypes.POINTER(_Problem), ip, ctypes.POINTER(ip), ctypes.POINTER(ctypes.c_double), vp]
    L.ffs_plan_profile.argtypes = [vp, ip]
    L.ffs_plan_profile_read.argtypes = [vp, ctypes.POINTER(_Profile), ip]
    L.ffs_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), ip]
    L.ffs_batch_execute.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), vp]
    L.ffs_batch_destroy.argtypes = [vp]
    L.ffs_batch_status.argtypes = [vp, ctypes.POINTER(ip)]
    L.ffs_execute_noalloc.argtypes = [ctypes.POINTER(_Problem), vp, vp, vp]
    L.ffs_noalloc_status.argtypes = [ctypes.POINTER(ip)]
    L.ffs_last_error_string.restype = ctypes.c_char_p
    L.ffs_abi_version.restype = ctypes.c_int
    for name in EXPORTS:
        getattr(L, name).restype = getattr(L, name).restype or ctypes.c_int
    L.ffs_last_error_string.restype = ctypes.c_char_p
    return L


lib = _load()


def _check(status: int) -> None:
    if status != OK:
        raise FFSError(status, lib.ffs_last_error_string().decode())


@dataclass
class ShapeInfo:
    name: str
    shape_id: int
    dim: int
    radius: int
    label: str
    weights: np.ndarray


def shape_info(name: str) -> ShapeInfo:
    sid, dim, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    label = ctypes.c_char_p()
    _check(lib.ffs_shape_lookup(name.encode(), ctypes.byref(sid), ctypes.byref(dim), ctypes.byref(r),
                                ctypes.byref(label), None, 0))
    w = np.zeros((2 * r.value + 1) ** dim.value)
    _check(lib.ffs_shape_lookup(name.encode(), None, None, None, None,
                                w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), w.size))
    return ShapeInfo(name, sid.value, dim.value, r.value, label.value.decode(), w)


def _make_problem(dim, shape, extents, T, weights=None, radius=None, boundary="periodic", form="fp64",
                  slices=0, tau=0, open_faces=0, tile=0):
    p = _Problem()
    p.dim = dim
    keep = None
    if shape is None or shape == "custom":
        if weights is None or radius is None:
            raise ValueError("a custom stencil needs weights and radius")
        p.shape = 0
        p.radius = int(radius)
    else:
        si = shape_info(shape)
        if si.dim != dim:
            raise ValueError(f"shape {shape} is {si.dim}-D, not {dim}-D")
        p.shape = si.shape_id
        p.radius = si.radius
    if weights is not None:
        keep = np.ascontiguousarray(weights, dtype=np.float64).reshape(-1)
        p.weights = keep.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ext = list(extents) + [1] * (3 - len(extents))
    for i in range(3):
        p.extents[i] = int(ext[i])
    p.T = int(T)
    p.boundary = BOUNDARY[boundary] if isinstance(boundary, str) else int(boundary)
    p.form = FORM[form] if isinstance(form, str) else int(form)
    p.slices = int(slices)
    p.tau = int(tau)
    p.open_faces = int(open_faces)
    p.tile = int(tile)
    return p, keep


def _info_dict(info: _Info) -> dict:
    d = {k: getattr(info, k) for k, _ in _Info._fields_}
    d["form"] = FORM_NAME.get(d["form"], d["form"])
    return d


def describe(dim, shape, extents, T, **kw) -> dict:
    """Plan geometry (tile, tau, passes ...) without touching the GPU."""
    p, _keep = _make_problem(dim, shape, extents, T, **kw)
    info = _Info()
    _check(lib.ffs_plan_describe(ctypes.byref(p), ctypes.byref(info)))
    return _info_dict(info)


def autotune(dim, shape, extents, T, candidates=0, stream=0, **kw):
    """Time the model's best fused step counts on the device; returns (tau, ms).

    The winner is remembered for this problem class, so later plans with tau=0 use it."""
    p, _keep = _make_problem(dim, shape, extents, T, **kw)
    tau, ms = ctypes.c_int(), ctypes.c_double()
    _check(lib.ffs_autotune(ctypes.byref(p), int(candidates), ctypes.byref(tau), ctypes.byref(ms),
                            ctypes.c_void_p(stream)))
    return tau.value, ms.value


class Plan:
    """A stencil problem bound to the current CUDA device.

    ``extents`` are (nx, ny, nz) with x fastest, i.e. a grid array of shape
    (nz, ny, nx) / (ny, nx) / (nx,) in row-major order.
    """

    def __init__(self, dim, shape, extents, T, weights=None, radius=None, boundary="periodic", form="fp64",
                 slices=0, tau=0, open_faces=0, tile=0):
        self.dim = dim
        self.extents = tuple(int(e) for e in extents)
        self.T = T
        p, _keep = _make_problem(dim, shape, extents, T, weights, radius, boundary, form, slices, tau, open_faces,
                                 tile)
        h = ctypes.c_void_p()
        _check(lib.ffs_plan_create(ctypes.byref(h), ctypes.byref(p)))
        self._h = h
        info = _Info()
        _check(lib.ffs_plan_get_info(h, ctypes.byref(info)))
        self.info = _info_dict(info)

    @property
    def handle(self):
        return self._h

    @property
    def shape(self):
        return tuple(reversed(self.extents[: self.dim]))

    def execute(self, d_in: int, d_out: int, stream: int = 0) -> None:
        """Raw device pointers (ints); asynchronous on `stream`."""
        _check(lib.ffs_execute(self._h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), ctypes.c_void_p(stream)))

    def run(self, x, out=None, stream=None):
        """Run on a CUDA torch tensor (float64, contiguous); returns `out`."""
        import torch
        if x.dtype != torch.float64 or not x.is_cuda or not x.is_contiguous():
            raise ValueError("expected a contiguous float64 CUDA tensor")
        if tuple(x.shape) != self.shape:
            raise ValueError(f"grid shape {tuple(x.shape)} != plan shape {self.shape}")
        if out is None:
            out = torch.empty_like(x)
        s = stream if stream is not None else torch.cuda.current_stream(x.device)
        self.execute(x.data_ptr(), out.data_ptr(), s.cuda_stream)
        return out

    def run_host(self, x: np.ndarray, out: np.ndarray | None = None, stream: int = 0) -> np.ndarray:
        """Host buffers in and out (copies inside; synchronous)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.shape != self.shape:
            raise ValueError(f"grid shape {x.shape} != plan shape {self.shape}")
        if out is None:
            out = np.empty_like(x)
        _check(lib.ffs_execute_host(self._h, ctypes.c_void_p(x.ctypes.data), ctypes.c_void_p(out.ctypes.data),
                                    ctypes.c_void_p(stream)))
        return out

    def run_host_many(self, xs, outs=None, stream: int = 0) -> list:
        """Several grids, host buffers in and out, copies pipelined across grids
        (see ffs_execute_host_many); pinned host arrays let the copies overlap."""
        xs = [np.ascontiguousarray(x, dtype=np.float64) for x in xs]
        for x in xs:
            if x.shape != self.shape:
                raise ValueError(f"grid shape {x.shape} != plan shape {self.shape}")
        if outs is None:
            outs = [np.empty_like(x) for x in xs]
        if len(outs) != len(xs):
            raise ValueError("need one output array per input grid")
        for o in outs:
            if o.shape != self.shape or o.dtype != np.float64 or not o.flags.c_contiguous:
                raise ValueError("outputs must be C-contiguous float64 arrays of the plan's shape")
        n = len(xs)
        ins = (ctypes.c_void_p * max(n, 1))(*[x.ctypes.data for x in xs])
        ous = (ctypes.c_void_p * max(n, 1))(*[o.ctypes.data for o in outs])
        _check(lib.ffs_execute_host_many(self._h, n, ins, ous, ctypes.c_void_p(stream)))
        return outs

    def profile(self, enable: bool = True) -> None:
        """Bracket every kernel launch with CUDA events (see ffs_plan_profile)."""
        _check(lib.ffs_plan_profile(self._h, int(enable)))

    def profile_read(self, reset: bool = True) -> dict:
        pr = _Profile()
        _check(lib.ffs_plan_profile_read(self._h, ctypes.byref(pr), int(reset)))
        return {k: getattr(pr, k) for k, _ in _Profile._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib.ffs_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def CreatePlan(k, K, dim, extents, T, boundary="periodic", form="auto", **kw) -> Plan:
    """Reference-named constructor: weights `k` of width K (K = 2r + 1) per dim; the default
    form is the fastest FP64-exact one (the butterfly kernels)."""
    return Plan(dim, "custom", extents, T, weights=np.asarray(k, dtype=np.float64), radius=(K - 1) // 2,
                boundary=boundary, form=form, **kw)


class Batch:
    """Many plans executed as one CUDA graph replay (ffs_batch_*)."""

    def __init__(self, plans):
        self.plans = list(plans)
        arr = (ctypes.c_void_p * len(self.plans))(*[p.handle for p in self.plans])
        h = ctypes.c_void_p()
        _check(lib.ffs_batch_create(ctypes.byref(h), arr, len(self.plans)))
        self._h = h

    def execute(self, d_ins, d_outs, stream: int = 0):
        n = len(self.plans)
        ins = (ctypes.c_void_p * n)(*d_ins)
        outs = (ctypes.c_void_p * n)(*d_outs)
        _check(lib.ffs_batch_execute(self._h, ins, outs, ctypes.c_void_p(stream)))

    def status(self) -> int:
        st = ctypes.c_int()
        _check(lib.ffs_batch_status(self._h, ctypes.byref(st)))
        return st.value

    def close(self):
        if getattr(self, "_h", None):
            lib.ffs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
