"""C-ABI checks that need no GPU: the library loads, exports every symbol that
include/ffs.h declares, validates problems with status codes (never exits), and
plans sensible tile geometry."""
import ctypes
import os
import re

import numpy as np
import pytest

import flashfftstencil_b200 as ffs

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "ffs.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(ffs_\w+)\s*\(", src, re.M)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert "ffs_plan_create" in names and len(names) >= 10
    for n in names:
        assert hasattr(ffs.lib, n), n
    assert set(names) == set(ffs.EXPORTS)


def test_abi_version():
    assert ffs.lib.ffs_abi_version() == 4


def test_shape_table():
    expect = {"Heat-1D": (1, 1, "1d1r"), "1D5P": (1, 2, "1d2r"), "1D7P": (1, 3, "1d3r"),
              "Heat-2D": (2, 1, "star_2d1r"), "Box2D9P": (2, 1, "box_2d1r"), "Star2D9P": (2, 2, "star_2d2r"),
              "Box2D25P": (2, 2, "box_2d2r"), "Heat-3D": (3, 1, "star_3d1r"), "Box3D27P": (3, 1, "box_3d1r")}
    for name, (dim, r, label) in expect.items():
        si = ffs.shape_info(name)
        assert (si.dim, si.radius, si.label) == (dim, r, label)
        assert si.weights.size == (2 * r + 1) ** dim
        assert abs(si.weights.sum() - 1.0) < 1e-14
    np.testing.assert_array_equal(ffs.shape_info("Heat-1D").weights, [0.25, 0.5, 0.25])
    # reference spelling in its README ("Box3d27P") is accepted too
    assert ffs.shape_info("Box3d27P").dim == 3
    with pytest.raises(ffs.FFSError) as e:
        ffs.shape_info("Hex-2D")
    assert e.value.status == ffs.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("kw,status", [
    (dict(dim=4, shape=None, extents=(8,), T=1, weights=np.ones(1), radius=0), ffs.ERR_INVALID_ARGUMENT),
    (dict(dim=2, shape="Box2D9P", extents=(0, 8), T=1), ffs.ERR_INVALID_ARGUMENT),
    (dict(dim=2, shape="Box2D9P", extents=(8, 8), T=-1), ffs.ERR_INVALID_ARGUMENT),
    (dict(dim=2, shape="Box2D9P", extents=(8, 8, 3), T=1), ffs.ERR_INVALID_ARGUMENT),
    (dict(dim=2, shape=None, extents=(8, 8), T=1, weights=np.ones(9), radius=9), ffs.ERR_INVALID_ARGUMENT),
    (dict(dim=2, shape=None, extents=(8, 8), T=1, weights=np.array([np.nan] * 9), radius=1),
     ffs.ERR_INVALID_ARGUMENT),
    (dict(dim=2, shape="Box2D9P", extents=(8, 8), T=1, tau=-2), ffs.ERR_INVALID_ARGUMENT),
    (dict(dim=2, shape="Box2D9P", extents=(8, 8), T=1, form="fp64_fft", slices=4), ffs.ERR_INVALID_ARGUMENT),
])
def test_validation_status_codes(kw, status):
    with pytest.raises(ffs.FFSError) as e:
        ffs.describe(**kw)
    assert e.value.status == status
    assert ffs.lib.ffs_last_error_string().decode() != ""


def test_form_selection():
    """auto picks the fastest FP64-exact form, the butterfly kernels, in every dimension;
    the butterfly form shares the DMMA form's tile geometry."""
    assert ffs.describe(2, "Box2D9P", (300, 200), 16, form="auto")["form"] == "fp64_fft"
    assert ffs.describe(1, "Heat-1D", (5000,), 16, form="auto")["form"] == "fp64_fft"
    assert ffs.describe(3, "Heat-3D", (40, 40, 40), 4, form="auto")["form"] == "fp64_fft"
    a = ffs.describe(2, "Box2D25P", (500, 300), 24, boundary="fixed", tau=6)
    b = ffs.describe(2, "Box2D25P", (500, 300), 24, boundary="fixed", tau=6, form="fp64_fft")
    for key in ("tile", "halo", "useful", "tau", "passes", "tiles", "hbm_bytes_per_pass", "flops_per_pass"):
        assert a[key] == b[key], key
    assert b["exec_flops_per_pass"] < a["exec_flops_per_pass"] / 3


def test_reserved_must_be_zero():
    p, _k = ffs._make_problem(2, "Box2D9P", (16, 16), 3)
    p.reserved[3] = 1
    info = ffs._Info()
    assert ffs.lib.ffs_plan_describe(ctypes.byref(p), ctypes.byref(info)) == ffs.ERR_INVALID_ARGUMENT


def test_open_faces_validation_and_geometry():
    base = ffs.describe(2, "Box2D9P", (300, 200), 16, boundary="fixed", tau=8)
    cut = ffs.describe(2, "Box2D9P", (300, 200), 16, boundary="fixed", tau=8, open_faces=0b1100)
    assert cut["tiles"] > base["tiles"]  # the tile path now reaches the open (y) faces
    with pytest.raises(ffs.FFSError):
        ffs.describe(2, "Box2D9P", (300, 200), 16, boundary="fixed", open_faces=1 << 4)  # no z faces in 2-D
    with pytest.raises(ffs.FFSError):
        ffs.describe(1, "Heat-1D", (300,), 16, boundary="fixed", open_faces=-1)


def test_null_arguments_return_codes():
    assert ffs.lib.ffs_plan_describe(None, None) == ffs.ERR_INVALID_ARGUMENT
    assert ffs.lib.ffs_plan_create(None, None) == ffs.ERR_INVALID_ARGUMENT
    assert ffs.lib.ffs_execute(None, None, None, None) == ffs.ERR_INVALID_ARGUMENT
    assert ffs.lib.ffs_execute_host(None, None, None, None) == ffs.ERR_INVALID_ARGUMENT
    assert ffs.lib.ffs_execute_host_many(None, 1, None, None, None) == ffs.ERR_INVALID_ARGUMENT
    assert ffs.lib.ffs_plan_destroy(None) == ffs.OK
    assert ffs.lib.ffs_batch_destroy(None) == ffs.OK


@pytest.mark.parametrize("shape,ext,T,bnd", [
    ("Box2D9P", (4096, 4096), 32, "fixed"), ("Box2D25P", (8192, 8192), 128, "periodic"),
    ("Heat-2D", (100, 37), 3, "fixed"), ("Star2D9P", (64, 64), 1, "periodic"), ("Box2D9P", (8192, 8192), 32, "fixed"),
])
def test_geometry_invariants(shape, ext, T, bnd):
    info = ffs.describe(2, shape, ext, T, boundary=bnd)
    r = info["radius"]
    assert info["halo"] % 2 == 0 and info["halo"] >= r * info["tau"]
    assert info["useful"] == info["tile"] - 2 * info["halo"] >= 8
    assert (info["passes"] - 1) * info["tau"] + info["tau_last"] == T
    assert 1 <= info["tau_last"] <= info["tau"]


def test_tau_override_and_zero_steps():
    info = ffs.describe(2, "Box2D9P", (256, 256), 20, tau=3)
    assert info["tau"] == 3 and info["passes"] == 7 and info["tau_last"] == 2
    info0 = ffs.describe(2, "Box2D9P", (256, 256), 0)
    assert info0["passes"] == 0


def test_noalloc_form_check_needs_no_device():
    """ffs_execute_noalloc runs the DMMA form only: another explicit form is refused before any
    device work (auto resolves to DMMA there; its acceptance is covered by the GPU test)."""
    import ctypes
    p, _keep = ffs._make_problem(2, "Box2D9P", (64, 64), 4, form="fp64_fft")
    st = ffs.lib.ffs_execute_noalloc(ctypes.byref(p), ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert st == ffs.ERR_UNSUPPORTED
    assert "FP64-DMMA" in ffs.lib.ffs_last_error_string().decode()


def test_noalloc_status_rejects_a_null_pointer():
    """ffs_noalloc_status checks its argument before touching a device."""
    assert ffs.lib.ffs_noalloc_status(None) == ffs.ERR_INVALID_ARGUMENT
    assert "null argument" in ffs.lib.ffs_last_error_string().decode()


def test_create_plan_defaults_to_the_fastest_form():
    """The reference-named constructor builds the butterfly form unless asked otherwise."""
    import inspect
    assert inspect.signature(ffs.CreatePlan).parameters["form"].default == "auto"
    assert ffs.describe(2, None, (300, 300), 8, weights=np.full((3, 3), 1 / 9), radius=1, form="auto")["form"] == "fp64_fft"


def test_plan_info_carries_the_cost_model_estimate():
    """ffs_plan_info.model_ms (ABI 3): the plan builder's modelled time of one execute; zero
    work models to zero, and a grid with four times the cells models to more."""
    small = ffs.describe(2, "Box2D9P", (1024, 1024), 32, boundary="fixed", form="fp64_fft")
    large = ffs.describe(2, "Box2D9P", (2048, 2048), 32, boundary="fixed", form="fp64_fft")
    none = ffs.describe(2, "Box2D9P", (1024, 1024), 0, boundary="fixed", form="fp64_fft")
    assert small["model_ms"] > 0 and large["model_ms"] > 2 * small["model_ms"]
    assert none["model_ms"] == 0


def test_tile_edge_request():
    """ffs_problem.tile (ABI 4): 0 lets the plan builder choose; the 3D FP64 butterfly form
    takes 16 or 32, every other form only its one edge (refused before any device work)."""
    for tile in (16, 32):
        info = ffs.describe(3, "Box3D27P", (100, 90, 80), 12, boundary="fixed", form="fp64_fft", tile=tile)
        assert info["tile"] == tile
        assert info["useful"] == tile - 2 * info["halo"] and info["halo"] >= info["tau"]
    assert ffs.describe(3, "Box3D27P", (100, 90, 80), 12, form="fp64_fft")["tile"] in (16, 32)
    assert ffs.describe(3, "Box3D27P", (100, 90, 80), 12, form="fp64", tile=16)["tile"] == 16
    assert ffs.describe(2, "Box2D9P", (256, 256), 8, form="fp64_fft", tile=64)["tile"] == 64
    info = ffs.describe(2, "Box2D9P", (1000, 900), 30, boundary="fixed", form="fp64_fft", tile=128)
    assert info["tile"] == 128 and info["useful"] == 128 - 2 * info["halo"]
    assert info["tiles"] == -(-1000 // info["useful"]) * -(-900 // info["useful"])  # single tiles, not pairs
    for dim, shape, ext, form, tile in [(3, "Box3D27P", (64, 64, 64), "fp64", 32), (3, "Box3D27P", (64, 64, 64), "ozaki", 32),
                                        (2, "Box2D9P", (256, 256), "fp64_fft", 32), (1, "Heat-1D", (4096,), "fp64_fft", 64),
                                        (2, "Box2D9P", (256, 256), "fp64", 128), (2, "Box2D9P", (256, 256), "ozaki", 128),
                                        (3, "Box3D27P", (64, 64, 64), "fp64_fft", 8)]:
        with pytest.raises(ffs.FFSError) as e:
            ffs.describe(dim, shape, ext, 4, form=form, tile=tile)
        assert e.value.status == ffs.ERR_UNSUPPORTED


def test_tile_32_lines_up_with_the_model():
    """The 32^3 tile's pair count and plan-info flops follow its geometry: a pass keeps u^3
    cells per tile, and the butterflies per pair are ~8-10x those of a 16^3 pair."""
    a = ffs.describe(3, "Box3D27P", (240, 240, 240), 8, boundary="periodic", form="fp64_fft", tile=16, tau=2)
    b = ffs.describe(3, "Box3D27P", (240, 240, 240), 8, boundary="periodic", form="fp64_fft", tile=32, tau=2)
    assert (a["useful"], b["useful"]) == (12, 28)
    assert a["tiles"] == 20 ** 3          # 20 tiles of 12 per axis, 10 pairs along x
    assert b["tiles"] == 2 * 5 * 9 * 9    # ceil(240 / 28) = 9 per axis, 5 pairs along x
    per_pair_a = a["exec_flops_per_pass"] / (a["tiles"] / 2)
    per_pair_b = b["exec_flops_per_pass"] / (b["tiles"] / 2)
    assert 7 < per_pair_b / per_pair_a < 12
