"""GPU parity of the slab pipeline of ffs_execute_host / ffs_execute_host_many: the
grid is cut along its slowest axis, each slab stepped with r*T ghost rows by a
sub-plan whose cut faces are open, and only slab interiors are copied back.
Results against the CPU oracle: max|y-r|/max|r| <= 1e-12 for the FP64 forms,
the tensor-core forms at their own bounds."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu
TOL = 1e-12
TOL_FORM = {"fp64_fft": TOL, "fp64": TOL, "ozaki": TOL, "bf16x3": 1e-5}  # Ozaki at 7 slices
TOL_FORM["fp64_fft128"] = TOL  # the butterfly form on its 128 x 128 edge

CASES = [
    # dim, shape, extents (x fastest), T, boundary, form, forced slab count
    (2, "Box2D9P", (256, 200), 8, "fixed", "fp64_fft", 3),
    (2, "Box2D9P", (200, 256), 12, "periodic", "fp64_fft", 4),    # end slabs wrap
    (2, "Box2D9P", (128, 96), 16, "fixed", "fp64_fft", 6),        # ghosts as tall as a slab: clipped faces
    (2, "Box2D9P", (64, 40), 24, "periodic", "fp64_fft", 2),      # ghosts longer than the grid: rows repeat
    (2, "Box2D25P", (180, 150), 7, "fixed", "fp64_fft", 3),
    (2, "Star2D9P", (130, 140), 5, "periodic", "fp64_fft", 5),
    (2, "Box2D9P", (256, 256), 10, "fixed", "fp64", 4),
    (2, "Box2D9P", (600, 700), 24, "fixed", "fp64_fft128", 3),  # 128 x 128 tiles on the slabs
    (2, "Box2D9P", (520, 480), 18, "periodic", "fp64_fft128", 4),
    (2, "Box2D9P", (192, 160), 9, "periodic", "fp64", 3),
    (2, "Box2D9P", (256, 192), 8, "fixed", "ozaki", 3),
    (2, "Box2D9P", (256, 192), 8, "periodic", "bf16x3", 3),
    (3, "Box3D27P", (40, 36, 48), 4, "fixed", "fp64_fft", 3),
    (3, "Heat-3D", (32, 32, 40), 6, "periodic", "fp64_fft", 5),
    (3, "Box3D27P", (48, 48, 48), 4, "fixed", "fp64", 4),
    (3, "Box3D27P", (36, 40, 44), 3, "periodic", "fp64", 2),
]


def grid_shape(ext):
    return tuple(reversed(ext))


@pytest.mark.parametrize("dim,shape,ext,T,bnd,form,k", CASES)
def test_forced_slabs_match_oracle(monkeypatch, dim, shape, ext, T, bnd, form, k):
    monkeypatch.setenv("FFS_HOST_SLABS", str(k))
    si = ffs.shape_info(shape)
    w = seeded_weights(dim, si.radius, 11 + k)
    tile = 128 if form == "fp64_fft128" else 0
    form = "fp64_fft" if form == "fp64_fft128" else form
    plan = ffs.Plan(dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form=form, tile=tile)
    assert plan.info["host_slabs"] == k
    x = seeded_grid(grid_shape(ext), 70 + k)
    got = plan.run_host(x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL_FORM[form], (mx, l2, plan.info)
    # a second call reuses the sub-plans and buffers
    x2 = seeded_grid(grid_shape(ext), 90 + k)
    got2 = plan.run_host(x2)
    ref2 = oracle.run(x2, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    assert rel_errors(got2, ref2)[0] <= TOL_FORM[form]


@pytest.mark.parametrize("bnd", ["fixed", "periodic"])
def test_slabs_across_many_grids(monkeypatch, bnd):
    """Five grids through ffs_execute_host_many on slabs: both input slots and all
    three output ring slots are reused."""
    import torch
    monkeypatch.setenv("FFS_HOST_SLABS", "3")
    plan = ffs.Plan(2, "Box2D9P", (260, 190), 11, boundary=bnd, form="fp64_fft")
    assert plan.info["host_slabs"] == 3
    xs = [torch.from_numpy(seeded_grid((190, 260), 140 + i)).pin_memory().numpy() for i in range(5)]
    outs = [torch.empty((190, 260), dtype=torch.float64).pin_memory().numpy() for _ in range(5)]
    plan.run_host_many(xs, outs)
    b = oracle.FIXED if bnd == "fixed" else oracle.PERIODIC
    for x, o in zip(xs, outs):
        assert rel_errors(o, oracle.run(x, ffs.shape_info("Box2D9P").weights, 1, 11, b))[0] <= TOL


def test_headline_size_auto_slabs_match_device_path(monkeypatch):
    """The model's own choice on Box2D9P 4096^2 T=32: the host path on slabs agrees
    with the device path on the whole grid to rounding (different tile anchors)."""
    import torch
    monkeypatch.delenv("FFS_HOST_SLABS", raising=False)
    plan = ffs.Plan(2, "Box2D9P", (4096, 4096), 32, boundary="fixed", form="fp64_fft")
    assert plan.info["host_slabs"] > 1
    x = torch.from_numpy(seeded_grid((4096, 4096), 5)).pin_memory()
    host = plan.run_host(x.numpy())
    dev = plan.run(x.cuda())
    torch.cuda.synchronize()
    d = dev.cpu().numpy()
    assert np.abs(host - d).max() / np.abs(d).max() <= 1e-13


def test_whole_grid_override_still_works(monkeypatch):
    monkeypatch.setenv("FFS_HOST_SLABS", "1")
    plan = ffs.Plan(2, "Box2D9P", (256, 200), 8, boundary="fixed", form="fp64_fft")
    assert plan.info["host_slabs"] == 1
    x = seeded_grid((200, 256), 3)
    assert rel_errors(plan.run_host(x), oracle.run(x, ffs.shape_info("Box2D9P").weights, 1, 8,
                                                   oracle.FIXED))[0] <= TOL


@pytest.mark.parametrize("bnd", ["fixed", "periodic"])
def test_slabs_keep_the_32_tile(monkeypatch, bnd):
    """A 3D butterfly plan on the 32^3 cluster tile through the slab pipeline: the sub-plans take
    the whole grid's tile edge and fused step count."""
    monkeypatch.setenv("FFS_HOST_SLABS", "3")
    w = seeded_weights(3, 1, 61)
    ext = (70, 64, 96)
    plan = ffs.Plan(3, None, ext, 9, weights=w, radius=1, boundary=bnd, form="fp64_fft", tile=32, tau=3)
    assert plan.info["host_slabs"] == 3 and plan.info["tile"] == 32
    x = seeded_grid(grid_shape(ext), 62)
    ref = oracle.run(x, w, 1, 9, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    assert rel_errors(plan.run_host(x), ref)[0] <= TOL
