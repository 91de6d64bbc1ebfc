"""Host-side choice of the slab pipeline of ffs_execute_host (no GPU): the slab
count the plan builder reports in ffs_plan_info.host_slabs, its limits, and the
FFS_HOST_SLABS override."""
import pytest

import flashfftstencil_b200 as ffs


def slabs(dim, shape, ext, T, **kw):
    return ffs.describe(dim, shape, ext, T, **kw)["host_slabs"]


@pytest.fixture(autouse=True)
def _no_override(monkeypatch):
    monkeypatch.delenv("FFS_HOST_SLABS", raising=False)


def test_headline_grid_is_split():
    # 4096^2 doubles = 128 MiB each way: the copies dominate, so the grid is cut into slabs
    k = slabs(2, "Box2D9P", (4096, 4096), 32, boundary="fixed", form="fp64_fft")
    assert 2 <= k <= 16
    assert 4096 / k >= 4 * 32  # slabs at least 4 r T rows


@pytest.mark.parametrize("dim,shape,ext,T", [
    (3, "Box3D27P", (512, 512, 512), 16),
    (2, "Box2D25P", (8192, 8192), 128),
    (2, "Box2D9P", (8192, 8192), 32),
])
def test_large_grids_are_split_within_limits(dim, shape, ext, T):
    r = ffs.shape_info(shape).radius
    k = slabs(dim, shape, ext, T, boundary="fixed")
    assert 2 <= k <= 16
    n = ext[dim - 1]
    h = -(-n // k)
    assert h >= 4 * r * T
    row_bytes = 8
    for e in ext[: dim - 1]:
        row_bytes *= e
    assert h * row_bytes >= 4 << 20


@pytest.mark.parametrize("dim,shape,ext,kw", [
    (1, "Heat-1D", (1 << 20,), {}),                           # 1-D grids are copied whole
    (2, "Box2D9P", (256, 256), {}),                           # slabs would be under 4 MiB
    (2, "Box2D9P", (4095, 4096), {}),                         # odd rows: views off 16-byte boundaries
    (2, "Box2D9P", (4096, 4096), {"open_faces": 0b1100}),     # a plan that is itself a slab
    (2, "Box2D9P", (4096, 200), {}),                          # two slabs would be under 4 r T rows
])
def test_whole_grid_cases(dim, shape, ext, kw):
    assert slabs(dim, shape, ext, 32, boundary="fixed", **kw) == 1


def test_override(monkeypatch):
    monkeypatch.setenv("FFS_HOST_SLABS", "1")
    assert slabs(2, "Box2D9P", (4096, 4096), 32, boundary="fixed") == 1
    monkeypatch.setenv("FFS_HOST_SLABS", "5")
    assert slabs(2, "Box2D9P", (256, 200), 8, boundary="fixed") == 5
    assert slabs(3, "Box3D27P", (40, 36, 48), 4, boundary="periodic") == 5
    # 100 rows in slabs of ceil(100 / 7) = 15 rows -> 7 slabs; 64 rows / 6 -> 11-row slabs -> 6
    monkeypatch.setenv("FFS_HOST_SLABS", "7")
    assert slabs(2, "Box2D9P", (64, 100), 8, boundary="fixed") == 7
    monkeypatch.setenv("FFS_HOST_SLABS", "6")
    assert slabs(2, "Box2D9P", (64, 64), 8, boundary="fixed") == 6
    # the override does not apply where slabs are not supported
    assert slabs(1, "Heat-1D", (4096,), 8, boundary="fixed") == 1
    assert slabs(2, "Box2D9P", (75, 60), 8, boundary="fixed") == 1


def test_many_grids_model_prefers_whole_for_compute_bound():
    """The model is per grid; for many grids ffs_execute_host_many compares both pipelines
    with the same model.  Box2D25P 8192^2 T=128 is compute-bound: its slab count stays
    small so the ghost rows cost at most half the stepped rows."""
    k = slabs(2, "Box2D25P", (8192, 8192), 128, boundary="fixed")
    assert k <= 8192 // (4 * 2 * 128)


@pytest.mark.parametrize("shape", ["Heat-2D", "Box2D9P", "Star2D9P", "Box2D25P", "Heat-3D", "Box3D27P"])
@pytest.mark.parametrize("bnd", ["fixed", "periodic"])
def test_every_shape_gets_slabs_on_a_large_grid(shape, bnd):
    """The slab sub-problems (open cut faces for a fixed boundary, a taller periodic grid for a
    periodic one) validate for every named 2D/3D shape, so large grids are pipelined in slabs."""
    si = ffs.shape_info(shape)
    ext = (4096, 4096) if si.dim == 2 else (384, 384, 384)
    k = slabs(si.dim, shape, ext, 16, boundary=bnd)
    assert 2 <= k <= 16, (shape, bnd, k)
    assert -(-ext[-1] // k) >= 4 * si.radius * 16


@pytest.mark.parametrize("form", ["fp64", "fp64_fft", "ozaki", "bf16x3"])
def test_slab_model_keeps_the_form(monkeypatch, form):
    """The sub-plans take the parent's resolved form, slices and tau: forcing slabs on every form
    validates (the describe path builds the same sub-problems the host path creates)."""
    monkeypatch.setenv("FFS_HOST_SLABS", "4")
    kw = {"slices": 7} if form == "ozaki" else {}
    assert slabs(2, "Box2D9P", (512, 512), 8, boundary="fixed", form=form, **kw) == 4
    assert slabs(3, "Box3D27P", (64, 64, 64), 4, boundary="periodic", form=form, **kw) == 4
