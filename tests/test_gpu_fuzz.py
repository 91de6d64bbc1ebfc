"""Seeded random problems across every dimension, shape, boundary and form,
checked against the CPU oracle (FP64 and Ozaki 8 slices: max|y-r|/max|r| <=
1e-12; 3-way BF16: <= 1e-5).  Sizes are small and irregular (odd extents,
grids smaller than a tile, tiles straddling every face) so that the oracle
finishes in well under a second per case."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors

pytestmark = pytest.mark.gpu

SHAPES = {1: ["Heat-1D", "1D5P", "1D7P"], 2: ["Heat-2D", "Box2D9P", "Star2D9P", "Box2D25P"],
          3: ["Heat-3D", "Box3D27P"]}


def make_case(k):
    rng = np.random.default_rng(1000 + k)
    dim = int(rng.integers(1, 4))
    custom = rng.random() < 0.3
    if custom:
        r = int(rng.integers(1, 3 if dim == 3 else 4))
        shape = None
    else:
        shape = str(rng.choice(SHAPES[dim]))
        r = ffs.shape_info(shape).radius
    if dim == 1:
        ext = (int(rng.integers(5, 30000)),)
    elif dim == 2:
        ext = tuple(int(v) for v in rng.integers(3, 400, size=2))
    else:
        ext = tuple(int(v) for v in rng.integers(3, 48, size=3))
    T = int(rng.integers(0, 40 if dim < 3 else 10))
    bnd = str(rng.choice(["fixed", "periodic"]))
    forms = ["fp64", "fp64_fft"] if dim == 1 else ["fp64", "fp64_fft", "ozaki", "bf16x3"]
    form = str(rng.choice(forms))
    tau = int(rng.integers(1, 6)) if rng.random() < 0.3 else 0
    w = rng.random((2 * r + 1,) * dim)
    w /= w.sum()
    return dim, shape, r, ext, T, bnd, form, tau, w


@pytest.mark.parametrize("k", range(40))
def test_random_problem_matches_oracle(k):
    import torch
    dim, shape, r, ext, T, bnd, form, tau, w = make_case(k)
    kw = dict(weights=w, radius=r, boundary=bnd, form=form, tau=tau)
    if form == "ozaki":
        kw["slices"] = 8
    try:
        plan = ffs.Plan(dim, None, ext, T, **kw)
    except ffs.FFSError as e:  # only a radius too large for the tile may be refused
        assert e.status == ffs.ERR_UNSUPPORTED, (k, str(e))
        return
    x = np.random.default_rng(k).random(tuple(reversed(ext)))
    y = plan.run(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    ref = oracle.run(x, w, r, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC) if T else x
    mx, l2 = rel_errors(y.cpu().numpy(), ref)
    tol = 1e-5 if form == "bf16x3" else 1e-12
    assert mx <= tol, (k, dim, shape, r, ext, T, bnd, form, tau, mx, plan.info)


UNALIGNED = [
    (1, (4099,), "fp64"), (1, (9001,), "fp64_fft"),
    (2, (256, 96), "fp64"), (2, (256, 96), "fp64_fft"), (2, (256, 96), "ozaki"), (2, (256, 96), "bf16x3"),
    (3, (40, 24, 20), "fp64"), (3, (40, 24, 20), "fp64_fft"), (3, (40, 24, 20), "ozaki"), (3, (40, 24, 20), "bf16x3"),
]


@pytest.mark.parametrize("dim,ext,form", UNALIGNED)
@pytest.mark.parametrize("bnd", ["fixed", "periodic"])
def test_eight_byte_aligned_pointers(dim, ext, form, bnd):
    """A C-ABI caller may pass grids that start on an 8-byte (not 16-byte) boundary:
    every form must then avoid 16-byte and bulk copies from them."""
    import torch
    r = 1
    w = np.random.default_rng(dim).random((2 * r + 1,) * dim)
    w /= w.sum()
    shape = tuple(reversed(ext))
    n = int(np.prod(shape))
    x = np.random.default_rng(7).random(shape)
    kw = dict(weights=w, radius=r, boundary=bnd, form=form)
    if form == "ozaki":
        kw["slices"] = 8
    plan = ffs.Plan(dim, None, ext, 6, **kw)
    src = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    dst = torch.zeros(n + 1, dtype=torch.float64, device="cuda")
    src[1:] = torch.from_numpy(x.ravel()).cuda()
    assert src[1:].data_ptr() % 16 == 8
    plan.execute(src[1:].data_ptr(), dst[1:].data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    y = dst[1:].cpu().numpy().reshape(shape)
    ref = oracle.run(x, w, r, 6, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, _ = rel_errors(y, ref)
    assert mx <= (1e-5 if form == "bf16x3" else 1e-12), (dim, ext, form, bnd, mx, plan.info)


def make_slab_case(k):
    rng = np.random.default_rng(5000 + k)
    dim = int(rng.integers(2, 4))
    r = int(rng.integers(1, 3))
    if dim == 2:
        ext = (2 * int(rng.integers(2, 150)), int(rng.integers(4, 300)))  # even rows: slab views aligned
    else:
        ext = (2 * int(rng.integers(2, 20)), int(rng.integers(3, 40)), int(rng.integers(4, 48)))
    T = int(rng.integers(1, 30 if dim == 2 else 8))
    bnd = str(rng.choice(["fixed", "periodic"]))
    form = str(rng.choice(["fp64", "fp64_fft", "fp64_fft", "ozaki", "bf16x3"]))
    slabs = int(rng.integers(2, 8))
    w = rng.random((2 * r + 1,) * dim)
    w /= w.sum()
    return dim, r, ext, T, bnd, form, slabs, w


@pytest.mark.parametrize("k", range(24))
def test_random_host_slabs_match_oracle(monkeypatch, k):
    """ffs_execute_host on a forced slab count (ghost rows r*T, open or wrapped cut faces),
    random sizes, boundaries and forms, against the oracle."""
    dim, r, ext, T, bnd, form, slabs, w = make_slab_case(k)
    monkeypatch.setenv("FFS_HOST_SLABS", str(slabs))
    kw = dict(weights=w, radius=r, boundary=bnd, form=form)
    if form == "ozaki":
        kw["slices"] = 8
    try:
        plan = ffs.Plan(dim, None, ext, T, **kw)
    except ffs.FFSError as e:
        assert e.status == ffs.ERR_UNSUPPORTED, (k, str(e))
        return
    assert plan.info["host_slabs"] > 1
    x = np.random.default_rng(k + 77).random(tuple(reversed(ext)))
    y = plan.run_host(x)
    ref = oracle.run(x, w, r, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, _ = rel_errors(y, ref)
    assert mx <= (1e-5 if form == "bf16x3" else 1e-12), (k, dim, r, ext, T, bnd, form, slabs, mx, plan.info)


def make_edge_case(k):
    """A seeded problem for the butterfly form's second tile edges: 2D on 128 x 128 tiles
    (sizes from below one tile to several, ragged) or 3D on 32^3 cluster tiles."""
    rng = np.random.default_rng(5000 + k)
    dim = 2 if k % 3 else 3
    r = int(rng.integers(1, 4 if dim == 2 else 3))
    if dim == 2:
        ext = tuple(int(v) for v in rng.integers(20, 700, size=2))
        T = int(rng.integers(1, 60))
    else:
        ext = tuple(int(v) for v in rng.integers(10, 90, size=3))
        T = int(rng.integers(1, 14))
    bnd = str(rng.choice(["fixed", "periodic"]))
    tau = int(rng.integers(1, 12)) if rng.random() < 0.4 else 0
    w = rng.random((2 * r + 1,) * dim)
    w /= w.sum()
    return dim, r, ext, T, bnd, tau, w


@pytest.mark.parametrize("k", range(24))
def test_second_tile_edges_match_oracle(k):
    import torch
    dim, r, ext, T, bnd, tau, w = make_edge_case(k)
    tile = 128 if dim == 2 else 32
    try:
        plan = ffs.Plan(dim, None, ext, T, weights=w, radius=r, boundary=bnd, form="fp64_fft", tau=tau, tile=tile)
    except ffs.FFSError as e:  # only a radius too large for the tile may be refused
        assert e.status == ffs.ERR_UNSUPPORTED, (k, str(e))
        return
    assert plan.info["tile"] == tile
    x = np.random.default_rng(k + 77).random(tuple(reversed(ext)))
    y = plan.run(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    ref = oracle.run(x, w, r, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(y.cpu().numpy(), ref)
    assert mx <= 1e-12, (k, dim, r, ext, T, bnd, tau, mx, plan.info)


@pytest.mark.parametrize("dim,ext,tile", [(2, (300, 260), 128), (3, (40, 36, 34), 32)])
@pytest.mark.parametrize("bnd", ["fixed", "periodic"])
def test_second_tile_edges_on_eight_byte_aligned_pointers(dim, ext, tile, bnd):
    """The second tile edges read and write 8-byte words only: grids starting on an 8-byte
    boundary solve the same as aligned ones."""
    import torch
    r = 1
    w = np.random.default_rng(dim + 10).random((2 * r + 1,) * dim)
    w /= w.sum()
    T = 9 if dim == 2 else 4
    plan = ffs.Plan(dim, None, ext, T, weights=w, radius=r, boundary=bnd, form="fp64_fft", tile=tile)
    shape = tuple(reversed(ext))
    x = np.random.default_rng(3).random(shape)
    n = int(np.prod(shape))
    buf = torch.empty(n + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(x.ravel()).cuda()
    obuf = torch.empty(n + 1, dtype=torch.float64, device="cuda")
    plan.execute(buf.data_ptr() + 8, obuf.data_ptr() + 8, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    got = obuf[1:].cpu().numpy().reshape(shape)
    ref = oracle.run(x, w, r, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    assert rel_errors(got, ref)[0] <= 1e-12
