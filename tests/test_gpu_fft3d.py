"""GPU parity of the 3-D FP64 butterfly form (fp64_fft: one DFT per thread and line) against the
CPU oracle, on both tile edges: 16^3 (one CTA per tile pair, radix-4 x 4) and 32^3 (a cluster
of four CTAs per pair in distributed shared memory, radix-4 x 8).  Tolerance:
max|y-r|/max|r| <= 1e-12."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run_gpu(plan, x):
    import torch
    out = plan.run(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("tile", [16, 32])
@pytest.mark.parametrize("shape,ext,T,bnd,tau", [
    ("Box3D27P", (64, 64, 64), 16, "fixed", 0),
    ("Box3D27P", (50, 41, 37), 7, "periodic", 0),   # odd sizes, edge tiles wrap
    ("Heat-3D", (96, 80, 40), 9, "fixed", 0),
    ("Heat-3D", (10, 12, 9), 4, "periodic", 0),     # smaller than one tile
    ("Box3D27P", (48, 48, 48), 5, "periodic", 1),
    ("Box3D27P", (34, 30, 66), 8, "fixed", 3),
    ("Box3D27P", (33, 31, 35), 6, "fixed", 0),      # odd width: scalar loads
    ("Box3D27P", (70, 45, 52), 13, "periodic", 6),  # 32^3: halo 6, 20^3 kept
    ("Heat-3D", (57, 66, 40), 12, "fixed", 4),      # 32^3: halo 4, 24^3 kept, two passes
])
def test_parity_3d(shape, ext, T, bnd, tau, tile):
    si = ffs.shape_info(shape)
    w = seeded_weights(3, si.radius, ext[0])
    plan = ffs.Plan(3, None, ext, T, weights=w, radius=si.radius, boundary=bnd, tau=tau, form="fp64_fft",
                    tile=tile)
    assert plan.info["form"] == "fp64_fft" and plan.info["tile"] == tile
    x = seeded_grid((ext[2], ext[1], ext[0]), 17)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL, (mx, l2, plan.info)


@pytest.mark.parametrize("tile", [16, 32])
def test_radius_two_custom(tile):
    w = np.random.default_rng(3).random((5, 5, 5))
    w /= w.sum()
    ext = (70, 36, 40)
    plan = ffs.Plan(3, None, ext, 5, weights=w, radius=2, boundary="periodic", form="fp64_fft", tile=tile)
    x = seeded_grid((ext[2], ext[1], ext[0]), 5)
    assert rel_errors(run_gpu(plan, x), oracle.run(x, w, 2, 5, oracle.PERIODIC))[0] <= TOL


@pytest.mark.parametrize("tau", [1, 2, 3])
def test_matches_dmma_form(tau):
    w = seeded_weights(3, 1, 9)
    x = seeded_grid((64, 72, 80), 10)
    a = run_gpu(ffs.Plan(3, None, (80, 72, 64), 12, weights=w, radius=1, boundary="fixed", tau=tau), x)
    b = run_gpu(ffs.Plan(3, None, (80, 72, 64), 12, weights=w, radius=1, boundary="fixed", tau=tau,
                         form="fp64_fft"), x)
    assert np.abs(a - b).max() / np.abs(a).max() <= 1e-13


@pytest.mark.parametrize("tile", [16, 32])
def test_box3d27p_512_full_size(tile):
    """Box3D27P 512^3 fixed shell, T = 16 (the 3-D target configuration)."""
    n = 512
    x = seeded_grid((n, n, n), 20251203 + 2)
    w = seeded_weights(3, 1, 20251203 + 2)
    plan = ffs.Plan(3, None, (n, n, n), 16, weights=w, radius=1, boundary="fixed", form="fp64_fft", tile=tile)
    mx, l2 = rel_errors(run_gpu(plan, x), oracle.run(x, w, 1, 16, oracle.FIXED))
    assert mx <= TOL, (mx, l2, plan.info)


@pytest.mark.parametrize("bnd", ["fixed", "periodic"])
def test_tiles_agree(bnd):
    """The two tile edges solve the same problem to within rounding."""
    w = seeded_weights(3, 1, 31)
    x = seeded_grid((90, 100, 110), 32)
    a = run_gpu(ffs.Plan(3, None, (110, 100, 90), 16, weights=w, radius=1, boundary=bnd, form="fp64_fft",
                         tile=16), x)
    b = run_gpu(ffs.Plan(3, None, (110, 100, 90), 16, weights=w, radius=1, boundary=bnd, form="fp64_fft",
                         tile=32), x)
    assert np.abs(a - b).max() / np.abs(a).max() <= 1e-13
