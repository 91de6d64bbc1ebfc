"""GPU parity of the 1-D FP64 butterfly form (fp64_fft: four-step DFT-4096 of radix-8 lines)
against the CPU oracle.  Tolerance: max|y-r|/max|r| <= 1e-12."""
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


@pytest.mark.parametrize("shape,n,T,bnd,tau", [
    ("Heat-1D", 1 << 20, 64, "fixed", 0),       # the Heat-1D benchmark configuration
    ("Heat-1D", 100003, 33, "periodic", 0),
    ("1D5P", 20000, 100, "fixed", 0),
    ("1D7P", 12345, 9, "periodic", 0),
    ("1D7P", 777, 5, "fixed", 0),               # smaller than one tile
    ("Heat-1D", 50000, 20, "periodic", 3),      # many passes
    ("1D5P", 4096 * 3, 1, "fixed", 0),
    ("Heat-1D", 100001, 40, "fixed", 0),        # odd length
    ("1D5P", 65537, 17, "fixed", 0),
])
def test_parity_1d(shape, n, T, bnd, tau):
    si = ffs.shape_info(shape)
    w = seeded_weights(1, si.radius, n % 997)
    plan = ffs.Plan(1, None, (n,), T, weights=w, radius=si.radius, boundary=bnd, tau=tau, form="fp64_fft")
    assert plan.info["form"] == "fp64_fft"
    x = seeded_grid((n,), 11)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL, (mx, l2, plan.info)


@pytest.mark.parametrize("tau", [1, 16, 64])
def test_matches_dmma_form(tau):
    w = seeded_weights(1, 2, 5)
    x = seeded_grid((300000,), 6)
    a = run_gpu(ffs.Plan(1, None, (300000,), 64, weights=w, radius=2, boundary="fixed", tau=tau), x)
    b = run_gpu(ffs.Plan(1, None, (300000,), 64, weights=w, radius=2, boundary="fixed", tau=tau,
                         form="fp64_fft"), x)
    assert np.abs(a - b).max() / np.abs(a).max() <= 1e-13


def test_single_tile_lone_partner():
    """An odd number of tiles leaves the last pair without its second tile: the partner plane
    is not copied and must read as zeros, not whatever the stage held."""
    w = seeded_weights(1, 1, 8)
    for n in (3 * 4000, 5 * 4000 + 17):
        plan = ffs.Plan(1, None, (n,), 30, weights=w, radius=1, boundary="periodic", form="fp64_fft")
        x = seeded_grid((n,), n)
        got = run_gpu(plan, x)
        assert np.isfinite(got).all()
        assert rel_errors(got, oracle.run(x, w, 1, 30, oracle.PERIODIC))[0] <= TOL
