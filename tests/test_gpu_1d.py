"""GPU parity of the 1-D FP64-DMMA fused tile path (4096-point four-step tiles)
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
    ("Heat-1D", 100001, 40, "fixed", 0),        # odd length: the last in-grid cell is loaded plainly
    ("1D5P", 65537, 17, "fixed", 0),
])
def test_parity_1d(shape, n, T, bnd, tau):
    si = ffs.shape_info(shape)
    w = seeded_weights(1, si.radius, n % 97)
    if shape == "Heat-1D" and n == 1 << 20:
        w = si.weights  # (0.25, 0.5, 0.25)
    plan = ffs.Plan(1, None, (n,), T, weights=w, radius=si.radius, boundary=bnd, tau=tau)
    x = seeded_grid((n,), 31)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL, (mx, l2, plan.info)


def test_named_1d_shapes():
    for shape in ("Heat-1D", "1D5P", "1D7P"):
        si = ffs.shape_info(shape)
        plan = ffs.Plan(1, shape, (30000,), 25, boundary="fixed")
        x = seeded_grid((30000,), 2)
        assert rel_errors(run_gpu(plan, x), oracle.run(x, si.weights, si.radius, 25, oracle.FIXED))[0] <= TOL
