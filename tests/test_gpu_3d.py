"""GPU parity of the 3-D FP64-DMMA fused tile path (16^3 tiles, radix-4 x 4
DFT-16 per axis) against the CPU oracle.  Tolerance: max|y-r|/max|r| <= 1e-12."""
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


@pytest.mark.parametrize("shape,ext,T,bnd,tau", [
    ("Box3D27P", (64, 64, 64), 16, "fixed", 0),
    ("Box3D27P", (50, 41, 37), 7, "periodic", 0),   # odd sizes, edge tiles wrap
    ("Heat-3D", (96, 80, 40), 9, "fixed", 0),
    ("Heat-3D", (10, 12, 9), 4, "periodic", 0),     # smaller than one tile
    ("Box3D27P", (48, 48, 48), 5, "periodic", 1),
    ("Box3D27P", (34, 30, 66), 8, "fixed", 3),
])
def test_parity_3d(shape, ext, T, bnd, tau):
    si = ffs.shape_info(shape)
    w = seeded_weights(3, si.radius, ext[0])
    plan = ffs.Plan(3, None, ext, T, weights=w, radius=si.radius, boundary=bnd, tau=tau)
    x = seeded_grid((ext[2], ext[1], ext[0]), 17)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL, (mx, l2, plan.info)


def test_named_3d_shapes():
    for shape in ("Heat-3D", "Box3D27P"):
        si = ffs.shape_info(shape)
        plan = ffs.Plan(3, shape, (40, 40, 40), 6, boundary="fixed")
        x = seeded_grid((40, 40, 40), 4)
        assert rel_errors(run_gpu(plan, x), oracle.run(x, si.weights, 1, 6, oracle.FIXED))[0] <= TOL


def test_box3d27p_512_full_size():
    """Box3D27P 512^3 fixed shell, T = 16 (the 3-D target configuration)."""
    n = 512
    x = seeded_grid((n, n, n), 20251203 + 2)
    w = seeded_weights(3, 1, 20251203 + 2)
    plan = ffs.Plan(3, None, (n, n, n), 16, weights=w, radius=1, boundary="fixed")
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, 1, 16, oracle.FIXED)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL, (mx, l2)
