"""GPU parity of the tcgen05 3-D forms against the CPU oracle: Ozaki INT8 slices
(FP64 level, max|y-r|/max|r| <= 1e-12 at 7-8 slices; error falling with the slice
count) and the 3-way BF16 split (six K = 32 GEMM stages, short FP32 accumulations
summed in FP64, tolerance 2e-6)."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-12
TOL_BF16X3 = 2e-6


def run_gpu(plan, x):
    import torch
    out = plan.run(torch.from_numpy(x).cuda())
    torch.cuda.synchronize()
    return out.cpu().numpy()


CASES = [
    ("Box3D27P", (48, 40, 36), 8, "fixed"),
    ("Box3D27P", (33, 30, 29), 5, "periodic"),   # odd sizes, partial tile pairs
    ("Heat-3D", (40, 24, 50), 6, "fixed"),
    ("Heat-3D", (10, 9, 7), 3, "periodic"),      # grid smaller than one tile
]


def oracle_ref(x, w, r, T, bnd):
    return oracle.run(x, w, r, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)


@pytest.mark.parametrize("shape,ext,T,bnd", CASES)
@pytest.mark.parametrize("slices", [7, 8])
def test_ozaki_fp64_level(shape, ext, T, bnd, slices):
    si = ffs.shape_info(shape)
    w = seeded_weights(3, si.radius, 3)
    plan = ffs.Plan(3, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form="ozaki", slices=slices)
    x = seeded_grid(tuple(reversed(ext)), 41)
    mx, l2 = rel_errors(run_gpu(plan, x), oracle_ref(x, w, si.radius, T, bnd))
    assert mx <= TOL_FP64, (mx, l2, plan.info)


def test_ozaki_error_falls_with_slices():
    w = seeded_weights(3, 1, 5)
    ext = (64, 48, 40)
    x = seeded_grid(tuple(reversed(ext)), 6)
    ref = oracle_ref(x, w, 1, 8, "fixed")
    errs = []
    for s in range(4, 9):
        plan = ffs.Plan(3, None, ext, 8, weights=w, radius=1, boundary="fixed", form="ozaki", slices=s)
        errs.append(rel_errors(run_gpu(plan, x), ref)[0])
    assert all(b < a for a, b in zip(errs[:3], errs[1:4])), errs
    assert errs[3] <= TOL_FP64 and errs[4] <= TOL_FP64, errs


@pytest.mark.parametrize("shape,ext,T,bnd", CASES)
def test_bf16x3(shape, ext, T, bnd):
    si = ffs.shape_info(shape)
    w = seeded_weights(3, si.radius, 4)
    plan = ffs.Plan(3, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form="bf16x3")
    x = seeded_grid(tuple(reversed(ext)), 42)
    mx, l2 = rel_errors(run_gpu(plan, x), oracle_ref(x, w, si.radius, T, bnd))
    assert mx <= TOL_BF16X3, (mx, l2, plan.info)


def test_forms_agree_with_fp64_form():
    """Same problem through the FP64-DMMA and Ozaki forms: within both error bounds."""
    w = seeded_weights(3, 1, 9)
    ext = (40, 40, 40)
    x = seeded_grid((40, 40, 40), 10)
    a = run_gpu(ffs.Plan(3, None, ext, 6, weights=w, radius=1, boundary="periodic"), x)
    b = run_gpu(ffs.Plan(3, None, ext, 6, weights=w, radius=1, boundary="periodic", form="ozaki", slices=8), x)
    assert np.abs(a - b).max() / np.abs(a).max() <= 2 * TOL_FP64
