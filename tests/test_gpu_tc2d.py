"""GPU parity of the tcgen05 2-D forms against the CPU oracle:
Ozaki INT8 slices (FP64-level: max|y-r|/max|r| <= 1e-12 at 7-8 slices) and the
3-way BF16 split (24-bit operands, short FP32 accumulations summed in FP64: four
K = 128 GEMM stages measure ~5e-7 normwise, tolerance 2e-6)."""
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
    ("Box2D9P", (512, 512), 32, "fixed"),
    ("Box2D9P", (300, 257), 17, "periodic"),
    ("Box2D25P", (200, 190), 12, "fixed"),
    ("Star2D9P", (130, 140), 5, "periodic"),
    ("Heat-2D", (10, 9), 4, "periodic"),
    ("Box2D9P", (275, 121), 15, "fixed"),       # odd width: every other row is 8-byte aligned
    ("Box2D25P", (301, 97), 9, "periodic"),
]


@pytest.mark.parametrize("shape,ext,T,bnd", CASES)
@pytest.mark.parametrize("slices", [7, 8])
def test_ozaki_fp64_level(shape, ext, T, bnd, slices):
    si = ffs.shape_info(shape)
    w = seeded_weights(2, si.radius, 3)
    plan = ffs.Plan(2, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form="ozaki", slices=slices)
    x = seeded_grid((ext[1], ext[0]), 41)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL_FP64, (mx, l2, plan.info)


def test_ozaki_error_decreases_with_slices():
    w = seeded_weights(2, 1, 5)
    x = seeded_grid((256, 256), 6)
    ref = oracle.run(x, w, 1, 16, oracle.FIXED)
    errs = []
    for s in range(4, 9):
        plan = ffs.Plan(2, None, (256, 256), 16, weights=w, radius=1, boundary="fixed", form="ozaki", slices=s)
        errs.append(rel_errors(run_gpu(plan, x), ref)[0])
    assert all(b < a for a, b in zip(errs[:3], errs[1:4])), errs  # 4 -> 7 slices: strictly better
    assert errs[3] <= TOL_FP64 and errs[4] <= TOL_FP64, errs


@pytest.mark.parametrize("shape,ext,T,bnd", CASES)
def test_bf16x3(shape, ext, T, bnd):
    si = ffs.shape_info(shape)
    w = seeded_weights(2, si.radius, 4)
    plan = ffs.Plan(2, None, ext, T, weights=w, radius=si.radius, boundary=bnd, form="bf16x3")
    x = seeded_grid((ext[1], ext[0]), 42)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL_BF16X3, (mx, l2, plan.info)


def test_bf16_two_way_split_is_coarser():
    w = seeded_weights(2, 1, 7)
    x = seeded_grid((256, 256), 8)
    ref = oracle.run(x, w, 1, 16, oracle.PERIODIC)
    e2 = rel_errors(run_gpu(ffs.Plan(2, None, (256, 256), 16, weights=w, radius=1, form="bf16x3", slices=2), x),
                    ref)[0]
    e3 = rel_errors(run_gpu(ffs.Plan(2, None, (256, 256), 16, weights=w, radius=1, form="bf16x3", slices=3), x),
                    ref)[0]
    assert e3 < e2 < 1e-3, (e2, e3)


def test_ozaki_bench_config():
    n = 4096
    x = seeded_grid((n, n), 20251203 + 1)
    w = seeded_weights(2, 1, 20251203 + 1)
    plan = ffs.Plan(2, None, (n, n), 32, weights=w, radius=1, boundary="fixed", form="ozaki")
    mx, l2 = rel_errors(run_gpu(plan, x), oracle.run(x, w, 1, 32, oracle.FIXED))
    assert mx <= TOL_FP64, (mx, l2)
