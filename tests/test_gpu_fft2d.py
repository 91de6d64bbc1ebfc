"""GPU parity of the 2-D FP64 butterfly form (fp64_fft) against the CPU oracle, through the
C ABI, on both tile edges: 64 x 64 (a pair of real tiles per complex tile, radix-8 DFT-64) and
128 x 128 (one real tile per CTA, two rows packed per complex FFT-128).  Tolerance:
max|y-r|/max|r| <= 1e-12, the same as the FP64-DMMA form it stands beside."""
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


CASES = [
    # shape, (nx, ny), T, boundary, tau
    ("Box2D9P", (512, 512), 32, "fixed", 0),
    ("Box2D9P", (300, 257), 17, "fixed", 0),     # odd height
    ("Box2D9P", (275, 121), 15, "fixed", 0),     # odd width: plain loads, no TMA
    ("Box2D9P", (256, 192), 9, "periodic", 0),
    ("Box2D25P", (200, 200), 12, "periodic", 0),
    ("Box2D25P", (222, 180), 7, "fixed", 0),
    ("Star2D9P", (130, 140), 5, "fixed", 0),
    ("Heat-2D", (10, 9), 4, "periodic", 0),      # grid smaller than one tile
    ("Heat-2D", (64, 64), 1, "fixed", 0),
    ("Box2D9P", (160, 96), 20, "periodic", 1),   # tau = 1, many passes
    ("Box2D9P", (97, 301), 6, "periodic", 0),
    ("Box2D9P", (700, 530), 40, "fixed", 20),    # 128 edge: halo 20, 88 kept per tile
    ("Box2D25P", (390, 333), 23, "periodic", 11),  # 128 edge: halo 22, two passes
]


@pytest.mark.parametrize("tile", [64, 128])
@pytest.mark.parametrize("shape,ext,T,bnd,tau", CASES)
def test_parity_random_weights(shape, ext, T, bnd, tau, tile):
    si = ffs.shape_info(shape)
    w = seeded_weights(2, si.radius, sum(map(ord, shape)))
    plan = ffs.Plan(2, None, ext, T, weights=w, radius=si.radius, boundary=bnd, tau=tau, form="fp64_fft",
                    tile=tile)
    assert plan.info["form"] == "fp64_fft" and plan.info["tile"] == tile
    x = seeded_grid((ext[1], ext[0]), 101)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL, (mx, l2, plan.info)


@pytest.mark.parametrize("tau", [2, 8, 12, 28])
def test_matches_dmma_form(tau):
    """Same plan geometry as the DMMA form: both forms agree to rounding at every tau."""
    w = seeded_weights(2, 1, 31)
    x = seeded_grid((384, 448), 32)
    a = run_gpu(ffs.Plan(2, None, (448, 384), 56, weights=w, radius=1, boundary="fixed", tau=tau), x)
    b = run_gpu(ffs.Plan(2, None, (448, 384), 56, weights=w, radius=1, boundary="fixed", tau=tau,
                         form="fp64_fft"), x)
    assert np.abs(a - b).max() / np.abs(a).max() <= 1e-13


@pytest.mark.parametrize("tile", [64, 128])
def test_inplace_and_odd_pass_counts(tile):
    import torch
    x = seeded_grid((128, 130), 3)
    w = seeded_weights(2, 1, 3)
    for T in (5, 12, 16):
        p = ffs.Plan(2, None, (130, 128), T, weights=w, radius=1, boundary="fixed", tau=4, form="fp64_fft",
                     tile=tile)
        d = torch.from_numpy(x).cuda()
        p.execute(d.data_ptr(), d.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        ref = oracle.run(x, w, 1, T, oracle.FIXED)
        assert rel_errors(d.cpu().numpy(), ref)[0] <= TOL, (T, p.info)


def test_host_pipeline_many_grids():
    import torch
    plan = ffs.Plan(2, "Box2D9P", (260, 190), 11, boundary="fixed", form="fp64_fft")
    xs = [torch.from_numpy(seeded_grid((190, 260), 40 + i)).pin_memory().numpy() for i in range(3)]
    outs = [torch.empty((190, 260), dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
    plan.run_host_many(xs, outs)
    for x, o in zip(xs, outs):
        assert rel_errors(o, oracle.run(x, ffs.shape_info("Box2D9P").weights, 1, 11, oracle.FIXED))[0] <= TOL


def test_batch_with_butterfly_plans():
    import torch
    specs = [("Box2D9P", (128, 96), 7, "fixed", "fp64_fft"), ("Heat-2D", (200, 64), 3, "periodic", "fp64"),
             ("Box2D25P", (90, 91), 11, "periodic", "fp64_fft")]
    plans, ins, outs, refs = [], [], [], []
    for i, (shape, ext, T, bnd, form) in enumerate(specs):
        p = ffs.Plan(2, shape, ext, T, boundary=bnd, form=form)
        x = torch.from_numpy(seeded_grid((ext[1], ext[0]), 20 + i)).cuda()
        plans.append(p)
        ins.append(x)
        outs.append(torch.empty_like(x))
        refs.append(run_gpu(p, x.cpu().numpy()))
    b = ffs.Batch(plans)
    for _ in range(2):
        for o in outs:
            o.zero_()
        b.execute([t.data_ptr() for t in ins], [t.data_ptr() for t in outs],
                  torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for o, r in zip(outs, refs):
            assert np.array_equal(o.cpu().numpy(), r)


@pytest.mark.parametrize("tile", [64, 128])
def test_bench_config_full_size(tile):
    """Box2D9P 4096^2, fixed ring, T = 32, normalised U(0,1) weights (the benchmark workload)."""
    n = 4096
    x = seeded_grid((n, n), 20251203 + 1)
    w = seeded_weights(2, 1, 20251203 + 1)
    plan = ffs.Plan(2, None, (n, n), 32, weights=w, radius=1, boundary="fixed", form="fp64_fft", tile=tile)
    mx, l2 = rel_errors(run_gpu(plan, x), oracle.run(x, w, 1, 32, oracle.FIXED))
    assert mx <= TOL, (mx, l2, plan.info)


@pytest.mark.parametrize("bnd", ["fixed", "periodic"])
def test_tiles_agree(bnd):
    """The two tile edges solve the same problem to within rounding."""
    w = seeded_weights(2, 1, 41)
    x = seeded_grid((900, 1000), 42)
    a = run_gpu(ffs.Plan(2, None, (1000, 900), 30, weights=w, radius=1, boundary=bnd, form="fp64_fft",
                         tile=64), x)
    b = run_gpu(ffs.Plan(2, None, (1000, 900), 30, weights=w, radius=1, boundary=bnd, form="fp64_fft",
                         tile=128), x)
    assert np.abs(a - b).max() / np.abs(a).max() <= 1e-13


def test_large_grid_properties():
    """8192^2: linearity, conservation of the total (periodic, sum-1 weights), constants kept."""
    import torch
    n = 8192
    w = seeded_weights(2, 1, 77)
    plan = ffs.Plan(2, None, (n, n), 16, weights=w, radius=1, boundary="periodic", form="fp64_fft")
    g = torch.Generator(device="cuda").manual_seed(5)
    a = torch.rand((n, n), dtype=torch.float64, device="cuda", generator=g)
    b = torch.rand((n, n), dtype=torch.float64, device="cuda", generator=g)
    sa, sb = plan.run(a), plan.run(b)
    sab = plan.run(2.0 * a - 3.0 * b)
    assert (sab - (2.0 * sa - 3.0 * sb)).abs().max().item() / sab.abs().max().item() < 1e-12
    assert abs(sa.sum().item() - a.sum().item()) / abs(a.sum().item()) < 1e-12
    c = torch.full((n, n), 0.5, dtype=torch.float64, device="cuda")
    pc = ffs.Plan(2, None, (n, n), 16, weights=w, radius=1, boundary="fixed", form="fp64_fft")
    assert (pc.run(c) - 0.5).abs().max().item() < 1e-13


def test_batch_many_butterfly_plans_and_a_repeated_plan():
    """Butterfly plans run on parallel graph branches; the same plan twice (two grids) shares one
    workspace, so both executions must stay ordered and each match its own single run."""
    import torch
    plans, ins, outs, refs = [], [], [], []
    shared = ffs.Plan(2, "Box2D9P", (200, 150), 13, boundary="fixed", form="fp64_fft")
    for i in range(12):
        p = shared if i in (3, 8) else ffs.Plan(2, "Heat-2D", (96 + 8 * i, 80 + 4 * i), 5 + i, boundary="periodic",
                                                form="fp64_fft")
        ext = p.extents
        x = torch.from_numpy(seeded_grid((ext[1], ext[0]), 70 + i)).cuda()
        plans.append(p)
        ins.append(x)
        outs.append(torch.empty_like(x))
        refs.append(run_gpu(p, x.cpu().numpy()))
    b = ffs.Batch(plans)
    for _ in range(3):
        for o in outs:
            o.zero_()
        b.execute([t.data_ptr() for t in ins], [t.data_ptr() for t in outs], torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for o, r in zip(outs, refs):
            assert np.array_equal(o.cpu().numpy(), r)
