"""GPU parity of the 2-D FP64-DMMA fused tile path against the CPU oracle,
called through the C ABI (libffs.so).  Tolerance: max|y-r|/max|r| <= 1e-12."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu
TOL = 1e-12


def torch_cuda():
    import torch
    return torch


def run_gpu(plan, x):
    torch = torch_cuda()
    d = torch.from_numpy(x).cuda()
    out = plan.run(d)
    torch.cuda.synchronize()
    return out.cpu().numpy()


CASES = [
    # shape, (nx, ny), T, boundary, tau
    ("Box2D9P", (512, 512), 32, "fixed", 0),
    ("Box2D9P", (300, 257), 17, "fixed", 0),     # odd width: plain-load path
    ("Box2D9P", (256, 192), 9, "periodic", 0),
    ("Box2D25P", (200, 200), 12, "periodic", 0),
    ("Box2D25P", (222, 180), 7, "fixed", 0),
    ("Star2D9P", (130, 140), 5, "fixed", 0),
    ("Heat-2D", (10, 9), 4, "periodic", 0),      # grid smaller than one tile
    ("Heat-2D", (64, 64), 1, "fixed", 0),
    ("Box2D9P", (160, 96), 20, "periodic", 1),   # tau = 1, many passes
    ("Box2D9P", (97, 301), 6, "periodic", 0),
]


@pytest.mark.parametrize("shape,ext,T,bnd,tau", CASES)
def test_parity_random_weights(shape, ext, T, bnd, tau):
    si = ffs.shape_info(shape)
    w = seeded_weights(2, si.radius, hash(shape) % 1000)
    plan = ffs.Plan(2, None, ext, T, weights=w, radius=si.radius, boundary=bnd, tau=tau)
    x = seeded_grid((ext[1], ext[0]), 101)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL, (mx, l2, plan.info)


@pytest.mark.parametrize("shape", ["Heat-2D", "Box2D9P", "Star2D9P", "Box2D25P"])
def test_named_shapes_default_weights(shape):
    si = ffs.shape_info(shape)
    ext = (180, 150)
    plan = ffs.Plan(2, shape, ext, 10, boundary="fixed")
    x = seeded_grid((ext[1], ext[0]), 7)
    got = run_gpu(plan, x)
    ref = oracle.run(x, si.weights, si.radius, 10, oracle.FIXED)
    assert rel_errors(got, ref)[0] <= TOL


def test_zero_steps_and_inplace():
    torch = torch_cuda()
    x = seeded_grid((128, 130), 3)
    w = seeded_weights(2, 1, 3)
    p0 = ffs.Plan(2, None, (130, 128), 0, weights=w, radius=1)
    assert np.array_equal(run_gpu(p0, x), x)
    for T in (5, 12, 16):  # odd and even pass counts
        p = ffs.Plan(2, None, (130, 128), T, weights=w, radius=1, boundary="fixed", tau=4)
        d = torch.from_numpy(x).cuda()
        p.execute(d.data_ptr(), d.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        ref = oracle.run(x, w, 1, T, oracle.FIXED)
        assert rel_errors(d.cpu().numpy(), ref)[0] <= TOL, (T, p.info)


def test_host_path_matches_device_path():
    x = seeded_grid((200, 210), 4)
    plan = ffs.Plan(2, "Box2D9P", (210, 200), 13, boundary="fixed")
    a = plan.run_host(x)
    b = run_gpu(plan, x)
    assert np.array_equal(a, b)
    assert rel_errors(a, oracle.run(x, ffs.shape_info("Box2D9P").weights, 1, 13, oracle.FIXED))[0] <= TOL


@pytest.mark.parametrize("count", [1, 2, 5])
def test_host_pipeline_many_grids(count):
    """ffs_execute_host_many: each grid's result equals its own single-grid run;
    outputs are pinned so the two device slots' copies really overlap."""
    torch = torch_cuda()
    plan = ffs.Plan(2, "Box2D9P", (260, 190), 11, boundary="fixed")
    xs = [torch.from_numpy(seeded_grid((190, 260), 40 + i)).pin_memory().numpy() for i in range(count)]
    outs = [torch.empty((190, 260), dtype=torch.float64).pin_memory().numpy() for _ in range(count)]
    plan.run_host_many(xs, outs)
    for x, o in zip(xs, outs):
        assert np.array_equal(o, plan.run_host(x))
    ref = oracle.run(xs[-1], ffs.shape_info("Box2D9P").weights, 1, 11, oracle.FIXED)
    assert rel_errors(outs[-1], ref)[0] <= TOL


@pytest.mark.parametrize("faces,T", [(0b1100, 16), (0b0100, 9), (0b0011, 12)])
def test_open_faces_exact_away_from_the_cut(faces, T):
    """Open faces are cuts, not boundaries: every cell at least r*T from them
    (the x faces keep their fixed ring) equals the oracle's fixed-boundary solve."""
    w = seeded_weights(2, 1, 8)
    ext = (230, 170)
    plan = ffs.Plan(2, None, ext, T, weights=w, radius=1, boundary="fixed", open_faces=faces)
    x = seeded_grid((ext[1], ext[0]), 9)
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, 1, T, oracle.FIXED)
    ylo = T if faces & 4 else 0
    yhi = ext[1] - T if faces & 8 else ext[1]
    xlo = T if faces & 1 else 0
    xhi = ext[0] - T if faces & 2 else ext[0]
    mx, l2 = rel_errors(got[ylo:yhi, xlo:xhi], ref[ylo:yhi, xlo:xhi])
    assert mx <= TOL, (mx, l2, plan.info)


def test_same_plan_on_two_streams_without_host_sync():
    """Both executions use the plan's workspace (4 passes): the second waits for the first."""
    torch = torch_cuda()
    w = seeded_weights(2, 1, 12)
    plan = ffs.Plan(2, None, (300, 260), 32, weights=w, radius=1, boundary="fixed", tau=8)
    assert plan.info["passes"] == 4
    xs = [seeded_grid((260, 300), 60 + i) for i in range(2)]
    d_in = [torch.from_numpy(x).cuda() for x in xs]
    d_out = [torch.empty_like(d) for d in d_in]
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    for s, a, b in zip(streams, d_in, d_out):
        plan.run(a, b, stream=s)
    torch.cuda.synchronize()
    for x, b in zip(xs, d_out):
        assert rel_errors(b.cpu().numpy(), oracle.run(x, w, 1, 32, oracle.FIXED))[0] <= TOL


def test_deterministic_repeat():
    x = seeded_grid((333, 256), 5)
    plan = ffs.Plan(2, "Box2D25P", (256, 333), 9, boundary="periodic")
    a = run_gpu(plan, x)
    b = run_gpu(plan, x)
    assert np.array_equal(a, b)


def test_batch_graph_replay_equals_individual_runs():
    torch = torch_cuda()
    specs = [("Box2D9P", (128, 96), 7, "fixed"), ("Heat-2D", (200, 64), 3, "periodic"),
             ("Box2D25P", (90, 91), 11, "periodic")]
    plans, ins, outs, refs = [], [], [], []
    for i, (shape, ext, T, bnd) in enumerate(specs):
        p = ffs.Plan(2, shape, ext, T, boundary=bnd)
        x = torch.from_numpy(seeded_grid((ext[1], ext[0]), 20 + i)).cuda()
        plans.append(p)
        ins.append(x)
        outs.append(torch.empty_like(x))
        refs.append(run_gpu(p, x.cpu().numpy()))
    b = ffs.Batch(plans)
    for _ in range(2):  # second call replays the captured graph
        for o in outs:
            o.zero_()
        b.execute([t.data_ptr() for t in ins], [t.data_ptr() for t in outs],
                  torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        for o, r in zip(outs, refs):
            assert np.array_equal(o.cpu().numpy(), r)


def test_bench_config_full_size():
    """Box2D9P 4096^2, fixed ring, T = 32, normalised U(0,1) weights (the benchmark workload)."""
    n = 4096
    x = seeded_grid((n, n), 20251203 + 1)
    w = seeded_weights(2, 1, 20251203 + 1)
    plan = ffs.Plan(2, None, (n, n), 32, weights=w, radius=1, boundary="fixed")
    got = run_gpu(plan, x)
    ref = oracle.run(x, w, 1, 32, oracle.FIXED)
    mx, l2 = rel_errors(got, ref)
    assert mx <= TOL, (mx, l2)


def test_large_grid_properties():
    """8192^2: linearity and (periodic, sum-1 weights) conservation of the total."""
    torch = torch_cuda()
    n = 8192
    w = seeded_weights(2, 1, 77)
    plan = ffs.Plan(2, None, (n, n), 16, weights=w, radius=1, boundary="periodic")
    g = torch.Generator(device="cuda").manual_seed(5)
    a = torch.rand((n, n), dtype=torch.float64, device="cuda", generator=g)
    b = torch.rand((n, n), dtype=torch.float64, device="cuda", generator=g)
    sa, sb = plan.run(a), plan.run(b)
    sab = plan.run(2.0 * a - 3.0 * b)
    err = (sab - (2.0 * sa - 3.0 * sb)).abs().max().item() / sab.abs().max().item()
    assert err < 1e-12
    tot_in, tot_out = a.sum().item(), sa.sum().item()
    assert abs(tot_out - tot_in) / abs(tot_in) < 1e-12
    c = torch.full((n, n), 0.5, dtype=torch.float64, device="cuda")
    pc = ffs.Plan(2, None, (n, n), 16, weights=w, radius=1, boundary="fixed")
    assert (pc.run(c) - 0.5).abs().max().item() < 1e-13
