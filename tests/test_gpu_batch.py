"""Many problems in one CUDA graph (ffs_batch_*: FP64-DMMA plans in one persistent kernel, the
other forms' launches on parallel branches): every output matches the
standalone plan's output (same per-item device code; the compiler may contract
a*b - c*d into FMAs differently in the two kernels, so last-bit differences are
allowed) and a sample matches the oracle."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu


def mixed_specs(count, seed):
    """A C5-style mix: 60 % 2D, 30 % 1D, 10 % 3D, uneven sizes, T in 1..64, both boundaries."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        u = rng.random()
        bnd = "fixed" if rng.random() < 0.5 else "periodic"
        T = int(rng.integers(1, 65))
        if u < 0.6:
            shape = ["Heat-2D", "Star2D9P", "Box2D9P"][int(rng.integers(0, 3))]
            ext = (int(np.exp(rng.uniform(np.log(16), np.log(300)))), int(np.exp(rng.uniform(np.log(16), np.log(300)))))
        elif u < 0.9:
            shape = ["1D5P", "1D7P"][int(rng.integers(0, 2))]
            ext = (int(np.exp(rng.uniform(np.log(2 ** 10), np.log(2 ** 16)))),)
        else:
            shape = ["Heat-3D", "Box3D27P"][int(rng.integers(0, 2))]
            ext = tuple(int(np.exp(rng.uniform(np.log(12), np.log(48)))) for _ in range(3))
        specs.append((shape, ext, T, bnd))
    return specs


def test_batch_equals_standalone_and_oracle():
    import torch
    specs = mixed_specs(40, 7) + [("Box2D9P", (64, 64), 0, "fixed")]  # one T = 0 problem
    plans, ins, outs, refs, hosts = [], [], [], [], []
    for i, (shape, ext, T, bnd) in enumerate(specs):
        si = ffs.shape_info(shape)
        w = seeded_weights(si.dim, si.radius, i)
        p = ffs.Plan(si.dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd)
        x = torch.from_numpy(seeded_grid(tuple(reversed(ext)), 100 + i)).cuda()
        plans.append(p)
        ins.append(x)
        outs.append(torch.empty_like(x))
        refs.append(p.run(x).cpu().numpy())
        hosts.append((x.cpu().numpy(), w, si.radius, T, bnd))
    torch.cuda.synchronize()
    b = ffs.Batch(plans)
    stream = torch.cuda.current_stream().cuda_stream
    for rep in range(2):  # capture, then replay
        for o in outs:
            o.fill_(-1.0)
        b.execute([t.data_ptr() for t in ins], [t.data_ptr() for t in outs], stream)
        torch.cuda.synchronize()
        assert b.status() == 0
        for k, (o, r) in enumerate(zip(outs, refs)):
            assert rel_errors(o.cpu().numpy(), r)[0] <= 1e-13, (rep, k, specs[k])
    for k in range(0, len(specs), 7):
        x, w, r, T, bnd = hosts[k]
        ref = oracle.run(x, w, r, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
        assert rel_errors(outs[k].cpu().numpy(), ref)[0] <= 1e-12, specs[k]


def test_batch_in_place_and_mixed_forms():
    import torch
    specs = [("Box2D9P", (200, 120), 17, "fixed", "fp64"), ("Heat-1D", (5000,), 9, "periodic", "fp64"),
             ("Box2D9P", (128, 128), 11, "periodic", "ozaki"), ("Heat-3D", (30, 20, 25), 5, "fixed", "fp64")]
    plans, bufs, refs = [], [], []
    for i, (shape, ext, T, bnd, form) in enumerate(specs):
        si = ffs.shape_info(shape)
        p = ffs.Plan(si.dim, shape, ext, T, boundary=bnd, form=form, tau=3 if form == "fp64" else 0)
        x = torch.from_numpy(seeded_grid(tuple(reversed(ext)), 300 + i)).cuda()
        refs.append(p.run(x).cpu().numpy())
        plans.append(p)
        bufs.append(x)
    b = ffs.Batch(plans)
    b.execute([t.data_ptr() for t in bufs], [t.data_ptr() for t in bufs], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert b.status() == 0
    for k, (o, r) in enumerate(zip(bufs, refs)):
        assert rel_errors(o.cpu().numpy(), r)[0] <= 1e-13, specs[k]


def test_batch_with_the_32_tile():
    """3D butterfly plans on both tile edges in one batch graph, out of place and in place."""
    import torch
    w = seeded_weights(3, 1, 71)
    specs = [((60, 50, 40), 7, "fixed", 32), ((60, 50, 40), 7, "fixed", 16), ((45, 70, 33), 10, "periodic", 32)]
    plans, ins, refs = [], [], []
    for i, (ext, T, bnd, tile) in enumerate(specs):
        p = ffs.Plan(3, None, ext, T, weights=w, radius=1, boundary=bnd, form="fp64_fft", tile=tile)
        assert p.info["tile"] == tile
        x = torch.from_numpy(seeded_grid(tuple(reversed(ext)), 400 + i)).cuda()
        refs.append(p.run(x).cpu().numpy())
        plans.append(p)
        ins.append(x)
    torch.cuda.synchronize()
    b = ffs.Batch(plans)
    stream = torch.cuda.current_stream().cuda_stream
    outs = [torch.empty_like(x) for x in ins]
    b.execute([t.data_ptr() for t in ins], [t.data_ptr() for t in outs], stream)
    torch.cuda.synchronize()
    assert b.status() == 0
    for k, (o, r) in enumerate(zip(outs, refs)):
        assert np.array_equal(o.cpu().numpy(), r), specs[k]
    b.execute([t.data_ptr() for t in ins], [t.data_ptr() for t in ins], stream)  # in place
    torch.cuda.synchronize()
    for k, (o, r) in enumerate(zip(ins, refs)):
        assert np.array_equal(o.cpu().numpy(), r), specs[k]
    x0 = seeded_grid((40, 50, 60), 400)
    assert rel_errors(refs[0], oracle.run(x0, w, 1, 7, oracle.FIXED))[0] <= 1e-12


def test_batch_with_the_128_tile():
    """2D butterfly plans on both tile edges (64 x 64 pairs, 128 x 128 single tiles) in one batch."""
    import torch
    w = seeded_weights(2, 1, 91)
    specs = [((700, 500), 33, "fixed", 128), ((700, 500), 33, "fixed", 64), ((333, 410), 12, "periodic", 128)]
    plans, ins, refs = [], [], []
    for i, (ext, T, bnd, tile) in enumerate(specs):
        p = ffs.Plan(2, None, ext, T, weights=w, radius=1, boundary=bnd, form="fp64_fft", tile=tile)
        assert p.info["tile"] == tile
        x = torch.from_numpy(seeded_grid(tuple(reversed(ext)), 500 + i)).cuda()
        refs.append(p.run(x).cpu().numpy())
        plans.append(p)
        ins.append(x)
    torch.cuda.synchronize()
    b = ffs.Batch(plans)
    outs = [torch.empty_like(x) for x in ins]
    b.execute([t.data_ptr() for t in ins], [t.data_ptr() for t in outs], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert b.status() == 0
    for k, (o, r) in enumerate(zip(outs, refs)):
        assert np.array_equal(o.cpu().numpy(), r), specs[k]
    x0 = seeded_grid((500, 700), 500)
    assert rel_errors(refs[0], oracle.run(x0, w, 1, 33, oracle.FIXED))[0] <= 1e-12
