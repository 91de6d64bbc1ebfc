"""Slab decomposition with the CUDA local solves: the ranks of a decomposition
are emulated inside one process on one GPU (ghosts copied between the slabs'
buffers; no kernel waits on another rank), and the joined result must match
the oracle's whole-grid solve to max|y-r|/max|r| <= 1e-12."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from flashfftstencil_b200.slab import SlabPlan, run_local
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("dim,shape,ext,T,bnd,tau,world", [
    (2, "Box2D9P", (512, 600), 24, "fixed", 0, 4),        # split passes (core + strips)
    (2, "Box2D9P", (512, 600), 24, "periodic", 0, 4),
    (2, "Box2D25P", (300, 200), 14, "periodic", 4, 3),
    (2, "Heat-2D", (200, 90), 16, "fixed", 8, 3),         # thin slabs (30 < 4g): one solve after the exchange
    (3, "Box3D27P", (40, 36, 64), 6, "fixed", 2, 2),
    (3, "Heat-3D", (32, 32, 48), 4, "periodic", 2, 3),
    (1, "1D7P", (30000,), 40, "fixed", 0, 3),
    (1, "Heat-1D", (20000,), 64, "periodic", 0, 2),
])
def test_emulated_slabs_match_oracle(dim, shape, ext, T, bnd, tau, world, overlap):
    import torch
    si = ffs.shape_info(shape)
    w = seeded_weights(dim, si.radius, 5)
    x = seeded_grid(tuple(reversed(ext)), 21)
    plans = [SlabPlan(dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd, rank=k, world=world, tau=tau,
                      overlap=overlap) for k in range(world)]
    xt = torch.from_numpy(x).cuda()
    got = torch.cat(run_local(plans, [xt[p.lo:p.hi].contiguous() for p in plans]))
    torch.cuda.synchronize()
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got.cpu().numpy(), ref)
    assert mx <= TOL, (mx, l2, [p.passes[0] for p in plans])


@pytest.mark.parametrize("dim,shape,ext,T,bnd,tau,world", [
    (2, "Box2D9P", (512, 600), 24, "fixed", 0, 4),
    (2, "Box2D25P", (300, 200), 14, "periodic", 4, 3),
    (3, "Box3D27P", (40, 36, 64), 6, "fixed", 2, 2),
    (1, "1D7P", (30000,), 40, "fixed", 0, 3),
])
def test_emulated_slabs_butterfly_form(dim, shape, ext, T, bnd, tau, world):
    """The slab solves on the FP64 butterfly kernels (open faces at the cuts)."""
    import torch
    si = ffs.shape_info(shape)
    w = seeded_weights(dim, si.radius, 6)
    x = seeded_grid(tuple(reversed(ext)), 22)
    plans = [SlabPlan(dim, None, ext, T, weights=w, radius=si.radius, boundary=bnd, rank=k, world=world, tau=tau,
                      form="fp64_fft") for k in range(world)]
    xt = torch.from_numpy(x).cuda()
    got = torch.cat(run_local(plans, [xt[p.lo:p.hi].contiguous() for p in plans]))
    torch.cuda.synchronize()
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, l2 = rel_errors(got.cpu().numpy(), ref)
    assert mx <= TOL, (mx, l2)
