"""Slab decomposition of one grid (flashfftstencil_b200.slab) on CPU.

The local tau-step solve is the oracle itself, so these tests check the
decomposition alone -- slab bounds, ghost widths, the exchange pattern, the
core/strip split and the pass structure -- and every result must equal the
oracle's solve of the whole grid bit for bit: a cell's value depends only on
the cells within r*T of it, computed in the same order either way.  The
multi-rank cases run real torch.distributed ranks over gloo."""
import os
import socket

import numpy as np
import pytest
import torch

import oracle
from flashfftstencil_b200.slab import SlabPlan, run_local, slab_bounds
from tests.helpers import seeded_grid, seeded_weights

MODES = {"fixed": oracle.FIXED, "periodic": oracle.PERIODIC}


def oracle_stepper(w, r, boundary):
    """The oracle holds (or wraps) every face, open or not: cells near an open face
    come out wrong, which the decomposition must never let through."""
    def make(ext, tau, open_faces):
        def step(src, dst):
            dst.copy_(torch.from_numpy(oracle.run(src.numpy(), w, r, tau, MODES[boundary])))
        return step
    return make


def case_grid(dim, ext, seed):
    return seeded_grid(tuple(reversed(ext)), seed)


@pytest.mark.parametrize("n,world", [(10, 3), (7, 7), (1000, 8), (5, 1)])
def test_slab_bounds_cover_evenly(n, world):
    b = [slab_bounds(n, world, k) for k in range(world)]
    assert b[0][0] == 0 and b[-1][1] == n
    assert all(b[k][1] == b[k + 1][0] for k in range(world - 1))
    sizes = [hi - lo for lo, hi in b]
    assert max(sizes) - min(sizes) <= 1


CASES = [
    # dim, ext (x fastest), T, boundary, tau, world, r
    (2, (37, 90), 12, "fixed", 3, 3, 1),       # split passes (rows 30 >= 4g = 12)
    (2, (37, 90), 12, "periodic", 3, 3, 1),
    (2, (40, 50), 9, "fixed", 4, 2, 2),        # rows 25 < 4g = 32: one solve after the exchange
    (2, (33, 64), 10, "periodic", 0, 4, 1),    # tau from the plan builder
    (1, (400,), 20, "fixed", 6, 3, 1),
    (1, (300,), 11, "periodic", 2, 4, 3),
    (3, (9, 10, 40), 5, "fixed", 2, 2, 1),
    (3, (8, 7, 48), 6, "periodic", 2, 3, 1),
    (2, (20, 31), 0, "fixed", 0, 2, 1),        # T = 0 returns the input
]


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("dim,ext,T,bnd,tau,world,r", CASES)
def test_emulated_ranks_equal_whole_grid(dim, ext, T, bnd, tau, world, r, overlap):
    w = seeded_weights(dim, r, 3)
    x = case_grid(dim, ext, 11)
    plans = [SlabPlan(dim, None, ext, T, weights=w, radius=r, boundary=bnd, rank=k, world=world, tau=tau,
                      stepper=oracle_stepper(w, r, bnd), overlap=overlap) for k in range(world)]
    xt = torch.from_numpy(x)
    slabs = [xt[pl.lo:pl.hi].contiguous() for pl in plans]
    got = torch.cat(run_local(plans, slabs)).numpy()
    ref = oracle.run(x, w, r, T, MODES[bnd]) if T else x
    assert np.array_equal(got, ref)


def test_split_and_single_solve_are_both_used():
    w = seeded_weights(2, 1, 3)
    kw = dict(weights=w, radius=1, boundary="fixed", world=3, tau=3, overlap=True)
    assert not any(p.split for p in SlabPlan(2, None, (37, 90), 12, rank=1, **dict(kw, overlap=False)).passes)
    assert all(p.split for p in SlabPlan(2, None, (37, 90), 12, rank=1, **kw).passes)
    assert not any(p.split for p in SlabPlan(2, None, (37, 30), 12, rank=1, **kw).passes)
    edge = SlabPlan(2, None, (37, 90), 12, rank=0, **kw)
    assert edge.up is None and edge.down == 1 and edge.passes[0].gl == 0 and edge.passes[0].gh == 3


def test_slab_thinner_than_ghost_raises():
    w = seeded_weights(2, 1, 3)
    with pytest.raises(ValueError, match="thinner"):
        SlabPlan(2, None, (16, 20), 16, weights=w, radius=1, boundary="periodic", rank=0, world=4, tau=8)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, dim, ext, T, bnd, tau, r, out_dir, overlap):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = seeded_weights(dim, r, 3)
        x = torch.from_numpy(case_grid(dim, ext, 11))
        pl = SlabPlan(dim, None, ext, T, weights=w, radius=r, boundary=bnd, rank=rank, world=world, tau=tau,
                      stepper=oracle_stepper(w, r, bnd), overlap=overlap)
        y = pl.run(x[pl.lo:pl.hi].contiguous())
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), y.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dim,ext,T,bnd,tau,world,r,overlap", [
    (2, (37, 90), 12, "fixed", 3, 2, 1, False),
    (2, (37, 90), 12, "periodic", 3, 2, 1, True),     # both neighbours are the same rank
    (2, (29, 60), 9, "periodic", 2, 3, 2, False),
    (3, (8, 7, 48), 6, "fixed", 2, 3, 1, True),
])
def test_gloo_ranks_equal_whole_grid(tmp_path, dim, ext, T, bnd, tau, world, r, overlap):
    torch.multiprocessing.spawn(_rank_main, args=(world, _free_port(), dim, ext, T, bnd, tau, r, str(tmp_path),
                                                  overlap), nprocs=world, join=True)
    got = np.concatenate([np.load(tmp_path / f"rank{k}.npy") for k in range(world)])
    x = case_grid(dim, ext, 11)
    w = seeded_weights(dim, r, 3)
    assert np.array_equal(got, oracle.run(x, w, r, T, MODES[bnd]))

