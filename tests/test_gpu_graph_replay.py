"""ffs_execute replays a captured CUDA graph of the pass sequence when a call repeats
the previous one (same plan and buffers).  The replayed solve must equal the directly
launched one bit for bit: repeated pairs, pairs that alternate (direct launches),
other plans' calls in between, in-place calls with an odd pass count (the first pass
reads a copy of the input), more pairs than the plan keeps graphs for, and while the
plan is traced (which launches directly)."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["fp64_fft", "fp64", "ozaki"])
def test_replayed_solves_equal_the_first(form):
    import torch
    ext, T = (300, 260), 20
    w = ffs.shape_info("Box2D9P").weights
    plan = ffs.Plan(2, "Box2D9P", ext, T, boundary="fixed", form=form, tau=6)  # 4 passes
    xs = [torch.from_numpy(seeded_grid((ext[1], ext[0]), k)).cuda() for k in range(6)]
    ref = [oracle.run(x.cpu().numpy(), w, 1, T, oracle.FIXED) for x in xs]
    outs = [torch.empty_like(x) for x in xs]
    first = None
    other = ffs.Plan(2, "Box2D9P", (64, 64), 4, boundary="fixed", form=form)
    xo = torch.from_numpy(seeded_grid((64, 64), 99)).cuda()
    for rep in range(4):  # six pairs: more than the four the plan keeps graphs for
        for k in (0, 0, 0, 1, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 5, 0, 0):
            if k == 1 and rep == 2:
                other.run(xo)  # another plan's call in between: the next call launches directly
            outs[k].fill_(np.nan)
            plan.run(xs[k], outs[k])
            torch.cuda.synchronize()
            got = outs[k].cpu().numpy()
            assert rel_errors(got, ref[k])[0] <= 1e-12, (form, rep, k)
            if k == 0:
                first = got if first is None else first
                assert np.array_equal(got, first), (form, rep)
    plan.profile(True)  # traced executions launch directly
    plan.run(xs[0], outs[0])
    torch.cuda.synchronize()
    assert np.array_equal(outs[0].cpu().numpy(), first)
    plan.profile(False)


def test_replayed_in_place_odd_passes():
    import torch
    ext, T = (260, 230), 15
    w = ffs.shape_info("Box2D9P").weights
    plan = ffs.Plan(2, "Box2D9P", ext, T, boundary="fixed", form="fp64_fft", tau=5)  # 3 passes
    assert plan.info["passes"] % 2 == 1
    h = seeded_grid((ext[1], ext[0]), 9)
    x = torch.from_numpy(h).cuda()
    for _ in range(5):  # the same buffer in and out, again and again: T steps each time
        plan.run(x, x)
        h = oracle.run(h, w, 1, T, oracle.FIXED)
    torch.cuda.synchronize()
    assert rel_errors(x.cpu().numpy(), h)[0] <= 1e-12


def test_replayed_32_tile_solves():
    """Repeated calls of a 32^3 cluster-tile plan replay its captured passes bit for bit."""
    import torch
    w = seeded_weights(3, 1, 81)
    ext, T = (72, 60, 50), 12
    plan = ffs.Plan(3, None, ext, T, weights=w, radius=1, boundary="fixed", form="fp64_fft", tile=32, tau=4)
    x = torch.from_numpy(seeded_grid((ext[2], ext[1], ext[0]), 82)).cuda()
    out = torch.empty_like(x)
    ref = oracle.run(x.cpu().numpy(), w, 1, T, oracle.FIXED)
    first = None
    for _ in range(4):
        out.fill_(np.nan)
        plan.run(x, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert rel_errors(got, ref)[0] <= 1e-12
        first = got if first is None else first
        assert np.array_equal(got, first)
