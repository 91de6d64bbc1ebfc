"""ffs_execute_noalloc -- the entry point for callers that may not allocate
device memory (frameworks that own every allocation through their own pool,
loops that must not block on the allocator).  It keeps its ping-pong scratch,
spectra and tables in static device arrays of libffs.so.  Checked here through
the C ABI against the planned path (ffs_plan_create + ffs_execute) on two calls
in a row, each a multi-pass solve that goes through the static scratch.

This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes

import numpy as np
import pytest

import flashfftstencil_b200 as ffs
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _noalloc(x, ext, T, w, r, bnd, tau, stream):
    import torch
    p, _keep = ffs._make_problem(2, None, ext, T, weights=w, radius=r, boundary=bnd, tau=tau)
    out = torch.empty_like(x)
    st = ffs.lib.ffs_execute_noalloc(ctypes.byref(p), ctypes.c_void_p(x.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert st == ffs.OK, ffs.lib.ffs_last_error_string().decode()
    return out


def test_noalloc_matches_planned_path_two_calls():
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    cases = [((300, 256), 17, "fixed", 1, 6, 1), ((512, 500), 9, "periodic", 2, 4, 2)]
    for ext, T, bnd, r, tau, seed in cases:  # two calls in a row, different sizes and boundaries
        x = torch.from_numpy(seeded_grid((ext[1], ext[0]), seed)).cuda()
        w = seeded_weights(2, r, seed)
        plan = ffs.Plan(2, None, ext, T, weights=w, radius=r, boundary=bnd, tau=tau)
        assert plan.info["passes"] >= 2  # the solve goes through the scratch
        ref = plan.run(x)
        got = _noalloc(x, ext, T, w, r, bnd, tau, stream)
        torch.cuda.synchronize()
        mx, _ = rel_errors(got.cpu().numpy(), ref.cpu().numpy())
        assert mx <= TOL, (ext, T, bnd, mx)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    w = seeded_weights(2, 1, 3)
    p, _keep = ffs._make_problem(2, None, (2048, 1024), 4, weights=w, radius=1)
    x = torch.zeros((1024, 2048), dtype=torch.float64, device="cuda")
    st = ffs.lib.ffs_execute_noalloc(ctypes.byref(p), ctypes.c_void_p(x.data_ptr()),
                                     ctypes.c_void_p(x.data_ptr()), None)
    assert st == ffs.ERR_UNSUPPORTED
    assert "exceeds the static scratch limit" in ffs.lib.ffs_last_error_string().decode()


def test_noalloc_auto_form_is_the_dmma_form():
    """A zeroed problem (form 0 = auto) runs on the DMMA form here, as plans of that form do."""
    import torch
    w = seeded_weights(2, 1, 4)
    ext = (200, 160)
    x = torch.from_numpy(seeded_grid((ext[1], ext[0]), 4)).cuda()
    p, _keep = ffs._make_problem(2, None, ext, 10, weights=w, radius=1, boundary="fixed", form="auto")
    out = torch.empty_like(x)
    st = ffs.lib.ffs_execute_noalloc(ctypes.byref(p), ctypes.c_void_p(x.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()),
                                     ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == ffs.OK, ffs.lib.ffs_last_error_string().decode()
    ref = ffs.Plan(2, None, ext, 10, weights=w, radius=1, boundary="fixed").run(x)
    torch.cuda.synchronize()
    assert rel_errors(out.cpu().numpy(), ref.cpu().numpy())[0] <= TOL
