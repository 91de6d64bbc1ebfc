"""ffs_execute_noalloc -- the entry point for callers that may not allocate
device memory (frameworks that own every allocation through their own pool,
loops that must not block on the allocator).  It keeps its ping-pong scratch,
spectra and tables in static device arrays of libffs.so.  Checked here through
the C ABI against the planned path (ffs_plan_create + ffs_execute) and against
the CPU oracle on two calls in a row, each a multi-pass solve that goes through
the static scratch; an in-place call with an odd pass count (its input is copied
into the scratch first); the device's free memory across calls; and the status
read-back ffs_noalloc_status.

This file sorts last so that a run stopping at the first failure has already
run every other test."""
import ctypes

import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import rel_errors, seeded_grid, seeded_weights

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _noalloc(x, ext, T, w, r, bnd, tau, stream, out=None):
    import torch
    p, _keep = ffs._make_problem(2, None, ext, T, weights=w, radius=r, boundary=bnd, tau=tau)
    out = torch.empty_like(x) if out is None else out
    st = ffs.lib.ffs_execute_noalloc(ctypes.byref(p), ctypes.c_void_p(x.data_ptr()),
                                     ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    assert st == ffs.OK, ffs.lib.ffs_last_error_string().decode()
    return out


def _status():
    word = ctypes.c_int(-1)
    assert ffs.lib.ffs_noalloc_status(ctypes.byref(word)) == ffs.OK, ffs.lib.ffs_last_error_string().decode()
    return word.value


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
        mode = oracle.FIXED if bnd == "fixed" else oracle.PERIODIC
        cpu = oracle.run(x.cpu().numpy(), w, r, T, mode)
        mx, _ = rel_errors(got.cpu().numpy(), cpu)
        assert mx <= TOL, ("oracle", ext, T, bnd, mx)
        assert _status() == 0


def test_noalloc_in_place_odd_passes_against_oracle():
    """d_in == d_out with an odd number of passes: the input is copied into the static
    scratch first, so the first pass does not overwrite cells other tiles still read."""
    import torch
    ext, T, r, tau = (260, 230), 15, 1, 6  # 3 passes
    w = seeded_weights(2, r, 11)
    host = seeded_grid((ext[1], ext[0]), 11)
    plan = ffs.Plan(2, None, ext, T, weights=w, radius=r, boundary="fixed", tau=tau)
    assert plan.info["passes"] % 2 == 1
    x = torch.from_numpy(host).cuda()
    ref = plan.run(x)
    _noalloc(x, ext, T, w, r, "fixed", tau, torch.cuda.current_stream().cuda_stream, out=x)
    torch.cuda.synchronize()
    got = x.cpu().numpy()
    assert rel_errors(got, ref.cpu().numpy())[0] <= TOL
    assert rel_errors(got, oracle.run(host, w, r, T, oracle.FIXED))[0] <= TOL
    assert _status() == 0


def test_noalloc_allocates_nothing():
    """After a first call (the per-device set-up), further calls leave the device's free
    memory unchanged: the scratch is the library's static array, not an allocation."""
    import torch
    ext, T, r, tau = (512, 384), 20, 1, 6
    w = seeded_weights(2, r, 12)
    x = torch.from_numpy(seeded_grid((ext[1], ext[0]), 12)).cuda()
    out = torch.empty_like(x)
    stream = torch.cuda.current_stream().cuda_stream
    _noalloc(x, ext, T, w, r, "periodic", tau, stream, out=out)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        _noalloc(x, ext, T, w, r, "periodic", tau, stream, out=out)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert _status() == 0


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
