"""Measured autotuning: ffs_autotune times the cost model's best candidates and the
winner is used by later plans of the same class (and persisted via FFS_TUNE_CACHE);
for the Ozaki form with slices = 0 it first calibrates the slice count."""
import os
import subprocess
import sys

import numpy as np
import pytest

import flashfftstencil_b200 as ffs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_autotune_choice_is_used_by_plans():
    tau, ms = ffs.autotune(2, "Box2D9P", (1536, 1024), 24, boundary="fixed", candidates=4)
    assert 1 <= tau <= 24 and ms > 0
    assert ffs.Plan(2, "Box2D9P", (1536, 1024), 24, boundary="fixed").info["tau"] == tau
    # a different class (other T) keeps the model's choice
    assert ffs.describe(2, "Box2D9P", (1536, 1024), 25, boundary="fixed")["tau"] >= 1


def test_tuning_table_persists_across_processes(tmp_path):
    cache = tmp_path / "tune.txt"
    env = dict(os.environ, FFS_TUNE_CACHE=str(cache))
    code = ("import sys; sys.path.insert(0, %r); import flashfftstencil_b200 as f; "
            "t, _ = f.autotune(1, 'Heat-1D', (300000,), 40, candidates=3); print(t)") % ROOT
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    tau = int(r.stdout.strip().splitlines()[-1])
    assert cache.exists() and cache.read_text().strip()
    code2 = ("import sys; sys.path.insert(0, %r); import flashfftstencil_b200 as f; "
             "print(f.describe(1, 'Heat-1D', (300000,), 40)['tau'])") % ROOT
    r2 = subprocess.run([sys.executable, "-c", code2], env=env, capture_output=True, text=True, timeout=300)
    assert r2.returncode == 0 and int(r2.stdout.strip()) == tau


def _splitmix_uniform(n, seed):
    """The autotuner's calibration grid: splitmix64 of (seed, index) -> uniform [0, 1)."""
    i = np.arange(n, dtype=np.uint64)
    z = np.uint64(seed) + (i + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    z ^= z >> np.uint64(31)
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


@pytest.mark.parametrize("dim,shape,ext,T", [(2, "Box2D9P", (2048, 1536), 32), (3, "Box3D27P", (96, 80, 64), 16)])
def test_autotune_calibrates_the_ozaki_slice_count(dim, shape, ext, T):
    """slices = 0: ffs_autotune keeps the smallest slice count whose solve of its seeded grid is
    within 1e-12 / 1.5 of the FP64 butterfly form's, and plans of the class use it."""
    import torch
    tau, _ = ffs.autotune(dim, shape, ext, T, boundary="fixed", form="ozaki", slices=0, candidates=3)
    plan = ffs.Plan(dim, shape, ext, T, boundary="fixed", form="ozaki", slices=0)
    s = plan.info["slices"]
    assert 4 <= s <= 8 and plan.info["tau"] == tau
    x = torch.from_numpy(_splitmix_uniform(int(np.prod(ext)), 0x5EED5EED).reshape(tuple(reversed(ext)))).cuda()
    ref = ffs.Plan(dim, shape, ext, T, boundary="fixed", form="fp64_fft").run(x).cpu().numpy()

    def err(sl):  # at the tuned fused step count, as the calibration ran
        y = ffs.Plan(dim, shape, ext, T, boundary="fixed", form="ozaki", slices=sl, tau=tau).run(x).cpu().numpy()
        return float(np.abs(y - ref).max() / np.abs(ref).max())

    assert err(s) <= 1e-12 / 1.5
    if s > 4:
        assert err(s - 1) > 1e-12 / 1.5  # the smallest count that meets the bound
    # and the calibrated plan meets 1e-12 against the oracle on other inputs
    import oracle
    h = np.random.default_rng(5).random(tuple(reversed(ext)))
    y = plan.run(torch.from_numpy(h).cuda()).cpu().numpy()
    r = oracle.run(h, ffs.shape_info(shape).weights, 1, T, oracle.FIXED)
    assert np.abs(y - r).max() / np.abs(r).max() <= 1e-12
