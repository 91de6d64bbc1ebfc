"""Measured autotuning: ffs_autotune times the cost model's best candidates and the
winner is used by later plans of the same class (and persisted via FFS_TUNE_CACHE)."""
import os
import subprocess
import sys

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
