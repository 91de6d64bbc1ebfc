"""The library baselines beside the fused tile path (bench.measure_competitors, the
counterpart of the reference's benchmarks/cufft-by-pytorch/rfft2D.py and
benchmarks/cudnn/cudnn-test.cpp): on periodic grids, one cuFFT round trip with the
spectrum raised to T and T cuDNN direct FP64 convolutions must give the fused path's
result (an independent check of both), and every method reports a rate."""
import pytest

import bench

pytestmark = pytest.mark.gpu


def test_library_baselines_agree_with_the_fused_path():
    out = bench.measure_competitors(cases=(("Box2D9P", (1024, 768), 8), ("Box3D27P", (96, 80, 64), 4)), reps=2)
    assert len(out["cases"]) == 2
    for c in out["cases"]:
        assert c["fused_vs_cufft_power_max_rel_diff"] <= 1e-12, c
        assert c["fused_vs_cudnn_max_rel_diff"] <= 1e-12, c
        for k in ("fused_tile_fp64", "cufft_spectrum_power", "cufft_per_step", "cudnn_direct_fp64"):
            assert c[k] > 0, (k, c)
