"""The overlap-save tile method with the plan's geometry (tile n, halo, crop,
exact window, band) reproduces the oracle -- checked with numpy FFTs on CPU."""
import numpy as np
import pytest

import flashfftstencil_b200 as ffs
import oracle
from tests.helpers import emulate_tiles, rel_errors, seeded_grid, seeded_weights


@pytest.mark.parametrize("shape,ext,T,bnd", [
    ("Box2D9P", (150, 130), 11, "fixed"),
    ("Box2D9P", (150, 130), 11, "periodic"),
    ("Box2D25P", (97, 120), 7, "fixed"),
    ("Star2D9P", (70, 66), 9, "periodic"),
    ("Heat-2D", (30, 20), 13, "fixed"),  # band covers almost everything
    ("Heat-2D", (10, 9), 4, "periodic"),  # grid smaller than a tile
])
def test_tile_method_matches_oracle(shape, ext, T, bnd):
    si = ffs.shape_info(shape)
    w = seeded_weights(2, si.radius, 11)
    info = ffs.describe(2, None, ext, T, weights=w, radius=si.radius, boundary=bnd)
    x = seeded_grid((ext[1], ext[0]), 12)
    got = emulate_tiles(x, w, si.radius, info, bnd)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    mx, _ = rel_errors(got, ref)
    assert mx < 1e-12, mx


@pytest.mark.parametrize("shape,n,T,bnd", [
    ("Heat-1D", 9000, 64, "fixed"),
    ("1D7P", 5000, 40, "periodic"),
    ("1D5P", 300, 7, "periodic"),
])
def test_tile_method_matches_oracle_1d(shape, n, T, bnd):
    si = ffs.shape_info(shape)
    w = seeded_weights(1, si.radius, 5)
    info = ffs.describe(1, None, (n,), T, weights=w, radius=si.radius, boundary=bnd)
    x = seeded_grid((n,), 6)
    got = emulate_tiles(x, w, si.radius, info, bnd)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    assert rel_errors(got, ref)[0] < 1e-12


@pytest.mark.parametrize("shape,ext,T,bnd", [
    ("Box3D27P", (40, 36, 34), 5, "fixed"),
    ("Heat-3D", (30, 20, 10), 5, "periodic"),
])
def test_tile_method_matches_oracle_3d(shape, ext, T, bnd):
    si = ffs.shape_info(shape)
    w = seeded_weights(3, si.radius, 8)
    info = ffs.describe(3, None, ext, T, weights=w, radius=si.radius, boundary=bnd)
    x = seeded_grid((ext[2], ext[1], ext[0]), 9)
    got = emulate_tiles(x, w, si.radius, info, bnd)
    ref = oracle.run(x, w, si.radius, T, oracle.FIXED if bnd == "fixed" else oracle.PERIODIC)
    assert rel_errors(got, ref)[0] < 1e-12
