"""The reference-compatible CLI (ffs 1d|2d|3d ..., and 1d.out/2d.out/3d.out)."""
import os
import subprocess

import pytest

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "flashfftstencil_b200")
FFS = os.path.join(PKG, "ffs")


def run(args, stdin=None):
    return subprocess.run(args, input=stdin, capture_output=True, text=True, timeout=300)


def test_help_and_usage_errors():
    r = run([FFS, "--help"])
    assert r.returncode == 0 and "stencil-shape" in r.stdout
    assert run([FFS, "2d", "Box2D9P", "64"]).returncode == 1          # missing T
    r = run([os.path.join(PKG, "2d.out"), "Hex-2D", "64", "3"])
    assert r.returncode == 1 and "unknown" in r.stdout
    assert run([FFS, "3d", "Box2D9P", "16", "3"]).returncode == 1      # 2-D shape for 3d
    assert run([FFS, "2d", "Box2D9P", "64", "3", "--nope"]).returncode == 1


def test_custom_needs_enough_weights():
    r = run([FFS, "2d", "Box2D9P", "64", "3", "--custom"], stdin="0.1 0.2\n")
    assert r.returncode == 1 and "expected 9 weights" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("argv,label,dims", [
    (["1d.out", "Heat-1D", "100000", "64"], "1d1r", ("1", "1", "100000")),
    (["2d.out", "Box2D9P", "1000", "32"], "box_2d1r", ("1", "1000", "1000")),
    (["3d.out", "Box3D27P", "64", "16"], "box_3d1r", ("64", "64", "64")),
    (["ffs", "2d", "Star2D9P", "300", "200", "5", "--boundary", "fixed"], "star_2d2r", ("1", "200", "300")),
    (["3d.out", "Box3D27P", "48", "4", "--form", "ozaki"], "box_3d1r", ("48", "48", "48")),
    (["3d.out", "Heat-3D", "40", "36", "32", "6", "--form", "bf16x3", "--boundary", "fixed"], "star_3d1r",
     ("32", "36", "40")),
    (["2d.out", "Box2D25P", "256", "12", "--form", "ozaki", "--slices", "6"], "box_2d2r", ("1", "256", "256")),
    (["2d.out", "Box2D9P", "500", "16", "--form", "fp64"], "box_2d1r", ("1", "500", "500")),  # DMMA form
])
def test_csv_line(argv, label, dims):
    r = run([os.path.join(PKG, argv[0])] + argv[1:])
    assert r.returncode == 0, r.stderr
    f = [s.strip() for s in r.stdout.strip().splitlines()[0].split(",")]
    assert f[0] == "FlashFFTStencil" and f[1] == label and tuple(f[2:5]) == dims
    assert float(f[6]) > 0 and float(f[7]) > 0


@pytest.mark.gpu
def test_custom_weights_from_stdin():
    r = run([FFS, "2d", "Box2D9P", "128", "4", "--custom", "--json"], stdin=" ".join(["0.111"] * 9))
    assert r.returncode == 0, r.stderr
    assert '"passes"' in r.stdout


def test_tensor_core_form_rejected_for_1d():  # validation runs before any device call
    r = run([os.path.join(PKG, "1d.out"), "Heat-1D", "4096", "8", "--form", "ozaki"])
    assert r.returncode != 0 and "2-D and 3-D" in r.stderr


def test_form_names():  # validation runs before any device call
    r = run([os.path.join(PKG, "2d.out"), "Box2D9P", "128", "4", "--form", "fp65"])
    assert r.returncode == 1 and "unknown --form" in r.stderr
