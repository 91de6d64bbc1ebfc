"""Generate tests/golden/ref_cpu_vectors.npz from the reference's own CPU stencils.

Runs the unmodified reference functions stencil1D (src/1D/check_correct.hpp:15-38)
and stencil2D / rotateKernel180 (src/2D/check_correct.hpp:17-33, 64-100), compiled
from the reference sources by oracle/Makefile into oracle/_ref/libffsref.so, on
the reference's debug inputs (src/1D/1d_main.cu:114-141, src/2D/2d_main.cu:96-126
use i+1 / 1 patterns) and on seeded random inputs.  Multi-step vectors iterate the
reference function T times (the reference itself has no T loop; its GPU driver
launches one step per launch, src/2D/2d_main.cu:150-170).

Run in a container that has the reference sources:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402


def main():
    oracle.build()
    if oracle.ref_lib() is None:
        raise SystemExit("oracle/_ref/libffsref.so missing: the reference sources are needed")
    rng = np.random.default_rng(20251203)
    out = {}
    # known answers: small hand-checkable inputs through the reference's own CPU stencil
    x = np.arange(8, dtype=np.float64)
    out["ka1d_in"] = x
    out["ka1d_w"] = np.array([0.25, 0.5, 0.25])
    out["ka1d_out"] = oracle.ref_stencil1d(x, out["ka1d_w"])
    g = np.arange(16, dtype=np.float64).reshape(4, 4)
    ident = np.zeros((3, 3))
    ident[1, 1] = 1.0
    out["ka2d_in"] = g
    out["ka2d_k"] = oracle.ref_rotate180(ident)
    out["ka2d_out"] = oracle.ref_stencil2d(g, out["ka2d_k"])
    # reference debug-mode style input (i+1) with kernel weights i+1
    x = np.arange(1, 57, dtype=np.float64)
    k = np.arange(1, 8, dtype=np.float64)
    out["dbg1d_in"], out["dbg1d_w"] = x, k
    out["dbg1d_out"] = oracle.ref_stencil1d(x, k)
    # seeded random cases, single and multi step (reference function iterated)
    cases1d = [(64, 3, 1), (101, 5, 3), (97, 7, 4), (256, 3, 16)]
    for i, (n, K, T) in enumerate(cases1d):
        x = rng.random(n)
        w = rng.random(K)
        w /= w.sum()
        y = x.copy()
        for _ in range(T):
            y = oracle.ref_stencil1d(y, w)
        out[f"r1d{i}_in"], out[f"r1d{i}_w"], out[f"r1d{i}_T"], out[f"r1d{i}_out"] = x, w, np.array(T), y
    cases2d = [(16, 3, 1), (21, 3, 3), (18, 5, 2), (33, 5, 5)]
    for i, (W, K, T) in enumerate(cases2d):
        x = rng.random((W, W))
        k = rng.random((K, K))
        k /= k.sum()
        y = x.copy()
        for _ in range(T):
            y = oracle.ref_stencil2d(y, k)
        out[f"r2d{i}_in"], out[f"r2d{i}_k"], out[f"r2d{i}_T"], out[f"r2d{i}_out"] = x, k, np.array(T), y
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_cpu_vectors.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    main()
