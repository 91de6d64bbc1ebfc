"""Shared test helpers: seeded inputs, error metrics, and a numpy emulation of
the overlap-save tile method (used to check the tile geometry on CPU)."""
from __future__ import annotations

import numpy as np

import oracle


def seeded_grid(shape, seed, lo=0.0, hi=1.0):
    rng = np.random.default_rng(seed)
    return lo + (hi - lo) * rng.random(shape)


def seeded_weights(dim, r, seed, normalise=True):
    rng = np.random.default_rng(seed + 7)
    w = rng.random((2 * r + 1,) * dim)
    if normalise:
        w /= w.sum()
    return w


def rel_errors(y, ref):
    """Normwise max relative error max|y-r|/max|r| and L2 relative error."""
    y = np.asarray(y, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    d = np.abs(y - ref)
    mx = float(d.max() / max(np.abs(ref).max(), 1e-300))
    l2 = float(np.linalg.norm((y - ref).ravel()) / max(np.linalg.norm(ref.ravel()), 1e-300))
    return mx, l2


def _round_even(v):
    return (v + 1) & ~1


def emulate_tiles(grid, w, r, info, boundary):
    """Run the plan's passes with numpy: overlap-save FFT tiles of edge n with
    halo round_even(r*tau) for the exact window, direct stepping (the oracle)
    for fixed-boundary band cells."""
    x = np.asarray(grid, dtype=np.float64)
    dim = x.ndim
    n = info["tile"]
    K = 2 * r + 1
    wk = np.asarray(w, dtype=np.float64).reshape((K,) * dim)
    ker = np.zeros((n,) * dim)
    for idx in np.ndindex(*wk.shape):
        pos = tuple((-(i - r)) % n for i in idx)
        ker[pos] += wk[idx]
    S = np.fft.fftn(ker)
    bnd = oracle.FIXED if boundary == "fixed" else oracle.PERIODIC
    for p in range(info["passes"]):
        tau = info["tau_last"] if p == info["passes"] - 1 else info["tau"]
        h = _round_even(r * tau)
        u = n - 2 * h
        St = S ** tau
        if bnd == oracle.FIXED:
            y = oracle.run(x, w, r, tau, oracle.FIXED)  # band cells: direct stepping
            vlo = [min(r * tau, e) for e in x.shape]
            vhi = [max(e - r * tau, lo) for e, lo in zip(x.shape, vlo)]
        else:
            y = np.empty_like(x)
            vlo = [0] * dim
            vhi = list(x.shape)
        if all(hi > lo for lo, hi in zip(vlo, vhi)):
            ranges = [range(lo // u, -(-hi // u)) for lo, hi in zip(vlo, vhi)]
            for t in np.ndindex(*[len(rg) for rg in ranges]):
                tidx = [rg[i] for rg, i in zip(ranges, t)]
                org = [ti * u - h for ti in tidx]
                sl = [np.arange(o, o + n) for o in org]
                if bnd == oracle.PERIODIC:
                    tile = x[np.ix_(*[s % e for s, e in zip(sl, x.shape)])]
                else:
                    ok = [(s >= 0) & (s < e) for s, e in zip(sl, x.shape)]
                    tile = np.zeros((n,) * dim)
                    sub = x[np.ix_(*[np.clip(s, 0, e - 1) for s, e in zip(sl, x.shape)])]
                    mask = np.ones((n,) * dim, dtype=bool)
                    for d_, o in enumerate(ok):
                        shp = [1] * dim
                        shp[d_] = n
                        mask &= o.reshape(shp)
                    tile[mask] = sub[mask]
                res = np.real(np.fft.ifftn(np.fft.fftn(tile) * St))
                # crop and store cells inside the exact window
                out_idx = [np.arange(ti * u, ti * u + u) for ti in tidx]
                keep = [(oi >= lo) & (oi < hi) for oi, lo, hi in zip(out_idx, vlo, vhi)]
                gsel = [oi[k] for oi, k in zip(out_idx, keep)]
                lsel = [np.arange(h, h + u)[k] for k in keep]
                y[np.ix_(*gsel)] = res[np.ix_(*lsel)]
        x = y
    return x
