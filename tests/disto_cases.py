"""Synthetic inputs of the distortion-parameter fit (test helpers): integer
reference positions in the distorted frame, a translation per image applied
in the undistorted frame (translations are equiprojective: the criterion
vanishes at the true parameters), and the tracked displacements that a
perfect tracker reports (the distorted positions found by inverting
undistor with the oracle's Newton inverse)."""
from __future__ import annotations

import numpy as np


def params(dimx: int, dimy: int, k1: float = -2e-9, k2: float = 1e-16) -> np.ndarray:
    X = np.zeros(14)
    X[0], X[1] = 0.5 * dimx, 0.5 * dimy
    X[2], X[3] = k1, k2
    X[8], X[9] = 0.5 * dimx, 0.5 * dimy
    return X


def case(oracle, seed: int, n: int = 150, n_tracked: int = 3, dimx: int = 2048, dimy: int = 1536,
         k1: float = -2e-9, k2: float = 1e-16, low_ncc: float = 0.05):
    rng = np.random.default_rng(seed)
    X = params(dimx, dimy, k1, k2)
    refx = rng.integers(60, dimx - 60, n).astype(np.int32)
    refy = rng.integers(60, dimy - 60, n).astype(np.int32)
    und = np.array([oracle.undistor(X, float(x), float(y)) for x, y in zip(refx, refy)])
    L = oracle.C.CDLL(str(oracle.PORT_SO))
    dx = np.zeros((n_tracked, n))
    dy = np.zeros((n_tracked, n))
    for im in range(n_tracked):
        t = rng.uniform(-20.0, 20.0, 2)
        moved = und + t
        for g in range(n):
            xd, yd = oracle.C.c_double(), oracle.C.c_double()
            L.orc_distort_point(oracle._p(X), oracle._D(moved[g, 0]), oracle._D(moved[g, 1]), oracle.C.byref(xd),
                                oracle.C.byref(yd))
            dx[im, g] = xd.value - refx[g]
            dy[im, g] = yd.value - refy[g]
    ncc = np.where(rng.random((n_tracked, n)) < low_ncc, 0.3, 0.98)
    return dict(X=X, refx=refx, refy=refy, dx=dx, dy=dy, ncc=ncc, dimx=dimx, dimy=dimy)
