"""The distortion-parameter fit on the GPU (ptk_disto_*) against the CPU
oracle: every residual of the equiprojectivity criterion bit for bit (the
kernel is compiled without FMA contraction, as the CPU restatement), the
criterion to 1e-12 (a different summation order), and the POWELL,
POWELL_ITER and LEVMAR minimisations on synthetic rigid motions seen through
radial distortion."""
from __future__ import annotations

import numpy as np
import pytest

from disto_cases import case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data(oracle):
    c = case(oracle, 21, n=80, n_tracked=2)
    c["pairs"] = oracle.disto_pairs(c["refx"], c["refy"], 200.0, 1200.0)
    return c


def _start(c):
    """The true parameters with K1 unknown (0) and default centres; only K1 is
    perturbed, so the minimisations are one-dimensional and quick on the CPU."""
    X0 = c["X"].copy()
    X0[2] = 0.0
    X0[0] = X0[1] = -1.0
    DX = np.zeros(14)
    DX[2] = 1e-10
    return X0, DX


def _fit(ptk, c):
    return ptk.DistoFit(c["dimx"], c["dimy"], c["refx"], c["refy"], c["dx"], c["dy"], c["ncc"], 0.7, c["pairs"])


def test_residuals_bitwise(ptk, oracle, cuda_device, data):
    c = data
    f = _fit(ptk, c)
    X = c["X"].copy()
    X[2] *= 0.3
    X[4], X[7], X[10], X[13] = 1e-22, 1e-9, 0.02, -3e-4
    v, res = f.residuals(X)
    ov, ores = oracle.disto_objective(X, c["refx"], c["refy"], c["dx"], c["dy"], c["ncc"], 0.7, c["pairs"],
                                      with_residuals=True)
    np.testing.assert_array_equal(res, ores)
    assert abs(v - ov) <= 1e-12 * ov
    assert abs(f.objective(X) - ov) <= 1e-12 * ov
    assert (res == 0).any(), "pairs with a low NCC must be skipped"
    f.close()


def test_fit_powell_matches_oracle(ptk, oracle, cuda_device, data):
    c = data
    X0, DX = _start(c)
    f = _fit(ptk, c)
    x, ini, end, _ = f.fit(X0, DX, ptk.DISTO_POWELL)
    ox, oini, oend, _, _, _ = oracle.disto_fit(X0, DX, 0, 0, c["dimx"], c["dimy"], c["refx"], c["refy"], c["dx"],
                                               c["dy"], c["ncc"], 0.7, c["pairs"])
    assert x[0] == 0.5 * c["dimx"] and x[1] == 0.5 * c["dimy"]
    assert abs(ini - oini) <= 1e-12 * oini
    assert end < 1e-12 * ini and oend < 1e-12 * oini
    np.testing.assert_allclose(x[2], ox[2], rtol=1e-6)
    np.testing.assert_allclose(x[2], c["X"][2], rtol=1e-6)
    f.close()


def test_fit_powell_iter_matches_oracle(ptk, oracle, cuda_device, data):
    c = data
    X0, DX = _start(c)
    f = _fit(ptk, c)
    x, ini, end, hist = f.fit(X0, DX, ptk.DISTO_POWELL_ITER, 2)
    ox, oini, oend, ohist, odx, ody = oracle.disto_fit(X0, DX, 1, 2, c["dimx"], c["dimy"], c["refx"], c["refy"],
                                                       c["dx"], c["dy"], c["ncc"], 0.7, c["pairs"])
    assert hist.shape == (2, 15)
    assert abs(ini - oini) <= 1e-12 * oini
    np.testing.assert_allclose(hist[:, 0], ohist[:, 0], rtol=1e-8)
    np.testing.assert_allclose(hist[:, 3], ohist[:, 3], rtol=1e-6)
    np.testing.assert_allclose(x[2], ox[2], rtol=1e-6)
    assert abs(end - oend) <= 1e-8 * oend
    gdx, gdy = f.tracked()
    np.testing.assert_allclose(gdx, odx, rtol=0, atol=1e-6)
    np.testing.assert_allclose(gdy, ody, rtol=0, atol=1e-6)
    f.close()


def test_fit_levmar_matches_minpack(ptk, oracle, cuda_device, data):
    """LEVMAR: all 14 parameters by Levenberg-Marquardt over the GPU residual
    vector, against MINPACK's lmdif (scipy) over the oracle's residuals, which
    the GPU's equal bit for bit, with lmdif1's settings and tol = DBL_EPSILON
    as the reference passes: same exit state and evaluation count, same
    parameters, and a criterion driven to zero (translations seen through the
    lens are equiprojective at a perfect fit; with all 14 parameters free the
    lens terms trade off against each other, as in the reference)."""
    from scipy.optimize import leastsq

    c = data
    X0 = c["X"].copy()
    X0[2] = 0.0
    f = _fit(ptk, c)
    x, ini, end, hist = f.fit(X0, np.zeros(14), ptk.DISTO_LEVMAR)
    info, nfev, text = f.levmar_info()
    f.close()

    def res(v):
        return oracle.disto_objective(np.asarray(v), c["refx"], c["refy"], c["dx"], c["dy"], c["ncc"], 0.7,
                                      c["pairs"], with_residuals=True)[1]

    eps = float(np.finfo(float).eps)
    xs, _, infod, msg, ier = leastsq(res, X0, full_output=True, ftol=eps, xtol=eps, gtol=0.0, maxfev=200 * 15,
                                     epsfcn=0.0, factor=100.0)
    assert info == ier and nfev == infod["nfev"], (info, ier, msg, nfev, infod["nfev"])
    assert text
    np.testing.assert_allclose(x, xs, rtol=1e-10, atol=1e-30)
    assert hist.shape == (1, 15) and hist[0, 0] == end
    assert end < 1e-18 * ini
