"""The Levenberg-Marquardt restatement behind the LEVMAR distortion fit
(p-tracker_b200/csrc/ptk_lmdif.hpp), pinned on the CPU to MINPACK's own lmdif
as scipy.optimize.leastsq runs it: the reference's LEVMAR calls lmdif1 from the
absent toofus library, whose published algorithm is MINPACK's.  Same
standard problems (Rosenbrock, Powell singular, an exponential fit, a
rank-deficient linear fit), same residual operations, lmdif1's settings
(ftol = xtol = tol, gtol = 0, maxfev = 200 (n + 1), sqrt(eps) differences,
factor 100, scaling by column norms): same minimiser within 1e-9 and the same
exit state."""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    so = tmp_path_factory.mktemp("lmdif") / "liblmdif_harness.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", str(HERE / "lmdif_harness.cpp"), "-o", str(so)],
                   check=True)
    L = C.CDLL(str(so))
    L.lm_run.restype = C.c_int
    L.lm_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.POINTER(C.c_int)]
    return L


def residuals(problem: int, x):
    if problem == 0:
        return [10.0 * (x[1] - x[0] * x[0]), 1.0 - x[0]]
    if problem == 1:
        return [x[0] + 10.0 * x[1], math.sqrt(5.0) * (x[2] - x[3]), (x[1] - 2.0 * x[2]) * (x[1] - 2.0 * x[2]),
                math.sqrt(10.0) * (x[0] - x[3]) * (x[0] - x[3])]
    if problem == 2:
        out = []
        for i in range(12):
            t = 0.5 * i
            y = 2.5 * math.exp(-0.7 * t) + 0.3 + 0.01 * math.sin(3.0 * t)
            out.append(x[0] * math.exp(-x[1] * t) + x[2] - y)
        return out
    return [x[0] + i * x[1] + i * x[2] - (1.0 + 2.0 * i + 0.1 * ((i * 7) % 3)) for i in range(6)]


CASES = [(0, 2, [-1.2, 1.0]), (1, 4, [3.0, -1.0, 0.0, 1.0]), (2, 12, [1.0, 0.2, 0.0]), (3, 6, [0.0, 0.0, 0.0])]


@pytest.mark.parametrize("problem,m,x0", CASES, ids=["rosenbrock", "powell_singular", "exp_fit", "rank_deficient"])
@pytest.mark.parametrize("tol", [1.49012e-8, np.finfo(float).eps])
def test_lmdif_matches_minpack(harness, problem, m, x0, tol):
    from scipy.optimize import leastsq

    n = len(x0)
    x = np.array(x0, dtype=np.float64)
    f = np.zeros(m)
    nfev = C.c_int()
    info = harness.lm_run(problem, m, n, x.ctypes.data, f.ctypes.data, tol, C.byref(nfev))
    xs, cov, infod, msg, ier = leastsq(lambda v: np.array(residuals(problem, list(v))), np.array(x0, dtype=float),
                                       full_output=True, ftol=tol, xtol=tol, gtol=0.0, maxfev=200 * (n + 1),
                                       epsfcn=0.0, factor=100.0)
    assert info == ier, (info, ier, msg)
    scale = max(1.0, float(np.abs(xs).max()))
    assert np.abs(x - xs).max() <= 1e-9 * scale, (x, xs)
    assert abs(nfev.value - infod["nfev"]) <= 1
    np.testing.assert_allclose(f, np.array(residuals(problem, list(x))), rtol=0, atol=1e-15)


def test_lmdif_on_distortion_residuals_matches_minpack(harness, oracle):
    """The LEVMAR fit's problem itself: the 14 undistor parameters from a
    start with K1 = 0, over the equiprojectivity residuals of the oracle
    (which the GPU kernel reproduces bit for bit).  Same exit state, same
    number of evaluations, and the same parameters as MINPACK's lmdif."""
    from scipy.optimize import leastsq

    from disto_cases import case

    c = case(oracle, 5, n=80, n_tracked=3)
    pairs = oracle.disto_pairs(c["refx"], c["refy"], 200.0, 1200.0)

    def res(x):
        return oracle.disto_objective(np.asarray(x), c["refx"], c["refy"], c["dx"], c["dy"], c["ncc"], 0.7, pairs,
                                      with_residuals=True)[1]

    X0 = c["X"].copy()
    X0[2] = 0.0
    m = res(X0).shape[0]
    cbtype = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double))

    def cb(xp, fp):
        np.ctypeslib.as_array(fp, shape=(m,))[:] = res(np.ctypeslib.as_array(xp, shape=(14,)).copy())
        return 0

    keep = cbtype(cb)
    harness.lm_run_cb.restype = C.c_int
    harness.lm_run_cb.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.POINTER(C.c_int), cbtype]
    x = X0.copy()
    f = np.zeros(m)
    nfev = C.c_int()
    eps = float(np.finfo(float).eps)
    info = harness.lm_run_cb(m, 14, x.ctypes.data, f.ctypes.data, eps, C.byref(nfev), keep)
    xs, _, infod, msg, ier = leastsq(res, X0, full_output=True, ftol=eps, xtol=eps, gtol=0.0, maxfev=200 * 15,
                                     epsfcn=0.0, factor=100.0)
    assert info == ier and nfev.value == infod["nfev"], (info, ier, msg, nfev.value, infod["nfev"])
    np.testing.assert_allclose(x, xs, rtol=1e-10, atol=1e-30)
    assert (f ** 2).sum() < 1e-18 * (res(X0) ** 2).sum()
