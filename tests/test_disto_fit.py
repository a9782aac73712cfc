"""The distortion-parameter fit's host pieces and its oracle (no GPU): the
pair list of precompute_paires from the C ABI against the port and the
reference's own member function, and the port's equiprojectivity criterion
against the loop around the reference's undistor (both functor forms)."""
from __future__ import annotations

import numpy as np
import pytest

from disto_cases import case


def test_pairs_match_reference(ptk, oracle):
    if not oracle.have_reference():
        pytest.skip("reference build unavailable")
    rng = np.random.default_rng(3)
    refx = rng.integers(0, 2000, 300).astype(np.int32)
    refy = rng.integers(0, 1500, 300).astype(np.int32)
    for dmin, dmax in ((0.0, 1000.0), (150.0, 420.0), (50.0, 50.0)):
        ours = ptk.disto_pairs(refx, refy, dmin, dmax)
        port = oracle.disto_pairs(refx, refy, dmin, dmax)
        ref = oracle.disto_pairs(refx, refy, dmin, dmax, reference=True)
        np.testing.assert_array_equal(port, ref)
        np.testing.assert_array_equal(ours, ref)
    assert len(ptk.disto_pairs(refx[:1], refy[:1], 0.0, 1e9)) == 0


def test_pairs_capacity_is_reported(ptk):
    import ctypes as C
    L = ptk.lib()
    rx = np.array([0, 10, 20], dtype=np.int32)
    ry = np.zeros(3, dtype=np.int32)
    out = np.zeros((1, 2), dtype=np.int32)
    n = C.c_int64()
    rc = L.ptk_disto_pairs(rx.ctypes.data, ry.ctypes.data, 3, 0.0, 100.0, out.ctypes.data, 1, C.byref(n))
    assert rc == 5 and n.value == 3 and list(out[0]) == [0, 1]


@pytest.mark.parametrize("use_orig", [False, True])
def test_objective_port_matches_reference(oracle, use_orig):
    if not oracle.have_reference():
        pytest.skip("reference build unavailable")
    c = case(oracle, 11, n=80, n_tracked=3)
    pairs = oracle.disto_pairs(c["refx"], c["refy"], 100.0, 900.0)
    X = c["X"].copy()
    X[2] *= 0.5
    X[5], X[6], X[11] = 1e-7, -2e-7, 1e-4
    kw = {}
    if use_orig:
        kw = dict(origx=c["refx"] + 0.25, origy=c["refy"] - 0.5)
    a = oracle.disto_objective(X, c["refx"], c["refy"], c["dx"], c["dy"], c["ncc"], 0.7, pairs, **kw)
    b = oracle.disto_objective(X, c["refx"], c["refy"], c["dx"], c["dy"], c["ncc"], 0.7, pairs, reference=True, **kw)
    assert a == b and a > 0.0
    # the true parameters make every retained pair equiprojective (rigid motions)
    t = oracle.disto_objective(c["X"], c["refx"], c["refy"], c["dx"], c["dy"], c["ncc"], 0.7, pairs)
    assert t < 1e-12 * a
