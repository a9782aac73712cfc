"""The differentiation form: adjoint Levenberg-Marquardt subpixel refinement
(FP32 samples and sums, FP64 3x3 solve and accumulation) against the FP64
Powell oracle, and its FP32 adjoint gradient against the FP64 CPU gradient and
central finite differences (h = 1e-3 px / 1e-5 rad)."""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))
POS_TOL = 0.01     # px, against the FP64 oracle
ROT_TOL = 1e-4     # rad


def _setup_gpu(ptk, wl, pair, **opts):
    p = pair["params"]
    o = wl.tracker_options(p)
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=o["rescue_level"], NCC_min=o["NCC_min"], iraz=1 << 30,
                    **opts)
    for lvl, z in enumerate(o["zones"]):
        if z is not None:
            t.set_zone(lvl, *z)
    t.set_grains(pair["rec"])
    t.make_patterns("grain_diameter", 1.0, 1.0)
    t.load_frame(0, pair["ref"])
    t.load_frame(1, pair["cur"])
    return t


def _oracle(oracle, wl, pair):
    o = wl.tracker_options(pair["params"])
    c = oracle.setup(oracle.Port, pair, threads=THREADS, zones=o["zones"],
                     params={"rescue_level": o["rescue_level"], "NCC_min": o["NCC_min"], "iraz": 1 << 30})
    c.track_frame(1)
    return c.get_grains()


@pytest.mark.parametrize("preset,seed,noise", [("small16", 11, None), ("small16", 12, 0.05 * 65535),
                                               ("tiny", 5, None)])
def test_lm_matches_fp64_powell(ptk, wl, oracle, cuda_device, preset, seed, noise):
    p = dict(wl.PRESETS[preset])
    if noise is not None:
        p["noise"] = noise
    pair = wl.make_pair(p, seed=seed)
    t = _setup_gpu(ptk, wl, pair, subpix_method=ptk.SUBPIX_ADJOINT_LM)
    t.track_frame(1)
    g = t.get_grains()
    c = _oracle(oracle, wl, pair)
    np.testing.assert_array_equal(g[:, :2], c[:, :2])
    assert np.abs(g[:, 4:6] - c[:, 4:6]).max() <= POS_TOL
    assert np.abs(g[:, 6] - c[:, 6]).max() <= ROT_TOL
    assert np.abs(g[:, 12] - c[:, 12]).max() <= 1e-4
    # against the synthetic truth the LM does as well as Powell
    err_lm = np.abs(g[:, 4:6] - pair["truth"][:, :2])
    err_pw = np.abs(c[:, 4:6] - pair["truth"][:, :2])
    assert np.median(err_lm) <= np.median(err_pw) + 2e-3


def test_lm_gradient_f32_vs_fp64_and_fd(ptk, wl, oracle, cuda_device):
    pair = wl.make_pair("small16", seed=7)
    t = _setup_gpu(ptk, wl, pair, subpix_method=ptk.SUBPIX_ADJOINT_LM)
    t.precompute()
    o = wl.tracker_options(pair["params"])
    c = oracle.setup(oracle.Port, pair, threads=THREADS, zones=o["zones"], params={"rescue_level": 0})
    c.precompute()
    rng = np.random.default_rng(4)
    X = rng.uniform(-0.6, 0.6, (t.n, 3)) * np.array([1, 1, 0.02])
    f, G = t.grad(X)
    Gc = np.array([c.gradient(i, X[i])[1] for i in range(t.n)])
    fc = np.array([c.gradient(i, X[i])[0] for i in range(t.n)])
    scale = np.abs(Gc).max(axis=0)
    assert (np.abs(G - Gc) <= 2e-3 * scale + 1e-7).all()
    assert np.abs(f - fc).max() <= 1e-5
    # central finite differences of the FP64 objective
    h = np.array([1e-3, 1e-3, 1e-5])
    for k in range(3):
        Xp, Xm = X.copy(), X.copy()
        Xp[:, k] += h[k]
        Xm[:, k] -= h[k]
        fd = np.array([(c.objective(i, Xp[i]) - c.objective(i, Xm[i])) / (2 * h[k]) for i in range(t.n)])
        assert np.abs(fd - G[:, k]).max() <= 3e-3 * scale[k] + 1e-7
