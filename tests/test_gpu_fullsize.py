"""Parity on the benchmark configurations at full size, through the C ABI,
against the CPU oracle (the project's restatement of the reference, bit for bit
equal to the compiled reference on the golden cases).

cfg2 (5616x3744 16-bit pair, 2000 bimodal grains, +-15 px, 21 rotation steps),
the bench's own pair (seed 1000), every grain:
  * exact and BF16 pixel stages: the same integer offset and rotation step on
    every grain whose two best NCC values differ by more than 1e-6, NCC within
    1e-5;
  * plain form (exact search + Powell): subpixel positions within 1e-5 px and
    rotations within 1e-6 rad (the bar is 1e-3 px / 1e-4 rad; the objective
    repeats the reference's arithmetic, so Powell takes its path);
  * headline form (BF16 search + adjoint LM): within 0.01 px and 1e-4 rad.
cfg4 (cfg2 with noise of 5 % of the range): the FP64 and FP32 adjoint
gradients of 1 - NCC on 200 sampled grains against the FP64 CPU gradient and
central finite differences (h = 1e-3 px / 1e-5 rad)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import assert_pixel_parity

pytestmark = pytest.mark.gpu

THREADS = max(1, min(48, os.cpu_count() or 1))


def _gpu(ptk, wl, pair, **form):
    p = pair["params"]
    o = wl.tracker_options(p)
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=o["rescue_level"], NCC_min=o["NCC_min"], iraz=1 << 30,
                    **form)
    for lvl, z in enumerate(o["zones"]):
        if z is not None:
            t.set_zone(lvl, *z)
    t.set_grains(pair["rec"])
    t.make_patterns("grain_diameter", 1.0, 1.0)
    t.load_frame(0, pair["ref"])
    t.load_frame(1, pair["cur"])
    return t


def _port(oracle, wl, pair):
    o = wl.tracker_options(pair["params"])
    return oracle.setup(oracle.Port, pair, threads=THREADS, zones=o["zones"],
                        params={"rescue_level": o["rescue_level"], "NCC_min": o["NCC_min"], "iraz": 1 << 30})


@pytest.fixture(scope="module")
def cfg2(wl):
    return wl.make_pair("cfg2", seed=1000)


@pytest.fixture(scope="module")
def cfg2_cpu(oracle, wl, cfg2):
    """The oracle's pixel stage (records and top-two NCC per grain) and its
    subpixel stage (FP64 Powell) over all 2000 grains."""
    c = _port(oracle, wl, cfg2)
    c.precompute()
    c.pixel_all()
    pix, top2 = c.get_grains(), c.top2()
    c.subpixel_all()
    sub = c.get_grains()
    c.close()
    return pix, top2, sub


@pytest.mark.parametrize("method", ["exact", "bf16"])
def test_cfg2_pixel_stage_all_grains(ptk, wl, oracle, cuda_device, cfg2, cfg2_cpu, method):
    pix, top2, _ = cfg2_cpu
    t = _gpu(ptk, wl, cfg2, search_method=ptk.SEARCH_EXACT if method == "exact" else ptk.SEARCH_BF16)
    t.precompute()
    t.search(0)
    checked = assert_pixel_parity(t.get_grains(), pix, top2)
    t.close()
    assert checked >= 0.99 * cfg2["rec"].shape[0]


def test_cfg2_plain_form_all_grains(ptk, wl, oracle, cuda_device, cfg2, cfg2_cpu):
    _, top2, sub = cfg2_cpu
    t = _gpu(ptk, wl, cfg2)
    t.track_frame(1)
    g = t.get_grains()
    t.close()
    clear = (top2[:, 0] - top2[:, 1]) > 1e-6
    assert np.abs(g[clear, 4:6] - sub[clear, 4:6]).max() <= 1e-5
    assert np.abs(g[clear, 6] - sub[clear, 6]).max() <= 1e-6
    assert np.abs(g[clear, 12] - sub[clear, 12]).max() <= 1e-5


def test_cfg2_headline_form_all_grains(ptk, wl, oracle, cuda_device, cfg2, cfg2_cpu):
    _, top2, sub = cfg2_cpu
    t = _gpu(ptk, wl, cfg2, search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM)
    t.track_frame(1)
    g = t.get_grains()
    t.close()
    clear = (top2[:, 0] - top2[:, 1]) > 1e-6
    assert np.abs(g[clear, 4:6] - sub[clear, 4:6]).max() <= 0.01
    assert np.abs(g[clear, 6] - sub[clear, 6]).max() <= 1e-4
    # and as close to the synthetic truth as the FP64 reference
    err_h = np.abs(g[:, 4:6] - cfg2["truth"][:, :2])
    err_r = np.abs(sub[:, 4:6] - cfg2["truth"][:, :2])
    assert np.median(err_h) <= np.median(err_r) + 1e-3


@pytest.mark.parametrize("method", ["fp64_adjoint", "lm_fp32_adjoint"])
def test_cfg4_gradient_200_grains(ptk, wl, oracle, cuda_device, method):
    pair = wl.make_pair("cfg4", seed=1000)
    n = pair["rec"].shape[0]
    form = dict(subpix_method=ptk.SUBPIX_ADJOINT_LM) if method == "lm_fp32_adjoint" else {}
    t = _gpu(ptk, wl, pair, **form)
    t.precompute()
    t.search(0)  # gradients around the integer optimum, where the refinement starts
    gpix = t.get_grains()
    c = _port(oracle, wl, pair)
    c.precompute()
    c.pixel_all()
    cpix = c.get_grains()
    idx = np.unique(np.linspace(0, n - 1, 200).round().astype(int))
    idx = idx[np.all(gpix[idx, 4:7] == cpix[idx, 4:7], axis=1)]  # same start state on both sides
    assert idx.shape[0] >= 190
    rng = np.random.default_rng(17)
    X = np.zeros((n, 3))
    X[idx] = rng.uniform(-0.5, 0.5, (idx.shape[0], 3)) * np.array([1.0, 1.0, 0.005])
    f, G = t.grad(X)
    Gc = np.array([c.gradient(int(i), X[i])[1] for i in idx])
    fc = np.array([c.gradient(int(i), X[i])[0] for i in idx])
    scale = np.abs(Gc).max(axis=0)
    tol = 1e-7 if method == "fp64_adjoint" else 3e-3  # FP32 samples and sums in the LM's adjoint
    assert (np.abs(G[idx] - Gc) <= tol * scale + 1e-9).all()
    assert np.abs(f[idx] - fc).max() <= (1e-12 if method == "fp64_adjoint" else 1e-5)
    # central finite differences of the FP64 objective, h = 1e-3 px / 1e-5 rad
    h = np.array([1e-3, 1e-3, 1e-5])
    t64 = _gpu(ptk, wl, pair)
    t64.precompute()
    t64.search(0)
    for k in range(3):
        Xp, Xm = X.copy(), X.copy()
        Xp[:, k] += h[k]
        Xm[:, k] -= h[k]
        fd = (t64.objective(Xp) - t64.objective(Xm)) / (2 * h[k])
        assert np.abs(fd[idx] - G[idx, k]).max() <= 3e-3 * scale[k] + 1e-7
    t64.close()
    t.close()
    c.close()
