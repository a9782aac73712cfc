"""Parity of the CUDA tracking path (through the C ABI) with the CPU oracle.

Bar (per the tracking path's contract): the same integer offset and rotation
step on every grain whose two best NCC values differ by more than 1e-6, NCC
within 1e-5, subpixel positions within 1e-3 px and 1e-4 rad.  The oracle is
the project's CPU restatement (bit-identical to the compiled reference on the
golden cases)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import assert_pixel_parity

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))
SUBPIX_TOL_PX = 1e-3
SUBPIX_TOL_RAD = 1e-4
NCC_TOL = 1e-5


def _gpu(ptk, pair, opts, pattern=("grain_diameter", 1.0, 1.0), masked=None, **extra):
    p = pair["params"]
    options = {k: v for k, v in opts.items() if k != "zones"}
    options.update(extra)
    t = ptk.Tracker(p["dimx"], p["dimy"], **options)
    for lvl, z in enumerate(opts["zones"]):
        if z is not None:
            t.set_zone(lvl, *z)
    t.set_grains(pair["rec"], masked)
    if pattern[0] == "patterns":
        t.set_patterns(pattern[1])
    else:
        t.make_patterns(pattern[0], pattern[1], pattern[2] if len(pattern) > 2 else 0.0)
    t.load_frame(0, pair["ref"])
    t.load_frame(1, pair["cur"])
    return t


def _cpu(oracle, pair, opts, pattern=("grain_diameter", 1.0, 1.0), masked=None, **extra):
    params = {"rescue_level": opts["rescue_level"], "NCC_min": opts.get("NCC_min", 0.7)}
    for k in ("NCC_min_super", "image_interpolator", "iraz", "subpix_tol", "overflow_stiffness",
              "subpix_displacement_max"):
        if k in opts:
            params[k] = opts[k]
    params.update(extra)
    t = oracle.setup(oracle.Port, pair, threads=THREADS, zones=opts["zones"], params=params,
                     pattern=pattern if pattern[0] != "patterns" else ("circ", 1))
    if pattern[0] == "patterns":
        for g, pts in enumerate(pattern[1]):
            t.set_pattern(g, pts)
    if masked is not None:
        t.set_grains(pair["rec"], masked)
    return t


def _opts(wl, pair, **over):
    o = wl.tracker_options(pair["params"])
    o.update(over)
    return o


def test_pixel_stage_8bit(ptk, wl, oracle, cuda_device, pair_cache):
    pair = pair_cache("tiny", 5)
    opts = _opts(wl, pair)
    g = _gpu(ptk, pair, opts)
    g.precompute()
    g.search(0)
    c = _cpu(oracle, pair, opts)
    c.precompute()
    c.pixel_all()
    n = assert_pixel_parity(g.get_grains(), c.get_grains(), c.top2())
    assert n >= pair["rec"].shape[0] - 1


@pytest.mark.parametrize("method", [0, 2], ids=["tiled", "direct"])
def test_pixel_stage_16bit(ptk, wl, oracle, cuda_device, pair_cache, method):
    pair = pair_cache("small16", 7)
    opts = _opts(wl, pair)
    g = _gpu(ptk, pair, opts, search_method=method)
    g.precompute()
    g.search(0)
    c = _cpu(oracle, pair, opts)
    c.precompute()
    c.pixel_all()
    gr, cr = g.get_grains(), c.get_grains()
    assert_pixel_parity(gr, cr, c.top2())
    # the other pixel-stage columns follow the accepted offset exactly
    np.testing.assert_array_equal(gr[:, 7:10], cr[:, 7:10])


def _compare_frame(gr, cr):
    np.testing.assert_array_equal(gr[:, 0:2], cr[:, 0:2])
    assert np.abs(gr[:, 4] - cr[:, 4]).max() <= SUBPIX_TOL_PX
    assert np.abs(gr[:, 5] - cr[:, 5]).max() <= SUBPIX_TOL_PX
    assert np.abs(gr[:, 6] - cr[:, 6]).max() <= SUBPIX_TOL_RAD
    assert np.abs(gr[:, 12] - cr[:, 12]).max() <= NCC_TOL
    assert np.abs(gr[:, 10] - cr[:, 10]).max() <= NCC_TOL


def test_full_frame_powell_16bit(ptk, wl, oracle, cuda_device, pair_cache):
    pair = pair_cache("small16", 11)
    opts = _opts(wl, pair, iraz=100)
    g = _gpu(ptk, pair, opts, iraz=100)
    g.track_frame(1)
    c = _cpu(oracle, pair, opts)
    c.track_frame(1)
    gr, cr = g.get_grains(), c.get_grains()
    _compare_frame(gr, cr)
    # error against the analytic truth is reported, and small
    err = np.abs(gr[:, 4:6] - pair["truth"][:, :2])
    assert np.median(err) < 0.02


def test_full_frame_cfg1_subset(ptk, wl, oracle, cuda_device, pair_cache):
    pair = pair_cache("cfg1", 1, 48)
    opts = _opts(wl, pair, iraz=100)
    g = _gpu(ptk, pair, opts, iraz=100)
    g.track_frame(1)
    c = _cpu(oracle, pair, opts)
    c.track_frame(1)
    _compare_frame(g.get_grains(), c.get_grains())


def test_stagewise_equals_graph(ptk, wl, cuda_device, pair_cache):
    pair = pair_cache("small16", 13)
    opts = _opts(wl, pair, iraz=100)
    a = _gpu(ptk, pair, opts, iraz=100)
    a.track_frame(1)
    b = _gpu(ptk, pair, opts, iraz=100)
    b.precompute()
    b.search(0)
    b.subpixel(0)
    b.end_frame(1)
    np.testing.assert_array_equal(a.get_grains(), b.get_grains())


def _rescue_pair(wl, seed, disp=7.0):
    p = dict(wl.PRESETS["small16"], disp=disp, n=30)
    return wl.make_pair(p, seed=seed)


@pytest.mark.parametrize("method", [0, 2], ids=["tiled", "direct"])
def test_rescue_levels(ptk, wl, oracle, cuda_device, method):
    pair = _rescue_pair(wl, 21)
    z0 = (2, 2, 2, 2, 2, 0.01)
    z1 = (5, 5, 5, 5, 2, 0.01)
    z2 = (9, 9, 9, 9, 3, 0.01)
    opts = dict(zones=[z0, z1, z2], rescue_level=2, NCC_min=0.8, NCC_min_super=0.75, subpixel=0)
    g = _gpu(ptk, pair, opts, search_method=method)
    g.precompute()
    g.search(0)
    g.search(1)
    g.search(2)
    c = _cpu(oracle, pair, opts)
    c.precompute()
    nres = c.pixel_all()
    nsup = c.rescue_all()
    c.super_rescue_all()
    assert nres > 0 and nsup > 0, "workload must exercise both rescue levels"
    assert g.rescue_counts() == (nres, nsup)
    gr, cr = g.get_grains(), c.get_grains()
    assert_pixel_parity(gr, cr, c.top2())
    assert np.abs(gr[:, 11] - cr[:, 11]).max() <= NCC_TOL
    st = g.status()
    res, sup = c.lists()
    assert all(st[i] & ptk.ST_RESCUED for i in res)
    assert all(st[i] & ptk.ST_SUPER_RESCUED for i in sup)


def test_masked_grains(ptk, wl, oracle, cuda_device, pair_cache):
    pair = pair_cache("tiny", 5)
    n = pair["rec"].shape[0]
    masked = np.zeros(n, np.uint8)
    masked[::3] = 1
    opts = _opts(wl, pair, iraz=100)
    g = _gpu(ptk, pair, opts, masked=masked, iraz=100)
    g.track_frame(1)
    c = _cpu(oracle, pair, opts, masked=masked)
    c.track_frame(1)
    gr, cr = g.get_grains(), c.get_grains()
    _compare_frame(gr, cr)
    np.testing.assert_array_equal(gr[masked == 1, 4:7], pair["rec"][masked == 1, 4:7])
    assert (g.status()[masked == 1] & ptk.ST_MASKED).all()


def test_out_of_bounds_grain_is_flagged(ptk, wl, cuda_device, pair_cache):
    pair = dict(pair_cache("tiny", 5))
    rec = pair["rec"].copy()
    rec[0, 0] = 3  # pattern + zone leave the frame on the left
    pair["rec"] = rec
    opts = _opts(wl, pair, iraz=100)
    g = _gpu(ptk, pair, opts, iraz=100)
    g.track_frame(1)
    st = g.status()
    assert st[0] & ptk.ST_OUT_OF_BOUNDS
    assert not (st[1:] & ptk.ST_OUT_OF_BOUNDS).any()


@pytest.mark.parametrize("interp", ["linear", "cubic", "quintic"])
def test_objective_matches(ptk, wl, oracle, cuda_device, pair_cache, interp):
    pair = pair_cache("small16", 7)
    opts = _opts(wl, pair, image_interpolator=ptk.INTERP[interp])
    g = _gpu(ptk, pair, opts)
    g.precompute()
    c = _cpu(oracle, pair, opts)
    c.precompute()
    rng = np.random.default_rng(0)
    X = rng.uniform(-0.8, 0.8, (g.n, 3)) * np.array([1, 1, 0.02])
    fg = g.objective(X)
    fc = np.array([c.objective(i, X[i]) for i in range(g.n)])
    np.testing.assert_allclose(fg, fc, rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("interp", ["linear", "cubic", "quintic"])
def test_objective_to_the_reference_rounding(ptk, wl, oracle, cuda_device, pair_cache, interp):
    """The subpixel objective on the device repeats the reference's
    NCC_to_minimize_xyR operation for operation (no FMA contraction, two
    passes, the sums in point order rounded after every point) with
    correctly rounded cos and sin: the values are the reference's bit for
    bit wherever the host C library's cos and sin are correctly rounded, and
    within its rounding elsewhere."""
    pair = pair_cache("small16", 7)
    opts = _opts(wl, pair, image_interpolator=ptk.INTERP[interp])
    g = _gpu(ptk, pair, opts)
    g.precompute()
    c = _cpu(oracle, pair, opts)
    c.precompute()
    rng = np.random.default_rng(11)
    for rep in range(3):
        X = rng.uniform(-0.8, 0.8, (g.n, 3)) * np.array([1, 1, 0.03])
        fg = g.objective(X)
        fc = np.array([c.objective(i, X[i]) for i in range(g.n)])
        assert np.abs(fg - fc).max() <= 2e-13, np.abs(fg - fc).max()
        assert np.mean(fg == fc) >= 0.99, np.mean(fg == fc)


def test_gradient_matches_fp64_and_fd(ptk, wl, oracle, cuda_device, pair_cache):
    pair = pair_cache("small16", 7)
    opts = _opts(wl, pair)
    g = _gpu(ptk, pair, opts)
    g.precompute()
    c = _cpu(oracle, pair, opts)
    c.precompute()
    rng = np.random.default_rng(1)
    X = rng.uniform(-0.6, 0.6, (g.n, 3)) * np.array([1, 1, 0.02])
    f, G = g.grad(X)
    Gc = np.array([c.gradient(i, X[i])[1] for i in range(g.n)])
    np.testing.assert_allclose(G, Gc, rtol=1e-7, atol=1e-9)
    # central finite differences, h = 1e-3 px / 1e-5 rad
    h = np.array([1e-3, 1e-3, 1e-5])
    for k in range(3):
        Xp, Xm = X.copy(), X.copy()
        Xp[:, k] += h[k]
        Xm[:, k] -= h[k]
        fd = (g.objective(Xp) - g.objective(Xm)) / (2 * h[k])
        scale = np.abs(G[:, k]).max()
        assert np.abs(fd - G[:, k]).max() <= 2e-3 * scale + 1e-9


def test_remap_bit_exact(ptk, wl, oracle, cuda_device):
    p = dict(wl.PRESETS["small16"])
    pair = wl.make_pair(p, seed=3)
    X = np.zeros(14)
    X[0], X[1], X[8], X[9] = 0.5 * p["dimx"], 0.5 * p["dimy"], 0.5 * p["dimx"], 0.5 * p["dimy"]
    X[2], X[3] = -4e-7, 2e-13  # strong distortion at this small frame size
    X[5], X[6], X[11], X[13], X[10] = 1e-5, -2e-5, 1e-3, -2e-3, 0.1
    opts = _opts(wl, pair)
    g = _gpu(ptk, pair, opts)
    g.set_distortion(X)
    g.remap(1)
    out = g.read_frame(1)
    ref = oracle.remap(X, pair["cur"], threads=THREADS)
    np.testing.assert_array_equal(out, ref)


def test_sequence_with_reference_change(ptk, wl, oracle, cuda_device):
    p = dict(wl.PRESETS["small16"], n=20, disp=2.0, rot=0.01)
    grains = wl.place(p, 31)
    ng = grains["cx"].shape[0]
    rng = np.random.default_rng(5)
    frames = []
    dx = np.zeros(ng)
    dy = np.zeros(ng)
    th = np.zeros(ng)
    for k in range(4):
        frames.append(wl.render(p, grains, dx, dy, th, noise_seed=100 + k))
        dx = dx + rng.uniform(-2, 2, ng)
        dy = dy + rng.uniform(-2, 2, ng)
        th = th + rng.uniform(-0.01, 0.01, ng)
    rec = wl.start_records(grains)
    pair = dict(params=p, ref=frames[0], cur=frames[1], rec=rec)
    opts = _opts(wl, pair, iraz=0)
    g = _gpu(ptk, pair, opts, iraz=0)
    c = _cpu(oracle, pair, opts, iraz=0)
    for k in range(1, 4):
        if k > 1:
            g.load_frame(1, frames[k])
            c.load_current(frames[k])
        g.track_frame(k)
        c.track_frame(k)
        gr, cr = g.get_grains(), c.get_grains()
        np.testing.assert_array_equal(gr[:, 0:2], cr[:, 0:2])
        assert np.abs(gr[:, 4:6] - cr[:, 4:6]).max() <= SUBPIX_TOL_PX
        assert np.abs(gr[:, 2] + gr[:, 6] - cr[:, 2] - cr[:, 6]).max() <= SUBPIX_TOL_RAD


def test_no_rotation_mode(ptk, wl, oracle, cuda_device, pair_cache):
    pair = pair_cache("tiny", 9)
    opts = _opts(wl, pair, rotations=0)
    g = _gpu(ptk, pair, opts)
    g.precompute()
    g.search(0)
    c = _cpu(oracle, pair, dict(opts, zones=[(4, 4, 4, 4, 0, 1.0), None, None]))
    c.precompute()
    c.pixel_all()
    assert_pixel_parity(g.get_grains(), c.get_grains(), c.top2())


@pytest.mark.parametrize("dups", [1, 3, 9], ids=["unique", "few_repeats", "many_repeats"])
def test_custom_patterns(ptk, wl, oracle, cuda_device, pair_cache, dups):
    """Sparse random patterns (many multiplicity runs per column, exercising the
    tiled kernel's entry-by-entry path) and repeated offsets (beyond 4 repeats
    the direct kernel is used)."""
    pair = pair_cache("tiny", 5)
    rng = np.random.default_rng(3 + dups)
    pats = []
    for _ in range(pair["rec"].shape[0]):
        k = rng.integers(20, 120)
        base = np.stack([rng.integers(-8, 9, k), rng.integers(-8, 9, k)], 1).astype(np.int32)
        pats.append(np.concatenate([base] + [base[:5]] * (dups - 1)) if dups > 1 else base)
    opts = _opts(wl, pair)
    g = _gpu(ptk, pair, opts, pattern=("patterns", pats))
    g.precompute()
    g.search(0)
    c = _cpu(oracle, pair, opts, pattern=("patterns", pats))
    c.precompute()
    c.pixel_all()
    assert_pixel_parity(g.get_grains(), c.get_grains(), c.top2())
