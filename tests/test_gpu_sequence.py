"""The full-sequence configuration in miniature: a cfg5-style sequence (shear
field, per-grain rotation walks, jumps that force the +-40 px rescue search,
radial lens distortion corrected by the on-device remap) tracked frame after
frame with a reference change after every frame, against the CPU oracle fed
the same remapped frames (the remap is bit-exact to the oracle's).

Headline form (BF16 search + adjoint LM): same integer positions and rescue
counts as the oracle's exact search, positions within 0.01 px and rotations
within 1e-4 rad of its FP64 Powell.  Plain form: within 1e-5 px / 1e-6 rad
(its objective is the reference's bit for bit wherever the C library's cos /
sin are correctly rounded, so Powell takes the reference's path)."""
from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))


@pytest.fixture(scope="module")
def seq(wl):
    p = dict(wl.PRESETS["cfg5"], dimx=1536, dimy=1024, n=80, shear=20.0, jump_frac=0.1)
    s = wl.make_sequence(p, seed=7, frames=5)
    assert s["jumpers"].any(), "the sequence must contain jumps (rescue searches)"
    return s


@pytest.fixture(scope="module")
def long_seq(wl):
    """24 frames (23 reference changes) of the same kind."""
    p = dict(wl.PRESETS["cfg5"], dimx=1536, dimy=1024, n=80, shear=30.0, jump_frac=0.05)
    return wl.make_sequence(p, seed=11, frames=24)


def _track(ptk, wl, oracle, s, tol_px, tol_rad=1e-4, **form):
    p = s["params"]
    o = wl.tracker_options(p)
    X = s["disto"]
    frames = s["frames"]
    remapped = [oracle.remap(X, f, threads=THREADS) for f in frames]
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=o["rescue_level"], NCC_min=o["NCC_min"], iraz=0, **form)
    for lvl, z in enumerate(o["zones"]):
        if z is not None:
            t.set_zone(lvl, *z)
    t.set_grains(s["rec"])
    t.make_patterns("grain_diameter", 1.0, 1.0)
    t.set_distortion(X)
    t.load_frame(0, frames[0])
    t.remap(0)
    pair = dict(params=p, ref=remapped[0], cur=remapped[1], rec=s["rec"])
    c = oracle.setup(oracle.Port, pair, threads=THREADS, zones=o["zones"],
                     params={"rescue_level": o["rescue_level"], "NCC_min": o["NCC_min"], "iraz": 0})
    rescued = 0
    for k in range(1, len(frames)):
        t.load_frame(1, frames[k])
        t.remap(1)
        t.track_frame(k)
        if k > 1:
            c.load_current(remapped[k])
        c.track_frame(k)
        gr, cr = t.get_grains(), c.get_grains()
        res, _ = c.lists()
        assert t.rescue_counts()[0] == len(res), f"frame {k}: rescue count"
        rescued += len(res)
        np.testing.assert_array_equal(gr[:, 0:2], cr[:, 0:2])
        assert np.abs(gr[:, 4:6] - cr[:, 4:6]).max() <= tol_px, f"frame {k}"
        assert np.abs(gr[:, 2] + gr[:, 6] - cr[:, 2] - cr[:, 6]).max() <= tol_rad, f"frame {k}"
    assert rescued > 0, "the jumps must trigger rescue searches"
    return t


def test_sequence_headline_form(ptk, wl, oracle, cuda_device, seq):
    _track(ptk, wl, oracle, seq, 0.01, search_method=ptk.SEARCH_BF16, subpix_method=ptk.SUBPIX_ADJOINT_LM)


def test_sequence_plain_form(ptk, wl, oracle, cuda_device, seq):
    _track(ptk, wl, oracle, seq, 1e-5, 1e-6)


def test_long_sequence_plain_form(ptk, wl, oracle, cuda_device, long_seq):
    """The plain form along 23 reference changes: every grain-frame within
    1e-5 px and 1e-6 rad of the oracle (the device objective and Powell repeat
    the reference's operations, so the two trajectories do not drift apart)."""
    _track(ptk, wl, oracle, long_seq, 1e-5, 1e-6)
