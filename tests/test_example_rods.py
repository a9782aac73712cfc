"""The reference's shipped example (examples/ParticleImageTracking: 9 rods
between TEST01.tiff and TEST02.tiff) on the CPU: the oracle's restatement
reproduces the reference's own tracking of it (tests/golden/example_rods.npz,
made by tests/golden/make_golden.py --example-only) bit for bit, and, where
the reference tree is present, this library's TIFF and grain-file readers
give the fixture's inputs from the example's own LZW files."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden"
ZONES = [(6, 6, 6, 6, 6, 0.0454), (30, 30, 30, 30, 69, 0.0454), (200, 200, 200, 200, 69, 0.045)]
PARAMS = {"rescue_level": 2, "NCC_min": 0.8, "NCC_min_super": 0.7, "iraz": 20000}


def test_port_reproduces_reference_example(oracle):
    g = np.load(GOLD / "example_rods.npz")
    pair = dict(params=dict(dimx=g["frame1"].shape[1], dimy=g["frame1"].shape[0]), ref=g["frame1"],
                cur=g["frame1"], rec=g["rec"])
    c = oracle.setup(oracle.Port, pair, threads=4, zones=ZONES, params=PARAMS, pattern=("circ", 10))
    c.track_frame(1)
    np.testing.assert_array_equal(c.get_grains(), g["grains1"])
    c.load_current(g["frame2"])
    c.track_frame(2)
    np.testing.assert_array_equal(c.get_grains(), g["grains2"])
    res, sup = c.lists()
    assert list(res) == list(g["rescued2"]) == [4] and list(sup) == []
    c.close()


def test_readers_on_the_example_files(ptk, oracle):
    ex = oracle.REF_SRC.parent / "examples"
    if not (ex / "ImageData" / "TEST01.tiff").exists():
        pytest.skip("reference example files not present")
    g = np.load(GOLD / "example_rods.npz")
    for k in (1, 2):
        frame, _ = ptk.read_image_file(str(ex / "ImageData" / f"TEST{k:02d}.tiff"))
        np.testing.assert_array_equal(frame, g[f"frame{k}"])
    rec = ptk.read_grains_file(str(ex / "ParticleImageTracking" / "recentered.data"), format13=False)
    np.testing.assert_array_equal(rec, g["rec"])
