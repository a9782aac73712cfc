"""The CPU oracle (oracle/port) pinned against the compiled reference.

Golden fixtures in tests/golden were produced by the reference's own tracking
code (tests/golden/make_golden.py, oracle/_ref); the port must reproduce every
stored value bit for bit.  Where the compiled reference is available, extra
randomised cases compare the two live."""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
GOLD = HERE / "golden"
sys.path.insert(0, str(GOLD))
mk = importlib.import_module("make_golden")


def _pair_from_fixture(name):
    d = np.load(GOLD / f"{name}.npz")
    p = dict(dimx=d["ref"].shape[1], dimy=d["ref"].shape[0], maxval=int(d["maxval"][0]))
    return d, dict(params=p, ref=d["ref"], cur=d["cur"], rec=d["rec"])


@pytest.mark.parametrize("name", list(mk.CASES))
def test_port_reproduces_golden_bitwise(oracle, name):
    c = mk.CASES[name]
    d, pair = _pair_from_fixture(name)
    t, out = mk.run_case(oracle.Port, pair, c)
    np.testing.assert_array_equal(out["grains"], d["grains"])
    for k in ("nres", "nsup", "rescued", "super_rescued", "mean0", "C0C0", "pattern0_g0"):
        if k in d.files:
            np.testing.assert_array_equal(out[k], d[k], err_msg=k)


def test_rescue_fixture_exercises_both_levels():
    d = np.load(GOLD / "rescue_small.npz")
    assert d["nres"][0] > 0 and d["nsup"][0] > 0


def test_interpolators_and_objective_golden(oracle):
    d = np.load(GOLD / "numerics.npz")
    c = mk.CASES["frame_small"]
    _, pair = _pair_from_fixture("frame_small")
    t = oracle.setup(oracle.Port, pair, threads=1, zones=c["zones"], params=c["params"])
    t.precompute()
    for k in range(3):
        got = np.array([t.interp(k, 1, x, y) for (x, y) in d["interp_pts"]])
        np.testing.assert_array_equal(got, d["interp_vals"][k])
    got = np.array([t.objective(g, d["obj_X"][g]) for g in range(t.n)])
    np.testing.assert_array_equal(got, d["obj_vals"])


def test_undistor_golden(oracle):
    d = np.load(GOLD / "numerics.npz")
    for k in range(d["undistor_params"].shape[0]):
        for j in range(d["undistor_pts"].shape[1]):
            got = oracle.undistor(d["undistor_params"][k], *d["undistor_pts"][k, j])
            np.testing.assert_array_equal(np.array(got), d["undistor_vals"][k, j])


def test_patterns_golden(oracle):
    d = np.load(GOLD / "patterns.npz")
    t = oracle.Port(64, 64, 1)
    t.set_grains(np.zeros((1, 13)))
    for key in d.files:
        kind, *args = key.split("_")
        t.make_pattern(0, {"circ": 0, "ring": 1, "rect": 2}[kind], *map(int, args))
        np.testing.assert_array_equal(t.pattern(0, 0), d[key], err_msg=key)


def test_rotation_steps_golden_and_counts(oracle):
    d = np.load(GOLD / "rotation_steps.npz")
    for key in d.files:
        inc = float(key.split("_")[0][3:])
        num = int(key.split("_")[1][3:])
        np.testing.assert_array_equal(oracle.rotation_steps(inc, num), d[key])
    # the loop's step count is not always 2 num + 1 (accumulated FP64 sums)
    assert len(oracle.rotation_steps(0.005, 10)) == 21
    assert len(oracle.rotation_steps(0.005, 4)) == 8
    assert len(oracle.rotation_steps(0.0025, 20)) == 40


def test_save_grains_golden(oracle, tmp_path):
    d, pair = _pair_from_fixture("frame_small")
    t = oracle.Port(pair["params"]["dimx"], pair["params"]["dimy"], 1)
    t.set_grains(d["grains"])
    out = tmp_path / "dic_out_1.txt"
    t.save_grains(str(out), "image0.tiff", "image1.tiff")
    assert out.read_bytes() == (GOLD / "dic_out_frame_small.txt").read_bytes()


def test_powell_finds_quadratic_minimum(oracle):
    # the objective of a grain against its own reference frame is minimal at X = 0
    _, pair = _pair_from_fixture("frame_small")
    same = dict(pair, cur=pair["ref"])
    c = mk.CASES["frame_small"]
    t = oracle.setup(oracle.Port, same, threads=4, zones=c["zones"], params=c["params"])
    rec = same["rec"].copy()
    rec[:, 4:6] = 0.0  # anchor exactly on refcoord
    t.set_grains(rec)
    t.precompute()
    t.subpixel_all()
    out = t.get_grains()
    assert np.abs(out[:, 4:6] - rec[:, 4:6]).max() < 1e-4
    assert np.abs(out[:, 6]).max() < 1e-5
    assert out[:, 12].min() > 1 - 1e-9


reference = pytest.mark.skipif(not Path(__file__).resolve().parents[1].joinpath("oracle/_ref/libptk_ref.so").exists(),
                               reason="compiled reference not built")


@reference
@pytest.mark.parametrize("seed", [31, 32])
def test_port_equals_reference_live(oracle, wl, seed):
    p = dict(wl.PRESETS["small16"], dimx=240, dimy=200, n=8, disp=3.0, rot=0.03)
    pair = wl.make_pair(p, seed=seed)
    rec = pair["rec"].copy()
    rec[:, 2] = np.linspace(-0.4, 0.4, rec.shape[0])  # nonzero refrot
    pair = dict(pair, rec=rec)
    masked = np.zeros(rec.shape[0], np.uint8)
    masked[1] = 1
    outs = []
    for cls in (oracle.Port, oracle.Reference):
        t = oracle.setup(cls, pair, threads=4, zones=[(4, 3, 2, 5, 3, 0.02)],
                         params={"rescue_level": 0, "iraz": 0, "image_interpolator": seed % 3})
        t.set_grains(rec, masked)
        if cls is oracle.Reference:  # its set_grains drops patterns; the port keeps them
            t.grain_diameter_patterns(rec)
        t.track_frame(1)
        outs.append((t.get_grains(), t.indices()))
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    assert outs[0][1] == outs[1][1]
