"""The C ABI library on CPU: it loads, exports every entry point include/ptk.h
declares, agrees with the binding on struct layouts, fails loudly without a
GPU, and its host-only grain-file functions follow the reference format."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden"


def declared_functions() -> list[str]:
    text = (ROOT / "include" / "ptk.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ptk_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported(ptk):
    L = ptk.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(ptk.exported_symbols()), "binding signatures out of date"


def test_struct_layouts_match(ptk):
    cfg, grain, zone = ptk.abi_sizes()
    assert cfg == C.sizeof(ptk.Config)
    assert grain == C.sizeof(ptk.Grain) == ptk.GRAIN_DTYPE.itemsize
    assert zone == C.sizeof(ptk.Zone)


def test_config_defaults_follow_reference(ptk):
    cfg = ptk.default_config(100, 80)
    # src/p-tracker.hpp:67-178
    assert cfg.rescue_level == 2 and cfg.NCC_min == 0.7 and cfg.NCC_min_super == 0.5
    assert cfg.subpixel == 1 and cfg.subpix_tol == 1e-8
    assert list(cfg.initial_direction) == [0.01, 0.01, 0.01]
    assert cfg.image_interpolator == ptk.INTERP["cubic"]
    assert cfg.subpix_displacement_max == 3.0 and cfg.overflow_stiffness == 0.0
    assert cfg.rotations == 1 and cfg.iraz == 0


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_cuda(), reason="checks the no-GPU failure path")
def test_create_fails_loudly_without_gpu(ptk):
    with pytest.raises(ptk.PtkError) as e:
        ptk.Tracker(64, 64)
    assert e.value.code == ptk.PTK_ERR_CUDA


def test_create_rejects_bad_sizes(ptk):
    with pytest.raises(ptk.PtkError) as e:
        ptk.Tracker(2, 64)
    assert e.value.code == ptk.PTK_ERR_ARG


def test_save_grains_file_matches_reference_bytes(ptk, tmp_path):
    d = np.load(GOLD / "frame_small.npz")
    out = tmp_path / "dic_out_1.txt"
    ptk.save_grains_file(str(out), d["grains"], from_image="image0.tiff", to_image="image1.tiff")
    assert out.read_bytes() == (GOLD / "dic_out_frame_small.txt").read_bytes()


def test_read_grains_file_13_columns(ptk):
    d = np.load(GOLD / "frame_small.npz")
    rec = ptk.read_grains_file(str(GOLD / "dic_out_frame_small.txt"), format13=True)
    np.testing.assert_array_equal(rec[:, :2], d["grains"][:, :2])
    np.testing.assert_allclose(rec[:, 2:], d["grains"][:, 2:], rtol=1e-14, atol=0)


def test_read_grains_file_4_columns(ptk, tmp_path):
    # grains_to_follow semantics (src/p-tracker.cpp:1253-1272)
    f = tmp_path / "start.txt"
    f.write_text("3\n231.192 132.667 0 71.7888\n143.978 200.569 0.5 28.8994\n10 20 0 5\n")
    rec = ptk.read_grains_file(str(f), format13=False)
    np.testing.assert_array_equal(rec[:, 0], [231, 143, 10])
    np.testing.assert_array_equal(rec[:, 1], [132, 200, 20])
    np.testing.assert_allclose(rec[:, 4], [0.192, 0.978, 0.0], atol=1e-12)
    np.testing.assert_array_equal(rec[:, 4], rec[:, 7])
    np.testing.assert_array_equal(rec[:, 5], rec[:, 8])
    np.testing.assert_array_equal(rec[:, 2], [0, 0.5, 0])
    np.testing.assert_array_equal(rec[:, 3], [71.7888, 28.8994, 5])


def test_read_grains_file_errors(ptk, tmp_path):
    with pytest.raises(ptk.PtkError):
        ptk.read_grains_file(str(tmp_path / "missing.txt"))
    bad = tmp_path / "bad.txt"
    bad.write_text("2\n1 2 3\n")
    with pytest.raises(ptk.PtkError):
        ptk.read_grains_file(str(bad), format13=False)
