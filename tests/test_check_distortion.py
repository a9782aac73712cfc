"""procedure check_distortion of the command-file driver (CPU; the procedure
needs no GPU): len_variation.txt from a set of dic files, against the
reference's own ptracker::check_distortion (src/check_distortion.cpp:25-100)
run by the oracle on copies of the same files."""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess

import numpy as np
import pytest

NAMES = ["xc_corrDistor", "yc_corrDistor", "K1_corrDistor", "K2_corrDistor", "K3_corrDistor", "P1_corrDistor",
         "P2_corrDistor", "P3_corrDistor", "xc_corrParallax", "yc_corrParallax", "angle1_corrParallax",
         "A1_corrParallax", "angle2_corrParallax", "A2_corrParallax"]


def _dic_files(ptk, where, n=40, files=4, seed=3):
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, 13))
    rec[:, 0] = rng.integers(50, 950, n)
    rec[:, 1] = rng.integers(50, 700, n)
    rec[:, 3] = rng.uniform(10, 20, n)
    for k in range(files):
        r = rec.copy()
        r[:, 4] = rng.normal(0.0, 0.3, n) + 0.8 * k  # a drift plus noise, as tracked positions
        r[:, 5] = rng.normal(0.0, 0.3, n) - 0.5 * k
        r[:, 6] = rng.normal(0.0, 0.01, n)
        r[:, 10:13] = 0.95
        ptk.save_grains_file(str(where / f"d_{k}.txt"), r, "a.tif", "b.tif")


@pytest.mark.parametrize("params", [
    [500.0, 380.0, -3e-8, 2e-14, 0.0, 1e-6, -2e-6, 0.0, 480.0, 360.0, 0.1, 0.002, -0.05, 0.001],
    [-1.0, -1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, -1.0, -1.0, 0.0, 0.0, 0.0, 0.0],
])
def test_len_variation_matches_reference(ptk, oracle, tmp_path, params):
    if not oracle.have_reference():
        pytest.skip("compiled reference not built here")
    mine = tmp_path / "mine"
    ref = tmp_path / "ref"
    mine.mkdir()
    _dic_files(ptk, mine)
    shutil.copytree(mine, ref)
    tokens = "\n".join(f"{nm} {v!r}" for nm, v in zip(NAMES, params))
    (mine / "commands.txt").write_text(f"""procedure check_distortion
dic_name d_%d.txt
iref 0 ibeg 1 iend 3 iinc 1
{tokens}
""")
    r = subprocess.run([str(ptk.cli_path()), "commands.txt"], capture_output=True, text=True, cwd=mine, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    L = C.CDLL(str(oracle.REF_SO))
    L.ref_create.restype = C.c_void_p
    h = C.c_void_p(L.ref_create(8, 8))
    P = np.ascontiguousarray(params, dtype=np.float64)
    import os
    cwd = os.getcwd()
    try:
        os.chdir(ref)
        L.ref_check_distortion(h, b"d_%d.txt", 0, 1, 3, 1, P.ctypes.data_as(C.c_void_p))
    finally:
        os.chdir(cwd)
        L.ref_destroy(h)
    got = (mine / "len_variation.txt").read_text()
    want = (ref / "len_variation.txt").read_text()
    assert got == want
    assert len(got.splitlines()) == 3


def test_odd_grain_count_and_bad_step(ptk, tmp_path):
    _dic_files(ptk, tmp_path, n=41, files=2)
    (tmp_path / "commands.txt").write_text("procedure check_distortion\ndic_name d_%d.txt\niref 0 ibeg 1 iend 1 iinc 1\n")
    r = subprocess.run([str(ptk.cli_path()), "commands.txt"], capture_output=True, text=True, cwd=tmp_path, timeout=60)
    assert r.returncode == 0, r.stderr
    line = (tmp_path / "len_variation.txt").read_text().split()
    assert line[0] == "1" and len(line) == 3
    (tmp_path / "commands.txt").write_text("procedure check_distortion\ndic_name d_%d.txt\niref 0 ibeg 1 iend 1 iinc 0\n")
    r = subprocess.run([str(ptk.cli_path()), "commands.txt"], capture_output=True, text=True, cwd=tmp_path, timeout=60)
    assert r.returncode != 0 and "iinc" in (r.stdout + r.stderr)
