"""The reference's shipped example (9 rods, TEST01 -> TEST02, rescue of the
rod that moved 9.8 px beyond the +-6 px zone) on the GPU, against the
reference's own tracking of it (tests/golden/example_rods.npz): through the
library in the plain form (same integer results, subpixel within 1e-3 px /
1e-4 rad) and the BF16 + adjoint-LM form (within 0.01 px / 1e-4 rad), and
through the command-file driver with the example's settings."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from imagefiles import write_pgm

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
ZONES = [(6, 6, 6, 6, 6, 0.0454), (30, 30, 30, 30, 69, 0.0454), (200, 200, 200, 200, 69, 0.045)]


def _check(got, want, px, rad):
    np.testing.assert_array_equal(got[:, 0:4], want[:, 0:4])
    assert np.abs(got[:, 4:6] - want[:, 4:6]).max() <= px
    assert np.abs(got[:, 6] - want[:, 6]).max() <= rad
    # pixel-stage NCC (exact integer sums here, FP64 two-pass in the reference) and the rescue's
    assert np.abs(got[:, 10:12] - want[:, 10:12]).max() <= 1e-9


@pytest.mark.parametrize("form,px", [({}, 1e-3), ({"search_method": 1, "subpix_method": 1}, 0.01)])
def test_library_on_example(ptk, cuda_device, form, px):
    g = np.load(GOLD / "example_rods.npz")
    h, w = g["frame1"].shape
    t = ptk.Tracker(w, h, rescue_level=2, NCC_min=0.8, NCC_min_super=0.7, iraz=20000, **form)
    for lvl, z in enumerate(ZONES):
        t.set_zone(lvl, *z)
    t.set_grains(g["rec"])
    t.make_patterns("circ", 10)
    t.set_iref(1)
    t.load_frame(0, g["frame1"])
    t.load_frame(1, g["frame1"])
    t.track_frame(1)
    _check(t.get_grains(), g["grains1"], px, 1e-4)
    t.load_frame(1, g["frame2"])
    t.track_frame(2)
    _check(t.get_grains(), g["grains2"], px, 1e-4)
    assert t.rescue_counts() == (1, 0)
    t.close()


def test_driver_on_example(ptk, cuda_device, tmp_path):
    g = np.load(GOLD / "example_rods.npz")
    for k in (1, 2):
        write_pgm(tmp_path / f"TEST{k:02d}.pgm", g[f"frame{k}"])
    rec = g["rec"]
    with open(tmp_path / "start.txt", "w") as f:  # the 4-column form: position, rotation, radius
        f.write(f"{rec.shape[0]}\n")
        for r in rec:
            f.write(f"{float(r[0] + r[4])!r} {float(r[1] + r[5])!r} {float(r[2])!r} {float(r[3])!r}\n")
    zone_lines = []
    for name, z in zip(["search_zone", "search_zone_rescue", "search_zone_super_rescue"], ZONES):
        for key, v in zip(["left", "right", "up", "down", "num_rot", "inc_rot"], z):
            zone_lines.append(f"{name}.{key} {v}")
    zl = "\n".join(zone_lines)
    (tmp_path / "commands.txt").write_text(f"""procedure particle_tracking
wanted_num_threads 8
image_name TEST%02d.pgm
grains_to_follow start.txt
iref 1 ibeg 1 iend 2 iinc 1 iraz 20000
rotations 1 subpixel 1 subpix_tol 1.e-8
initial_direction_dx 0.01 initial_direction_dy 0.01 initial_direction_dr 0.01
image_interpolator cubic overflow_stiffness 0.0 subpix_displacement_max 3.0
rescue_level 2 use_neighbour_list 1
NCC_min 0.8 NCC_min_super 0.7
{zl}
pattern circ 10
""")
    r = subprocess.run([str(ptk.cli_path()), "commands.txt"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for k in (1, 2):
        got = ptk.read_grains_file(str(tmp_path / f"dic_out_{k}.txt"), format13=True)
        want = g[f"grains{k}"]
        np.testing.assert_array_equal(got[:, 0:2], want[:, 0:2])
        assert np.abs(got[:, 4:6] - want[:, 4:6]).max() <= 1e-3
        assert np.abs(got[:, 6] - want[:, 6]).max() <= 1e-4
