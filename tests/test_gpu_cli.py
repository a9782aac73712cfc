"""The command-file driver (ptracker_b200) end to end on the GPU: a short
sequence of frame files tracked through the reference's command tokens, every
dic_out_<n>.txt compared with the CPU oracle run on the same grey levels.

Plain form (8-bit TIFF frames, reference change after every frame): same
integer positions, subpixel within 1e-3 px / 1e-4 rad.  BF16 search + adjoint
LM (16-bit PGM frames, reference kept): same integer positions, within
0.01 px / 1e-4 rad of the FP64 oracle."""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from imagefiles import reference_grey, write_pgm, write_tiff

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))


def _sequence(wl, p, seed, frames=4, step=1.5, rot=0.008):
    grains = wl.place(p, seed)
    ng = grains["cx"].shape[0]
    rng = np.random.default_rng(seed + 1)
    out, dx, dy, th = [], np.zeros(ng), np.zeros(ng), np.zeros(ng)
    for k in range(frames):
        out.append(wl.render(p, grains, dx, dy, th, noise_seed=seed * 10 + k))
        dx = dx + rng.uniform(-step, step, ng)
        dy = dy + rng.uniform(-step, step, ng)
        th = th + rng.uniform(-rot, rot, ng)
    return grains, out


def _zone_tokens(zones):
    names = ["search_zone", "search_zone_rescue", "search_zone_super_rescue"]
    lines = []
    for lvl, z in enumerate(zones):
        if z is None:
            continue
        for key, v in zip(["left", "right", "up", "down", "num_rot", "inc_rot"], z):
            lines.append(f"{names[lvl]}.{key} {v}")
    return "\n".join(lines)


def _run(ptk, tmp_path, commands: str):
    (tmp_path / "commands.txt").write_text(commands)
    r = subprocess.run([str(ptk.cli_path()), "commands.txt"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def _start_file(path, grains):
    with open(path, "w") as f:
        f.write(f"{grains['cx'].shape[0]}\n")
        for x, y, r in zip(grains["cx"], grains["cy"], grains["r"]):
            f.write(f"{float(x)!r} {float(y)!r} 0.0 {float(r)!r}\n")


def _oracle(oracle, p, frames16, rec, zones, params):
    pair = dict(params=p, ref=frames16[0], cur=frames16[1], rec=rec)
    return oracle.setup(oracle.Port, pair, threads=THREADS, zones=zones, params=params)


def test_cli_plain_sequence_tiff(ptk, wl, oracle, cuda_device, tmp_path):
    p = dict(wl.PRESETS["tiny"])
    grains, frames = _sequence(wl, p, 61)
    for k, f in enumerate(frames):
        write_tiff(tmp_path / f"frame_{k}.tif", f.astype(np.uint8), datetime=f"2024:01:01 00:00:0{k}")
    grey = [reference_grey(f.astype(np.uint8), f.astype(np.uint8), f.astype(np.uint8)) for f in frames]
    _start_file(tmp_path / "start.txt", grains)
    o = wl.tracker_options(p)
    out = _run(ptk, tmp_path, f"""image_name frame_%d.tif
grains_to_follow start.txt
iref 0 ibeg 1 iend {len(frames) - 1} iinc 1 iraz 0
rescue_level {o['rescue_level']} NCC_min {o['NCC_min']}
{_zone_tokens(o['zones'])}
pattern grain_diameter 1.0 1.0
""")
    assert "dic_out_3.txt written" in out
    rec = ptk.read_grains_file(str(tmp_path / "start.txt"), format13=False)
    c = _oracle(oracle, p, grey, rec, o["zones"], {"rescue_level": o["rescue_level"], "NCC_min": o["NCC_min"],
                                                   "iraz": 0})
    for k in range(1, len(frames)):
        if k > 1:
            c.load_current(grey[k])
        c.track_frame(k)
        cr = c.get_grains()
        gr = ptk.read_grains_file(str(tmp_path / f"dic_out_{k}.txt"), format13=True)
        np.testing.assert_array_equal(gr[:, 0:2], cr[:, 0:2])
        assert np.abs(gr[:, 4:6] - cr[:, 4:6]).max() <= 1e-3
        assert np.abs(gr[:, 2] + gr[:, 6] - cr[:, 2] - cr[:, 6]).max() <= 1e-4
        text = (tmp_path / f"dic_out_{k}.txt").read_text().splitlines()
        assert text[-4:] == [f"#_FROM_image: frame_{k - 1}.tif", f"#___dateTime: 2024:01:01 00:00:0{k - 1}",
                             f"#___TO_image: frame_{k}.tif", f"#___dateTime: 2024:01:01 00:00:0{k}"]


def test_cli_bf16_lm_sequence_pgm_with_mask(ptk, wl, oracle, cuda_device, tmp_path):
    p = dict(wl.PRESETS["small16"], n=24)
    grains, frames = _sequence(wl, p, 62, frames=3, step=2.0)
    for k, f in enumerate(frames):
        write_pgm(tmp_path / f"f{k:03d}.pgm", f.astype(np.uint16))
    _start_file(tmp_path / "start.txt", grains)
    o = wl.tracker_options(p)
    rec = ptk.read_grains_file(str(tmp_path / "start.txt"), format13=False)
    # mask the grains of the left quarter of the frame
    x_mask = p["dimx"] // 4
    _run(ptk, tmp_path, f"""image_name f%03d.pgm
start_file start.txt
iref 0 ibeg 1 iend 2 iinc 1 iraz 1000
rescue_level {o['rescue_level']}
{_zone_tokens(o['zones'])}
pattern grain_diameter 1.0 1.0
mask_rect 0 {x_mask} 0 {p['dimy']}
search_method bf16
subpix_method adjoint_lm
""")
    masked = rec[:, 0] <= x_mask
    assert masked.any() and (~masked).any()
    c = _oracle(oracle, p, [f.astype(np.uint16) for f in frames], rec, o["zones"],
                {"rescue_level": o["rescue_level"], "NCC_min": o["NCC_min"], "iraz": 1000})
    c.set_grains(rec, masked.astype(np.uint8))
    for k in (1, 2):
        if k > 1:
            c.load_current(frames[k].astype(np.uint16))
        c.track_frame(k)
        cr = c.get_grains()
        gr = ptk.read_grains_file(str(tmp_path / f"dic_out_{k}.txt"), format13=True)
        np.testing.assert_array_equal(gr[:, 0:2], cr[:, 0:2])
        assert np.abs(gr[:, 4:6] - cr[:, 4:6]).max() <= 0.01
        assert np.abs(gr[:, 6] - cr[:, 6]).max() <= 1e-4
        # masked grains do not move (the file keeps 15 significant digits)
        assert np.abs(gr[masked][:, 4:7] - rec[masked][:, 4:7]).max() <= 1e-12
