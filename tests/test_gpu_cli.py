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


def test_cli_correction_distortion(ptk, wl, oracle, cuda_device, tmp_path):
    """procedure correction_distortion end to end: frames of translated grains
    seen through radial distortion, tracked from image 0 into images 1 and 2
    (compared with the oracle's pixel search + Powell from the same imposed
    displacements), then the POWELL fit of K1 (compared with the oracle's fit
    on the oracle's tracked displacements) and the output files."""
    from disto_cases import params
    p = dict(wl.PRESETS["small16"], dimx=1024, dimy=768, n=60, disp=0.0, rot=0.0, zone=6, disto=(-3e-8, 0.0))
    X = params(p["dimx"], p["dimy"], -3e-8, 0.0)
    grains = wl.place(p, 71)
    ng = grains["cx"].shape[0]
    shifts = [(0.0, 0.0), (6.3, -4.1), (-7.4, 5.2)]
    imposed = [(0.0, 0.0), (6.0, -4.0), (-7.0, 5.0)]
    frames = []
    for k, (tx, ty) in enumerate(shifts):
        f = wl.render(p, grains, np.full(ng, tx), np.full(ng, ty), np.zeros(ng), noise_seed=710 + k, disto=X)
        frames.append(f)
        write_pgm(tmp_path / f"f{k}.pgm", f.astype(np.uint16))
    L = oracle.C.CDLL(str(oracle.PORT_SO))
    with open(tmp_path / "start.txt", "w") as fh:
        fh.write(f"{ng}\n")
        for x, y, r in zip(grains["cx"], grains["cy"], grains["r"]):
            xd, yd = oracle.C.c_double(), oracle.C.c_double()
            L.orc_distort_point(oracle._p(X), oracle._D(float(x)), oracle._D(float(y)), oracle.C.byref(xd),
                                oracle.C.byref(yd))
            fh.write(f"{xd.value!r} {yd.value!r} 0.0 {float(r)!r}\n")
    perturb = " ".join(f"d{nm} 0" for nm in ("xc_corrDistor", "yc_corrDistor", "K2_corrDistor", "K3_corrDistor",
                                            "P1_corrDistor", "P2_corrDistor", "P3_corrDistor", "xc_corrParallax",
                                            "yc_corrParallax", "angle1_corrParallax", "A1_corrParallax",
                                            "angle2_corrParallax", "A2_corrParallax"))
    z = (6, 6, 6, 6, 2, 0.005)
    out = _run(ptk, tmp_path, f"""procedure correction_distortion
image_name f%d.pgm
start_file start.txt
image_numbers_corrDisto 3 0 1 2
imposedDisplApprox_corrDisto 6 -4 -7 5
equiProj_dist_range 100 700
NCC_min 0.7
{_zone_tokens([z])}
pattern grain_diameter 1.0 1.0
optim_algo POWELL
dK1_corrDistor 1e-9 {perturb}
""")
    assert "Number of points for equiprojectivity computations" in out
    rec = ptk.read_grains_file(str(tmp_path / "start.txt"), format13=False)
    pair = dict(params=p, ref=frames[0].astype(np.uint16), cur=frames[1].astype(np.uint16), rec=rec)
    c = oracle.setup(oracle.Port, pair, threads=THREADS, zones=[z], params={"rescue_level": 0, "NCC_min": 0.7})
    state = rec.copy()
    dx, dy, ncc = np.zeros((2, ng)), np.zeros((2, ng)), np.zeros((2, ng))
    for k in (1, 2):
        if k > 1:
            c.load_current(frames[k].astype(np.uint16))
        state[:, 4], state[:, 5] = imposed[k]  # every search starts from the imposed displacement
        c.set_grains(state)
        c.grain_diameter_patterns(state, 1.0, 1.0)
        c.precompute()
        c.pixel_all()
        c.subpixel_all()
        cr = c.get_grains()
        gr = ptk.read_grains_file(str(tmp_path / f"dic_out_{k}.txt"), format13=True)
        np.testing.assert_array_equal(gr[:, 0:2], cr[:, 0:2])
        assert np.abs(gr[:, 4:6] - cr[:, 4:6]).max() <= 1e-3
        assert np.abs(gr[:, 6] - cr[:, 6]).max() <= 1e-4
        dx[k - 1], dy[k - 1], ncc[k - 1] = cr[:, 4], cr[:, 5], cr[:, 12]
        state = cr.copy()
    log = dict()
    for line in (tmp_path / "corrDisto_log.txt").read_text().splitlines():
        key, _, val = line.rpartition(" ")
        log[key.strip()] = float(val)
    refx, refy = rec[:, 0].astype(np.int32), rec[:, 1].astype(np.int32)
    pairs = oracle.disto_pairs(refx, refy, 100.0, 700.0)
    X0 = np.zeros(14)
    X0[0] = X0[1] = X0[8] = X0[9] = -1.0
    DX = np.zeros(14)
    DX[2] = 1e-9
    # the fit stage: the oracle's Powell on the displacements the driver wrote
    cols = [ptk.read_grains_file(str(tmp_path / f"dic_out_{k}.txt"), format13=True) for k in (1, 2)]
    gdx = np.stack([r[:, 4] for r in cols])
    gdy = np.stack([r[:, 5] for r in cols])
    gncc = np.stack([r[:, 12] for r in cols])
    fx, fini, fend, _, _, _ = oracle.disto_fit(X0, DX, 0, 0, p["dimx"], p["dimy"], refx, refy, gdx, gdy, gncc, 0.7,
                                               pairs)
    np.testing.assert_allclose(log["Initial distorsion index"], fini, rtol=1e-9)
    np.testing.assert_allclose(log["Final distorsion index"], fend, rtol=1e-6)
    np.testing.assert_allclose(log["K1_corrDistor"], fx[2], rtol=1e-6)
    # tracking + fit: the oracle end to end, and the distortion the frames were rendered with
    ox = oracle.disto_fit(X0, DX, 0, 0, p["dimx"], p["dimy"], refx, refy, dx, dy, ncc, 0.7, pairs)[0]
    np.testing.assert_allclose(log["K1_corrDistor"], ox[2], rtol=0.02)
    np.testing.assert_allclose(log["K1_corrDistor"], -3e-8, rtol=0.25)
    # the residual floor is the tracking noise (about 0.01 px): a gain of 9 on this case
    assert log["Final distorsion index"] < 0.2 * log["Initial distorsion index"]
    assert log["xc_corrDistor"] == 512.0 and log["yc_corrParallax"] == 384.0
    assert len((tmp_path / "errors.txt").read_text().split("\n\n")) >= 50
    assert (tmp_path / "distobox.txt").read_text().count("\n") > 4 * 50
