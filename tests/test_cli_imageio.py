"""Host side of the command-file driver (no GPU): the image decoder against the
reference's grey-level conversion, and the command-file parser against the
reference's token rules (read_data, src/p-tracker.cpp:1487-1784)."""
from __future__ import annotations

import json
import subprocess

import numpy as np
import pytest

from imagefiles import reference_grey, write_pgm, write_tiff


@pytest.fixture(scope="module")
def rng():
    return np.random.default_rng(42)


@pytest.mark.parametrize("big_endian", [False, True])
@pytest.mark.parametrize("rows_per_strip", [None, 7])
def test_tiff_grey8(ptk, tmp_path, rng, big_endian, rows_per_strip):
    a = rng.integers(0, 256, (37, 53), dtype=np.uint8)
    p = tmp_path / "g8.tif"
    write_tiff(p, a, big_endian=big_endian, rows_per_strip=rows_per_strip, datetime="2023:01:02 03:04:05")
    got, when = ptk.read_image_file(str(p))
    np.testing.assert_array_equal(got, reference_grey(a, a, a))
    assert when == "2023:01:02 03:04:05"


def test_tiff_grey8_min_is_white(ptk, tmp_path, rng):
    a = rng.integers(0, 256, (20, 30), dtype=np.uint8)
    p = tmp_path / "w.tif"
    write_tiff(p, a, photometric=0)
    got, when = ptk.read_image_file(str(p))
    inv = (255 - a.astype(np.int32)).astype(np.uint8)
    np.testing.assert_array_equal(got, reference_grey(inv, inv, inv))
    assert when == "dateTime unknown"


def test_tiff_grey16_keeps_high_byte(ptk, tmp_path, rng):
    a = rng.integers(0, 65536, (25, 31), dtype=np.uint16)
    p = tmp_path / "g16.tif"
    write_tiff(p, a, big_endian=True)
    got, _ = ptk.read_image_file(str(p))
    hi = (a >> 8).astype(np.uint8)
    np.testing.assert_array_equal(got, reference_grey(hi, hi, hi))


@pytest.mark.parametrize("spp", [3, 4])
def test_tiff_rgb8(ptk, tmp_path, rng, spp):
    a = rng.integers(0, 256, (19, 23, spp), dtype=np.uint8)
    p = tmp_path / "rgb.tif"
    write_tiff(p, a, rows_per_strip=5)
    got, _ = ptk.read_image_file(str(p))
    np.testing.assert_array_equal(got, reference_grey(a[..., 0], a[..., 1], a[..., 2]))


def test_tiff_rgb16_rounds_to_8_bits(ptk, tmp_path, rng):
    a = rng.integers(0, 65536, (11, 13, 3), dtype=np.uint16)
    p = tmp_path / "rgb16.tif"
    write_tiff(p, a)
    got, _ = ptk.read_image_file(str(p))
    c = ((a.astype(np.uint32) + 128) // 257).astype(np.uint8)
    np.testing.assert_array_equal(got, reference_grey(c[..., 0], c[..., 1], c[..., 2]))


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_pgm_as_stored(ptk, tmp_path, rng, dtype):
    a = rng.integers(0, np.iinfo(dtype).max + 1, (17, 29)).astype(dtype)
    p = tmp_path / "f.pgm"
    write_pgm(p, a)
    got, _ = ptk.read_image_file(str(p))
    np.testing.assert_array_equal(got, a.astype(np.uint16))


def test_unsupported_and_missing_files(ptk, tmp_path, rng):
    a = rng.integers(0, 256, (8, 8), dtype=np.uint8)
    p = tmp_path / "jpeg.tif"
    write_tiff(p, a, compression=7)  # JPEG-in-TIFF
    with pytest.raises(ptk.PtkError, match="compression not supported"):
        ptk.read_image_file(str(p))
    p = tmp_path / "lzw.tif"
    write_tiff(p, a, compression=5)  # raw bytes under an LZW tag: not a valid code stream
    with pytest.raises(ptk.PtkError, match="corrupt"):
        ptk.read_image_file(str(p))
    write_tiff(p, a.astype(np.uint16) * 257, compression=8, rows_per_strip=4, truncate=6)  # cut Deflate strips
    with pytest.raises(ptk.PtkError, match="corrupt or short"):
        ptk.read_image_file(str(p))
    write_tiff(p, a, predictor=3)  # floating-point prediction
    with pytest.raises(ptk.PtkError, match="predictor"):
        ptk.read_image_file(str(p))
    with pytest.raises(ptk.PtkError, match="cannot open"):
        ptk.read_image_file(str(tmp_path / "absent.tif"))
    (tmp_path / "junk.bin").write_bytes(b"not an image")
    with pytest.raises(ptk.PtkError, match="unknown image format"):
        ptk.read_image_file(str(tmp_path / "junk.bin"))


def _check(ptk, cmd_path, cwd):
    r = subprocess.run([str(ptk.cli_path()), "--check", str(cmd_path)], capture_output=True, text=True, cwd=cwd,
                       timeout=60)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    return json.loads(lines[-1]), lines[:-1], r.stderr


def test_command_file_tokens(ptk, tmp_path):
    (tmp_path / "start.txt").write_text("3\n10.5 20.25 0.0 12\n100 200 0.1 30\n400 50 0 30\n")
    (tmp_path / "commands.txt").write_text("""# a comment line with tokens iref 99
image_name frame_%04d.tif   ! trailing comment
grains_to_follow start.txt
iref 2 ibeg 3 iend 9 iinc 2 iraz 4
rescue_level 1
NCC_min 0.8  NCC_min_super 0.55
subpixel 1  subpix_tol 1e-7
initial_direction_dx 0.02 initial_direction_dy 0.03 initial_direction_dr 0.004
image_interpolator quintic
overflow_stiffness 2.5 subpix_displacement_max 4
search_zone.left 5 search_zone.right 6 search_zone.up 7 search_zone.down 8
search_zone.num_rot 10 search_zone.inc_rot 0.005
search_zone_rescue.left 20 search_zone_rescue.right 20 search_zone_rescue.up 20 search_zone_rescue.down 20
search_zone_rescue.num_rot 2 search_zone_rescue.inc_rot 0.01
targetRadiusPattern 30
pattern grain_diameter 0.9 5
targetRadiusPattern -1
pattern circ 7
mask_rect 0 150 0 250
use_neighbour_list 1 neighbour_dist_pix 100 wanted_num_threads 16
K1_corrDistor -2e-9 xc_corrDistor 2808 dK1_corrDistor 1e-10
search_method bf16 subpix_method adjoint_lm undistort_images 1 autotune 1
no_such_token
""")
    cfg, out, err = _check(ptk, tmp_path / "commands.txt", tmp_path)
    assert cfg["image_name"] == "frame_%04d.tif"
    assert (cfg["iref"], cfg["ibeg"], cfg["iend"], cfg["iinc"], cfg["iraz"]) == (2, 3, 9, 2, 4)
    assert cfg["grains"] == 3 and cfg["masked"] == 2   # (10, 20) and (100, 200) lie in the rectangle
    assert cfg["rescue_level"] == 1 and cfg["NCC_min"] == 0.8 and cfg["NCC_min_super"] == 0.55
    assert cfg["subpix_tol"] == 1e-7 and cfg["initial_direction"] == [0.02, 0.03, 0.004]
    assert cfg["image_interpolator"] == 2
    assert cfg["overflow_stiffness"] == 2.5 and cfg["subpix_displacement_max"] == 4
    assert cfg["zones"][0] == [5, 6, 7, 8, 10, 0.005]
    assert cfg["zones"][1] == [20, 20, 20, 20, 2, 0.01]
    # patterns keep the targetRadiusPattern in force when their token was read
    assert cfg["patterns"] == [[3, 0.9, 5, 30, ""], [0, 7, 0, -1, ""]]
    assert cfg["disto"][0] == 2808 and cfg["disto"][2] == -2e-9
    assert cfg["search_method"] == 1 and cfg["subpix_method"] == 1 and cfg["undistort_images"] == 1
    assert cfg["autotune"] == 1
    assert cfg["unknown_tokens"] == 1 and "Unknown token: no_such_token" in out


def test_grain_reload_drops_earlier_patterns(ptk, tmp_path):
    """A grain file read after `pattern` replaces the grains, and with them the
    patterns, as read_grains rebuilds ptracker::grain."""
    (tmp_path / "a.txt").write_text("1\n10 10 0 5\n")
    (tmp_path / "commands.txt").write_text("start_file a.txt\npattern circ 3\nrestart_file b.txt\n")
    (tmp_path / "b.txt").write_text("1\n" + " ".join(["12", "14"] + ["0"] * 11) + "\n")
    cfg, _, _ = _check(ptk, tmp_path / "commands.txt", tmp_path)
    assert cfg["grains"] == 1 and cfg["patterns"] == []


def test_missing_command_file_fails(ptk, tmp_path):
    r = subprocess.run([str(ptk.cli_path()), "--check", str(tmp_path / "none.txt")], capture_output=True,
                       text=True, timeout=60)
    assert r.returncode != 0 and "cannot open command file" in r.stderr


def test_correction_distortion_tokens(ptk, tmp_path):
    """The tokens of the correction_distortion procedure (src/p-tracker.cpp:
    1553-1566, 1696-1772): images, imposed displacements, pair range, the 14
    initial parameters and their perturbations, the minimiser."""
    (tmp_path / "start.txt").write_text("2\n10 20 0 12\n400 300 0 15\n")
    (tmp_path / "commands.txt").write_text("""procedure correction_distortion
image_name img_%d.pgm
start_file start.txt
image_numbers_corrDisto 3 10 11 12
imposedDisplApprox_corrDisto 1.5 -2 3 4
equiProj_dist_range 100 900
optim_algo POWELL_ITER powell_num_iter 3
K1_corrDistor -1e-9 dK1_corrDistor 1e-11 dxc_corrParallax 0.5 angle2_corrParallax 0.01
optim_algo NEWTON
""")
    cfg, out, _ = _check(ptk, tmp_path / "commands.txt", tmp_path)
    assert cfg["procedure"] == "correction_distortion"
    assert cfg["corr_images"] == [10, 11, 12]
    assert cfg["imposed"] == [[0, 0], [1.5, -2], [3, 4]]
    assert cfg["equiproj_range"] == [100, 900]
    assert cfg["optim_algo"] == 1 and cfg["powell_num_iter"] == 3
    # defaults of ptracker::ptracker: negative centres, perturbations 1e-6
    assert cfg["disto"] == [-1, -1, -1e-9, 0, 0, 0, 0, 0, -1, -1, 0, 0, 0.01, 0]
    assert cfg["disto_perturb"][2] == 1e-11 and cfg["disto_perturb"][8] == 0.5
    assert cfg["disto_perturb"][0] == 1e-6 and cfg["disto_perturb"][13] == 1e-6
    assert any("unknown for optim_algo" in line for line in out)




@pytest.mark.parametrize("compression", ["tiff_lzw", "tiff_adobe_deflate", "tiff_deflate", "packbits"])
@pytest.mark.parametrize("kind", ["rgb", "grey8", "grey16"])
def test_compressed_tiff_matches_reference_grey(ptk, tmp_path, compression, kind):
    """Compressed TIFFs written by another encoder (Pillow's libtiff) decode
    to the grey levels the reference's libtiff RGBA path gives."""
    PIL = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(len(compression) * 7 + len(kind))
    h, w = 157, 211  # several strips of uneven size
    if kind == "rgb":
        a = rng.integers(0, 256, (h, w, 3)).astype(np.uint8)
        a[40:90, 30:150] = (200, 120, 40)  # runs, so the dictionary and PackBits repeats get used
        im = PIL.fromarray(a)
        want = reference_grey(a[..., 0], a[..., 1], a[..., 2])
    elif kind == "grey8":
        a = rng.integers(0, 256, (h, w)).astype(np.uint8)
        a[::3, 50:120] = 17
        im = PIL.fromarray(a)
        want = reference_grey(a, a, a)
    else:
        a = rng.integers(0, 65536, (h, w)).astype(np.uint16)
        a[20:60] = 40000
        im = PIL.fromarray(a)
        hi = (a >> 8).astype(np.uint8)
        want = reference_grey(hi, hi, hi)
    path = tmp_path / "f.tif"
    im.save(path, compression=compression, tiffinfo={278: 16})  # 16 rows per strip
    got, _ = ptk.read_image_file(str(path))
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("big_endian", [False, True])
def test_tiff_horizontal_predictor(ptk, tmp_path, big_endian):
    """Predictor 2 (horizontal differencing) with Deflate, written here: each
    sample stored as the difference to the same channel's left neighbour
    (8-bit RGB and 16-bit grey, both byte orders, several strips)."""
    rng = np.random.default_rng(4)
    a = rng.integers(0, 256, (23, 31, 3)).astype(np.uint8)
    d = a.copy()
    d[:, 1:] = (a[:, 1:].astype(np.int16) - a[:, :-1].astype(np.int16)).astype(np.uint8)
    path = tmp_path / "p.tif"
    write_tiff(path, d, predictor=2, compression=8, rows_per_strip=5, big_endian=big_endian)
    got, _ = ptk.read_image_file(str(path))
    np.testing.assert_array_equal(got, reference_grey(a[..., 0], a[..., 1], a[..., 2]))
    g = rng.integers(0, 65536, (19, 27)).astype(np.uint16)
    dg = g.copy()
    dg[:, 1:] = (g[:, 1:].astype(np.int32) - g[:, :-1].astype(np.int32)).astype(np.uint16)
    write_tiff(path, dg, predictor=2, compression=8, rows_per_strip=4, big_endian=big_endian)
    got, _ = ptk.read_image_file(str(path))
    hi = (g >> 8).astype(np.uint8)
    np.testing.assert_array_equal(got, reference_grey(hi, hi, hi))


@pytest.mark.parametrize("alea", [0, 9])
def test_make_grid_matches_reference(ptk, oracle, tmp_path, alea):
    """make_grid seeds the grains as the reference's make_grid does (grid
    steps, the random displacement drawn from the C library's rand() in the
    same order), compared with the reference's own function."""
    (tmp_path / "commands.txt").write_text(f"make_grid 74 2507 75 1865 14 14 {alea}\npattern rect 23 23\n")
    cfg, out, _ = _check(ptk, tmp_path / "commands.txt", tmp_path)
    assert cfg["grains"] == 196 and "Create grid with 196 points" in "\n".join(out)
    if not oracle.have_reference():
        pytest.skip("compiled reference not built here")
    import ctypes as C
    L = C.CDLL(str(oracle.REF_SO))
    L.ref_create.restype = C.c_void_p
    h = C.c_void_p(L.ref_create(8, 8))
    xy = np.zeros(2 * 196, dtype=np.int32)
    n = L.ref_make_grid(h, C.c_double(74), C.c_double(2507), C.c_double(75), C.c_double(1865), 14, 14, alea,
                        xy.ctypes.data_as(C.c_void_p))
    L.ref_destroy(h)
    assert n == 196
    assert cfg["grain_xy"] == xy.reshape(-1, 2).tolist()
