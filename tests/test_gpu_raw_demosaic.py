"""RAW mosaic -> grey frame on the GPU (ptk_load_frame_raw): the frame a
context holds after the call equals the reference's read_raw_image output
(golden fixtures) and the oracle's restatement, bit for bit, for the three
demosaic modes with and without the grey rescale; MinGray/MaxGray as the
reference prints them; full-size frames; the device-pointer variant; and the
rejection of mosaics the stencil would leave."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_golden_mosaics(ptk, oracle, cuda_device):
    g = np.load(GOLDEN / "raw_demosaic.npz")
    k = 0
    while f"case_{k}" in g:
        mode, resc, w, h, left, top = (int(v) for v in g[f"case_{k}"])
        t = ptk.Tracker(w, h)
        mm = t.load_frame_raw(0, g[f"raw_{k}"], left, top, mode, bool(resc))
        np.testing.assert_array_equal(t.read_frame(0), g[f"frame_{k}"], err_msg=f"case {k}")
        port = oracle.raw_demosaic(g[f"raw_{k}"], w, h, left, top, mode, bool(resc))
        assert mm == port[1], k
        t.close()
        k += 1
    assert k == 6


@pytest.mark.parametrize("mode,rescale", [(-1, False), (-2, True), (-20, True), (-2, False)])
def test_full_size_frame(ptk, oracle, cuda_device, mode, rescale):
    """5616x3744 frame in a 5680x3760 mosaic (margins 24 / 8), against the
    oracle, in both frame slots; the device-pointer variant gives the same."""
    import torch
    rng = np.random.default_rng(5 + abs(mode))
    raw = rng.integers(0, 16384, (3760, 5680)).astype(np.uint16)
    raw[1000:1040, 2000:2600] = 65535 - raw[1000:1040, 2000:2600] // 8
    want, mm_want = oracle.raw_demosaic(raw, 5616, 3744, 24, 8, mode, rescale)
    t = ptk.Tracker(5616, 3744)
    assert t.load_frame_raw(1, raw, 24, 8, mode, rescale) == mm_want
    np.testing.assert_array_equal(t.read_frame(1), want)
    d = torch.from_numpy(raw.view(np.int16)).cuda()
    t.load_frame_raw_device(0, d.data_ptr(), 5680, 3760, 24, 8, mode, rescale)
    np.testing.assert_array_equal(t.read_frame(0), want)
    t.close()


def test_rejections(ptk, cuda_device):
    t = ptk.Tracker(30, 20)
    raw = np.zeros((20, 30), dtype=np.uint16)
    with pytest.raises(ptk.PtkError, match="outside"):
        t.load_frame_raw(0, raw, 0, 0, ptk.DEMOSAIC_BINOMIAL3)  # column -1 of row -1
    with pytest.raises(ptk.PtkError, match="outside"):
        t.load_frame_raw(0, raw, 0, 0, ptk.DEMOSAIC_BOX2)  # past the last row
    with pytest.raises(ptk.PtkError, match="libraw"):
        t.load_frame_raw(0, raw, 0, 0, 0)
    assert t.load_frame_raw(0, raw, 0, 0, ptk.DEMOSAIC_GREY) == (0, 0)
    t.close()


@pytest.mark.parametrize("mode", [-1, -2, -20])
@pytest.mark.parametrize("geom", [((64, 96), (87, 60), 8, 1), ((40, 1040), (1031, 37), 8, 2),
                                  ((33, 2072), (2057, 30), 16, 1)])
def test_aligned_mosaics_vector_path(ptk, oracle, cuda_device, mode, geom):
    """Mosaics whose rows start 16-byte aligned (left margin and raw width
    multiples of 8) take the 8-column kernel: frames whose width is not a
    multiple of 8, that span several CTAs, and whose last column reaches the
    mosaic's last one, against the oracle, host and device mosaics."""
    import torch
    (rh, rw), (w, h), left, top = geom
    rng = np.random.default_rng(rw + mode)
    raw = rng.integers(0, 65536, (rh, rw)).astype(np.uint16)
    raw[::5] //= 7
    want = oracle.raw_demosaic(raw, w, h, left, top, mode, True)
    assert want is not None
    t = ptk.Tracker(w, h)
    assert t.load_frame_raw(0, raw, left, top, mode, True) == want[1]
    np.testing.assert_array_equal(t.read_frame(0), want[0])
    d = torch.from_numpy(raw.view(np.int16)).cuda()
    t.load_frame_raw_device(1, d.data_ptr(), rw, rh, left, top, mode, False)
    np.testing.assert_array_equal(t.read_frame(1), oracle.raw_demosaic(raw, w, h, left, top, mode, False)[0])
    t.close()
