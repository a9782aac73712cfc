"""RAW mosaic -> grey frame on the CPU: the oracle's restatement of
read_raw_image's demosaic modes (-1, -2, -20) and grey rescale against the
reference's own code (golden fixtures made by running read_raw_image through
the libraw stand-in, and live when the compiled reference is present)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _cases():
    g = np.load(GOLDEN / "raw_demosaic.npz")
    k = 0
    while f"case_{k}" in g:
        mode, resc, w, h, left, top = (int(v) for v in g[f"case_{k}"])
        yield k, g[f"raw_{k}"], g[f"frame_{k}"], mode, resc, w, h, left, top
        k += 1


def test_port_matches_reference_fixtures(oracle):
    n = 0
    for k, raw, frame, mode, resc, w, h, left, top in _cases():
        got = oracle.raw_demosaic(raw, w, h, left, top, mode, bool(resc))
        assert got is not None, k
        np.testing.assert_array_equal(got[0], frame, err_msg=f"case {k}")
        n += 1
    assert n == 6


@pytest.mark.parametrize("mode", [-1, -2, -20])
@pytest.mark.parametrize("rescale", [False, True])
def test_port_matches_reference_live(oracle, mode, rescale):
    if not oracle.have_reference():
        pytest.skip("compiled reference not built here")
    rng = np.random.default_rng(abs(mode) * 10 + rescale)
    raw = rng.integers(0, 65536, (97, 131)).astype(np.uint16)
    raw[::7] //= 16
    a = oracle.raw_demosaic(raw, 126, 92, 2, 3, mode, rescale)
    b = oracle.raw_demosaic(raw, 126, 92, 2, 3, mode, rescale, reference=True)
    np.testing.assert_array_equal(a[0], b[0])
    assert a[1] == (int(a[0].min()), int(a[0].max())) or rescale


def test_port_rejects_stencil_outside_mosaic(oracle):
    raw = np.zeros((20, 30), dtype=np.uint16)
    assert oracle.raw_demosaic(raw, 30, 20, 0, 0, -2, False) is None  # reads index -1
    assert oracle.raw_demosaic(raw, 30, 20, 0, 0, -1, False) is None  # reads past the last row
    assert oracle.raw_demosaic(raw, 29, 19, 0, 0, -1, False) is not None
    assert oracle.raw_demosaic(raw, 30, 20, 0, 0, -20, False) is not None
    assert oracle.raw_demosaic(raw, 10, 10, 1, 1, 0, False) is None  # libraw's own modes
