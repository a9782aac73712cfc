"""The allocation-free pixel search (ptk_search_pixel_noalloc) against the
context path (ptk_search level 0).

Some callers cannot call cudaMalloc (a plug-in whose host application owns
all device memory, or a loop that must not allocate), so this entry point
works only on buffers the caller passes in and keeps its scratch in one fixed
device array.  This test owns every device buffer (allocated through torch),
calls the entry point through the C ABI twice in a row -- the second call
finds the first call's leftovers in the shared scratch -- and checks both
results against the context path: same offsets and rotation step, NCC within
the tolerance of the other parity tests.  It lives in its own file, collected
last, and passes alone in a fresh process as well as after the other tests."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NCC_TOL = 1e-5


def _context_search(ptk, pair, zone):
    p = pair["params"]
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=0, NCC_min=-1.0)  # accept every grain's best
    t.set_zone(0, *zone)
    t.set_grains(pair["rec"])
    t.make_patterns("grain_diameter", 1.0, 1.0)
    t.load_frame(0, pair["ref"])
    t.load_frame(1, pair["cur"])
    t.precompute()
    t.search(0)
    out = t.get_grains()
    t.close()
    return out


def _patterns(rec):
    """grain_diameter 1.0 1.0 (src/p-tracker.cpp:1656-1666) as CSR int16 pairs."""
    pts, starts = [], [0]
    for r in rec[:, 3]:
        rad = max(int(r * 1.0), 1)
        yy, xx = np.mgrid[-rad:rad + 1, -rad:rad + 1]
        keep = np.sqrt(xx.astype(float) ** 2 + yy.astype(float) ** 2) <= rad
        xy = np.stack([xx[keep], yy[keep]], 1)
        pts.append(xy)
        starts.append(starts[-1] + xy.shape[0])
    return np.concatenate(pts).astype(np.int16), np.array(starts, np.int32), max(x.shape[0] for x in pts), \
        int(np.abs(np.concatenate(pts)).max())


def test_noalloc_matches_context_path(ptk, wl, cuda_device, pair_cache):
    import torch

    pair = pair_cache("small16", 7)
    z = wl.tracker_options(pair["params"])["zones"][0]
    ctx_rec = _context_search(ptk, pair, z)
    rec = pair["rec"]
    n = rec.shape[0]
    dev = torch.device("cuda", 0)
    ref = torch.from_numpy(np.ascontiguousarray(pair["ref"]).view(np.int16)).to(dev)
    cur = torch.from_numpy(np.ascontiguousarray(pair["cur"]).view(np.int16)).to(dev)
    refx = torch.tensor(rec[:, 0].astype(np.int32), device=dev)
    refy = torch.tensor(rec[:, 1].astype(np.int32), device=dev)
    refrot = torch.tensor(rec[:, 2], dtype=torch.float64, device=dev)
    drot = torch.tensor(rec[:, 6], dtype=torch.float64, device=dev)
    dx = torch.tensor(rec[:, 4], dtype=torch.float64, device=dev)
    dy = torch.tensor(rec[:, 5], dtype=torch.float64, device=dev)
    xy, starts, maxp, maxr = _patterns(rec)
    pxy = torch.from_numpy(xy).to(dev)
    pst = torch.from_numpy(starts).to(dev)
    L = ptk.lib()
    zone = ptk.Zone(*z)
    stream = torch.cuda.current_stream().cuda_stream
    # the context path adds the offset to round(dx) (half away from zero; dx >= 0 here)
    gdx = np.floor(rec[:, 4] + 0.5)
    gdy = np.floor(rec[:, 5] + 0.5)
    expect_u = (ctx_rec[:, 4] - gdx).round().astype(np.int64)
    expect_v = (ctx_rec[:, 5] - gdy).round().astype(np.int64)
    expect_rot = ctx_rec[:, 6] - rec[:, 6]
    for call in range(2):
        ncc = torch.full((n,), -7.0, dtype=torch.float64, device=dev)
        bu = torch.full((n,), 12345, dtype=torch.int32, device=dev)
        bv = torch.full((n,), 12345, dtype=torch.int32, device=dev)
        br = torch.full((n,), 9.0, dtype=torch.float64, device=dev)
        rc = L.ptk_search_pixel_noalloc(
            C.c_void_p(ref.data_ptr()), C.c_void_p(cur.data_ptr()), ref.stride(0) * 2, pair["ref"].shape[1],
            pair["ref"].shape[0], n, C.c_void_p(refx.data_ptr()), C.c_void_p(refy.data_ptr()),
            C.c_void_p(refrot.data_ptr()), C.c_void_p(drot.data_ptr()), C.c_void_p(dx.data_ptr()),
            C.c_void_p(dy.data_ptr()), C.c_void_p(pst.data_ptr()), C.c_void_p(pxy.data_ptr()), maxp, maxr,
            C.byref(zone), 1, C.c_void_p(ncc.data_ptr()), C.c_void_p(bu.data_ptr()), C.c_void_p(bv.data_ptr()),
            C.c_void_p(br.data_ptr()), C.c_void_p(stream))
        assert rc == 0, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        got_ncc, got_u, got_v, got_r = ncc.cpu().numpy(), bu.cpu().numpy(), bv.cpu().numpy(), br.cpu().numpy()
        assert np.abs(got_ncc - ctx_rec[:, 10]).max() <= NCC_TOL, f"call {call}: NCC differs"
        np.testing.assert_array_equal(got_u, expect_u, err_msg=f"call {call}: x offsets differ")
        np.testing.assert_array_equal(got_v, expect_v, err_msg=f"call {call}: y offsets differ")
        np.testing.assert_array_equal(got_r, expect_rot, err_msg=f"call {call}: rotation steps differ")


def _buffers(pair, rec, xy, starts):
    """The entry point's inputs and outputs as torch-owned device buffers."""
    import torch

    dev = torch.device("cuda", 0)
    n = rec.shape[0]
    b = dict(
        ref=torch.from_numpy(np.ascontiguousarray(pair["ref"]).view(np.int16)).to(dev),
        cur=torch.from_numpy(np.ascontiguousarray(pair["cur"]).view(np.int16)).to(dev),
        ints=[torch.tensor(rec[:, k].astype(np.int32), device=dev) for k in (0, 1)],
        dbl=[torch.tensor(rec[:, k], dtype=torch.float64, device=dev) for k in (2, 6, 4, 5)],
        pxy=torch.from_numpy(xy).to(dev), pst=torch.from_numpy(starts).to(dev),
        ncc=torch.full((n,), -7.0, dtype=torch.float64, device=dev),
        bu=torch.full((n,), 12345, dtype=torch.int32, device=dev),
        bv=torch.full((n,), 12345, dtype=torch.int32, device=dev),
        br=torch.full((n,), 9.0, dtype=torch.float64, device=dev))
    torch.cuda.synchronize()
    return b


def _enqueue(ptk, pair, b, maxp, maxr, z):
    """One call through the C ABI on the default stream; returns its status."""
    zone = ptk.Zone(*z)
    vp = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    return ptk.lib().ptk_search_pixel_noalloc(
        vp(b["ref"]), vp(b["cur"]), b["ref"].stride(0) * 2, pair["ref"].shape[1], pair["ref"].shape[0],
        b["ncc"].shape[0], vp(b["ints"][0]), vp(b["ints"][1]), *[vp(t) for t in b["dbl"]], vp(b["pst"]),
        vp(b["pxy"]), maxp, maxr, C.byref(zone), 1, vp(b["ncc"]), vp(b["bu"]), vp(b["bv"]), vp(b["br"]), None)


def _results(b):
    import torch

    torch.cuda.synchronize()
    return b["ncc"].cpu().numpy(), b["bu"].cpu().numpy(), b["bv"].cpu().numpy(), b["br"].cpu().numpy()


def test_noalloc_rect_pattern_limits(ptk, wl, cuda_device, pair_cache):
    """A 25 x 17 rectangle at refrot 0.3 rad: its corners (Euclidean radius
    14.4) rotate to |x| = 14 at every searched angle.  With max_radius 16 (the
    radius rounded up, plus one) the results equal the context path's; with
    max_radius 12 every grain reports the caller-limit code (NaN,
    INT_MIN + 1), not the frame-edge code."""
    pair = dict(pair_cache("small16", 7))
    rec = pair["rec"].copy()
    rec[:, 2] = 0.3
    pair["rec"] = rec
    z = wl.tracker_options(pair["params"])["zones"][0]
    p = pair["params"]
    t = ptk.Tracker(p["dimx"], p["dimy"], rescue_level=0, NCC_min=-1.0)
    t.set_zone(0, *z)
    t.set_grains(rec)
    t.make_patterns("rect", 12, 8)
    t.load_frame(0, pair["ref"])
    t.load_frame(1, pair["cur"])
    t.precompute()
    t.search(0)
    ctx = t.get_grains()
    st = t.status()
    t.close()
    yy, xx = np.mgrid[-8:9, -12:13]
    one = np.stack([xx.ravel(), yy.ravel()], 1).astype(np.int16)  # rows of dy, then dx (make_rect_pattern)
    n = rec.shape[0]
    xy = np.concatenate([one] * n)
    starts = (np.arange(n + 1) * one.shape[0]).astype(np.int32)
    b = _buffers(pair, rec, xy, starts)
    assert _enqueue(ptk, pair, b, one.shape[0], 16, z) == 0
    ncc, bu, bv, br = _results(b)
    # grains both paths searched (a footprint at the frame edge is skipped by both)
    ok = (st == 0) & (bu > np.iinfo(np.int32).min + 1)
    assert ok.sum() > n // 2
    gdx, gdy = np.floor(rec[:, 4] + 0.5), np.floor(rec[:, 5] + 0.5)
    np.testing.assert_array_equal(bu[ok], (ctx[ok, 4] - gdx[ok]).round().astype(np.int64))
    np.testing.assert_array_equal(bv[ok], (ctx[ok, 5] - gdy[ok]).round().astype(np.int64))
    assert np.abs(ncc[ok] - ctx[ok, 10]).max() <= NCC_TOL
    assert _enqueue(ptk, pair, b, one.shape[0], 12, z) == 0
    ncc, bu, bv, br = _results(b)
    assert np.isnan(ncc).all()
    assert (bu == np.iinfo(np.int32).min + 1).all() and (bv == np.iinfo(np.int32).min + 1).all()


def test_noalloc_leaves_pending_error_alone(ptk, wl, cuda_device, pair_cache):
    """An error left pending in the calling thread by earlier, unrelated CUDA
    runtime work (here a cudaSetDevice to a device that does not exist, which
    touches no GPU) is neither returned as this call's failure nor cleared.
    The buffers are made before the error is planted and read after it is
    cleared, so that no other library sees it."""
    rt = C.CDLL("libcudart.so.12")
    rt.cudaSetDevice.argtypes = [C.c_int]
    pair = pair_cache("small16", 7)
    z = wl.tracker_options(pair["params"])["zones"][0]
    xy, starts, maxp, maxr = _patterns(pair["rec"])
    b = _buffers(pair, pair["rec"], xy, starts)
    rt.cudaGetLastError()
    assert rt.cudaSetDevice(1 << 20) != 0
    pending = rt.cudaPeekAtLastError()
    assert pending != 0
    try:
        rc = _enqueue(ptk, pair, b, maxp, maxr, z)
        still = rt.cudaPeekAtLastError()
    finally:
        rt.cudaGetLastError()
    assert rc == 0
    assert still == pending
    ncc, *_ = _results(b)
    assert np.isfinite(ncc).all()


def test_noalloc_rejects_oversized_work(ptk, cuda_device):
    import torch

    dev = torch.device("cuda", 0)
    buf = torch.zeros(64 * 64, dtype=torch.int16, device=dev)
    d = torch.zeros(1 << 20, dtype=torch.float64, device=dev)
    zone = ptk.Zone(200, 200, 200, 200, 10, 0.005)  # 21 steps x 13 x 13 tiles x grains
    rc = ptk.lib().ptk_search_pixel_noalloc(
        C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()), 128, 64, 64, 100000,
        *[C.c_void_p(d.data_ptr())] * 8, 10, 5, C.byref(zone), 1, *[C.c_void_p(d.data_ptr())] * 4, None)
    assert rc == ptk.PTK_ERR_LIMIT
