"""Generates tests/golden/*.npz and dic_out_frame_small.txt by running the
reference's own tracking code, compiled from its sources into
oracle/_ref/libptk_ref.so (oracle/Makefile, target `ref`).

Run where the reference sources exist:
    python tests/golden/make_golden.py             (all fixtures)
    python tests/golden/make_golden.py --raw-only  (raw_demosaic.npz only)
    python tests/golden/make_golden.py --example-only  (example_rods.npz only)
Inputs are seeded synthetic frames (p-tracker_b200/workloads.py); every
output stored here is what the compiled reference returned.
"""
from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import bind  # noqa: E402

CASES = {
    "pixel_tiny": dict(preset="tiny", seed=5, n=None, stages="pixel",
                       zones=[(4, 4, 4, 4, 4, 0.005)], params={"rescue_level": 0}),
    "frame_small": dict(preset="small16", seed=7, n=14, dims=(320, 256), stages="frame",
                        zones=[(6, 6, 6, 6, 10, 0.005)], params={"rescue_level": 0, "iraz": 100}),
    "frame_linear_ring": dict(preset="small16", seed=8, n=10, dims=(256, 224), stages="frame",
                              zones=[(5, 4, 3, 6, 3, 0.01)], pattern=("ring", 4, 9),
                              params={"rescue_level": 0, "iraz": 100, "image_interpolator": 0}),
    "frame_quintic_rect": dict(preset="small16", seed=9, n=10, dims=(256, 224), stages="frame",
                               zones=[(4, 4, 4, 4, 2, 0.02)], pattern=("rect", 6, 4),
                               params={"rescue_level": 0, "iraz": 100, "image_interpolator": 2}),
    "rescue_small": dict(preset="small16", seed=21, n=24, dims=(320, 256), disp=7.0, stages="rescue",
                         zones=[(2, 2, 2, 2, 2, 0.01), (5, 5, 5, 5, 2, 0.01), (9, 9, 9, 9, 3, 0.01)],
                         params={"rescue_level": 2, "NCC_min": 0.8, "NCC_min_super": 0.75, "subpixel": 0}),
}
STEP_CASES = [(0.005, 10), (0.005, 4), (0.0025, 20), (0.0454, 6), (0.045, 69), (0.01, 3)]


def rotation_steps(inc: float, num: int) -> np.ndarray:
    """The reference's loop (src/p-tracker.cpp:684-686) in IEEE double."""
    out = []
    rotmax = abs(inc * num)
    d = -rotmax
    while d <= rotmax:
        out.append(d)
        d += inc
    return np.array(out)


def case_pair(wl, c):
    p = dict(wl.PRESETS[c["preset"]])
    if "dims" in c:
        p["dimx"], p["dimy"] = c["dims"]
    if "disp" in c:
        p["disp"] = c["disp"]
    if c.get("n"):
        p["n"] = c["n"]
    return wl.make_pair(p, seed=c["seed"])


def run_case(cls, pair, c):
    t = bind.setup(cls, pair, threads=4, zones=c["zones"], params=c["params"],
                   pattern=c.get("pattern", ("grain_diameter", 1.0, 1.0)))
    out = {}
    if c["stages"] == "pixel":
        t.precompute()
        out["nres"] = np.array([t.pixel_all()])
        out["mean0"], out["C0C0"] = t.get_precomp()
        out["pattern0_g0"] = t.pattern(0, 1)
    elif c["stages"] == "rescue":
        t.precompute()
        out["nres"] = np.array([t.pixel_all()])
        out["nsup"] = np.array([t.rescue_all()])
        t.super_rescue_all()
        res, sup = t.lists()
        out["rescued"] = np.array(res, dtype=np.int32)
        out["super_rescued"] = np.array(sup, dtype=np.int32)
    else:
        t.track_frame(1)
    out["grains"] = t.get_grains()
    return t, out


# RAW mosaics: (mode, rescale, raw (height, width), frame (width, height), left, top); the third case
# puts the frame at column 0, so the -2 stencil of column 0 reads the previous row's last pixel and
# the last column's right neighbour is the next row's first pixel (the flat indexing of the reference)
RAW_CASES = [(-1, 0, (61, 83), (80, 58), 1, 2), (-2, 1, (64, 100), (98, 61), 1, 1), (-2, 0, (50, 70), (70, 46), 0, 2),
             (-20, 1, (40, 60), (57, 37), 3, 3), (-1, 1, (33, 47), (45, 30), 0, 0), (-2, 1, (48, 66), (61, 44), 2, 2)]


def raw_demosaic_fixtures():
    """read_raw_image (src/p-tracker.cpp:214-387) of the reference, run on
    seeded mosaics through the libraw stand-in: raw_demosaic.npz."""
    rng = np.random.default_rng(77)
    out = {}
    for k, (mode, resc, (rh, rw), (w, h), left, top) in enumerate(RAW_CASES):
        raw = rng.integers(0, 4096, (rh, rw)).astype(np.uint16)
        raw[rng.random((rh, rw)) < 0.05] = 65535
        raw[rh // 3: rh // 3 + 4, 5:25] = rng.integers(50000, 65536, (4, 20))
        frame, _ = bind.raw_demosaic(raw, w, h, left, top, mode, bool(resc), reference=True)
        out[f"raw_{k}"] = raw
        out[f"frame_{k}"] = frame
        out[f"case_{k}"] = np.array([mode, resc, w, h, left, top])
    np.savez_compressed(HERE / "raw_demosaic.npz", **out)


# the reference's example (examples/ParticleImageTracking/commands.txt): 9 rods between TEST01 and TEST02
EXAMPLE_ZONES = [(6, 6, 6, 6, 6, 0.0454), (30, 30, 30, 30, 69, 0.0454), (200, 200, 200, 200, 69, 0.045)]
EXAMPLE_PARAMS = {"rescue_level": 2, "NCC_min": 0.8, "NCC_min_super": 0.7, "iraz": 20000}


def example_fixture():
    """The reference's shipped example: examples/ImageData/TEST01.tiff and
    TEST02.tiff (LZW RGB) decoded with Pillow through the reference's grey
    conversion, the 9 rods of examples/ParticleImageTracking/recentered.data
    read by the reference's own read_grains (4-column form), tracked with that
    example's settings (pattern circ 10; zones and thresholds above) by the
    reference's own code from image 1 to image 1, then to image 2:
    example_rods.npz."""
    from PIL import Image
    sys.path.insert(0, str(HERE.parent))
    from imagefiles import reference_grey
    ex = bind.REF_SRC.parent / "examples"
    frames = []
    for k in (1, 2):
        a = np.asarray(Image.open(ex / "ImageData" / f"TEST{k:02d}.tiff").convert("RGB"))
        frames.append(reference_grey(a[..., 0], a[..., 1], a[..., 2]))
    h, w = frames[0].shape
    t = bind.Reference(w, h, 1)
    t.n = t._f("read_grains")(t.h, str(ex / "ParticleImageTracking" / "recentered.data").encode(), 0)
    rec = t.get_grains()
    t.close()
    pair = dict(params=dict(dimx=w, dimy=h), ref=frames[0], cur=frames[0], rec=rec)
    c = bind.setup(bind.Reference, pair, threads=4, zones=EXAMPLE_ZONES, params=EXAMPLE_PARAMS, pattern=("circ", 10))
    c.track_frame(1)
    g1 = c.get_grains()
    c.load_current(frames[1])
    c.track_frame(2)
    g2 = c.get_grains()
    res, sup = c.lists()
    c.close()
    np.savez_compressed(HERE / "example_rods.npz", frame1=frames[0], frame2=frames[1], rec=rec, grains1=g1,
                        grains2=g2, rescued2=np.array(res, dtype=np.int32),
                        super_rescued2=np.array(sup, dtype=np.int32))


def main():
    if "--raw-only" in sys.argv:
        bind.build()
        raw_demosaic_fixtures()
        return
    if "--example-only" in sys.argv:
        bind.build()
        example_fixture()
        return
    assert bind.REF_SO.exists() or (bind.REF_SRC / "p-tracker.cpp").exists(), "reference sources needed"
    bind.build()
    sys.path.insert(0, str(ROOT))
    wl = importlib.import_module("p-tracker_b200.workloads")
    for name, c in CASES.items():
        pair = case_pair(wl, c)
        t, out = run_case(bind.Reference, pair, c)
        ref = np.ascontiguousarray(pair["ref"]).astype(np.uint16)
        cur = np.ascontiguousarray(pair["cur"]).astype(np.uint16)
        np.savez_compressed(HERE / f"{name}.npz", ref=ref, cur=cur, rec=pair["rec"],
                            maxval=np.array([pair["params"]["maxval"]]), **out)
        if name == "frame_small":
            t.save_grains(str(HERE / "dic_out_frame_small.txt"), 1)
        t.close()
        print(name, pair["rec"].shape[0], "grains")
    # interpolators and objective on the frame_small frames
    c = CASES["frame_small"]
    pair = case_pair(wl, c)
    t = bind.setup(bind.Reference, pair, threads=1, zones=c["zones"], params=c["params"])
    t.precompute()
    rng = np.random.default_rng(123)
    pts = np.stack([rng.uniform(3, c["dims"][0] - 4, 400), rng.uniform(3, c["dims"][1] - 4, 400)], 1)
    vals = np.array([[t.interp(k, 1, x, y) for (x, y) in pts] for k in range(3)])
    X = rng.uniform(-0.7, 0.7, (t.n, 3)) * np.array([1, 1, 0.03])
    obj = np.array([t.objective(g, X[g]) for g in range(t.n)])
    params = np.zeros((8, 14))
    upts = rng.uniform(0, 320, (8, 16, 2))
    uvals = np.zeros((8, 16, 2))
    for k in range(8):
        P = params[k]
        P[0], P[1], P[8], P[9] = rng.uniform(100, 220, 4)
        P[2], P[3], P[4] = rng.uniform(-1e-6, 1e-6), rng.uniform(-1e-12, 1e-12), rng.uniform(-1e-18, 1e-18)
        P[5], P[6], P[7] = rng.uniform(-1e-5, 1e-5, 3)
        P[10], P[11], P[12], P[13] = rng.uniform(-0.2, 0.2, 4) * np.array([1, 0.01, 1, 0.01])
        for j in range(16):
            uvals[k, j] = t.undistor(P, upts[k, j, 0], upts[k, j, 1])
    np.savez_compressed(HERE / "numerics.npz", interp_pts=pts, interp_vals=vals, obj_X=X, obj_vals=obj,
                        undistor_params=params, undistor_pts=upts, undistor_vals=uvals)
    # patterns of the reference's generators
    pats = {}
    tp = bind.Reference(64, 64, 1)
    tp.set_grains(np.zeros((1, 13)))
    for r in range(2, 16):  # radius 1 overflows the reference's allocation (src/p-tracker.cpp:1388)
        tp.make_pattern(0, 0, r)
        pats[f"circ_{r}"] = tp.pattern(0, 0)
    tp.make_pattern(0, 1, 5, 9)
    pats["ring_5_9"] = tp.pattern(0, 0)
    tp.make_pattern(0, 2, 3, 4)
    pats["rect_3_4"] = tp.pattern(0, 0)
    np.savez_compressed(HERE / "patterns.npz", **pats)
    np.savez_compressed(HERE / "rotation_steps.npz",
                        **{f"inc{inc}_num{num}": rotation_steps(inc, num) for inc, num in STEP_CASES})
    raw_demosaic_fixtures()
    example_fixture()
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
