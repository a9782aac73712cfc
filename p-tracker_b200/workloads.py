"""Seeded synthetic tracking workloads.

Five presets follow the five benchmark configurations of this path:

  cfg1  2048x1536, 8-bit values, 400 discs r~U(20,30), speckle sigma 2 px,
        density 0.02/px^2, amplitudes U(60,220), noise sigma 2 GL,
        d~U(-3,3) px, theta~U(-0.02,0.02) rad, zone +-8 px, 21 rotation steps.
  cfg2  5616x3744, 16-bit, 2000 discs, r: 60% U(10,18) + 40% U(30,40),
        sigma~U(1.5,3), d~U(-10,10), theta~U(-0.05,0.05), zone +-15, 21 steps.
  cfg3  = cfg2 (precision form runs on the same pair).
  cfg4  = cfg2 with noise sigma = 5% of the 16-bit range.
  cfg5  50-frame sequence, 5616x3744 16-bit, 5000 discs r~U(8,40), smooth
        cumulative shear (<= 60 px), rotation random walk (0.01 rad/step),
        radial distortion k1=-2e-9, k2=1e-16 about the centre, 3% of grains
        jump 25 px once (rescue at +-40 px, NCC_min 0.7).

16-bit presets scale the 8-bit grey levels (background, amplitudes, noise) by
256.  Grain records follow the 4-column start-file semantics of read_grains
(src/p-tracker.cpp:1253-1272): refcoord = floor(centre), dx = upix = the
fractional part.  `truth` is what a perfect tracker reports in the 13-column
dx, dy, drot after the pair: the rigid motion applied to the pattern anchor
refcoord (patterns rotate about refcoord, not about the true centre).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import synth as _synth_lib

PRESETS = {
    "tiny": dict(dimx=256, dimy=192, maxval=255, n=12, mix=[(1.0, 9.0, 13.0)], sig=(2.0, 2.0), density=0.02,
                 amp=(60.0, 220.0), bg=10.0, noise=2.0, disp=2.0, rot=0.02, zone=4, num_rot=4, inc_rot=0.005,
                 rescue_zone=0),
    "small16": dict(dimx=512, dimy=384, maxval=65535, n=40, mix=[(0.6, 10.0, 18.0), (0.4, 20.0, 26.0)],
                    sig=(1.5, 3.0), density=0.02, amp=(60.0 * 256, 220.0 * 256), bg=10.0 * 256, noise=2.0 * 256,
                    disp=5.0, rot=0.05, zone=6, num_rot=10, inc_rot=0.005, rescue_zone=0),
    "cfg1": dict(dimx=2048, dimy=1536, maxval=255, n=400, mix=[(1.0, 20.0, 30.0)], sig=(2.0, 2.0), density=0.02,
                 amp=(60.0, 220.0), bg=10.0, noise=2.0, disp=3.0, rot=0.02, zone=8, num_rot=10, inc_rot=0.005,
                 rescue_zone=0),
    "cfg2": dict(dimx=5616, dimy=3744, maxval=65535, n=2000, mix=[(0.6, 10.0, 18.0), (0.4, 30.0, 40.0)],
                 sig=(1.5, 3.0), density=0.02, amp=(60.0 * 256, 220.0 * 256), bg=10.0 * 256, noise=2.0 * 256,
                 disp=10.0, rot=0.05, zone=15, num_rot=10, inc_rot=0.005, rescue_zone=0),
}
PRESETS["cfg3"] = dict(PRESETS["cfg2"])
PRESETS["cfg4"] = dict(PRESETS["cfg2"], noise=0.05 * 65535)
PRESETS["cfg5"] = dict(dimx=5616, dimy=3744, maxval=65535, n=5000, mix=[(1.0, 8.0, 40.0)], sig=(1.5, 3.0),
                       density=0.02, amp=(60.0 * 256, 220.0 * 256), bg=10.0 * 256, noise=2.0 * 256, disp=0.0,
                       rot=0.0, zone=15, num_rot=10, inc_rot=0.005, rescue_zone=40, frames=50, shear=60.0,
                       rot_walk=0.01, jump=25.0, jump_frac=0.03,
                       disto=(-2e-9, 1e-16), gap=20.0)  # 5000 grains fit; a jump may overlap a neighbour by <= 5 px


def _threads() -> int:
    return max(1, min(32, os.cpu_count() or 1))


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def place(p: dict, seed: int, n: int | None = None):
    n = p["n"] if n is None else n
    L = _synth_lib()
    mix = p["mix"]
    w = np.array([m[0] for m in mix])
    rlo = np.array([m[1] for m in mix])
    rhi = np.array([m[2] for m in mix])
    cx, cy, r, sig = (np.zeros(n) for _ in range(4))
    gseed = np.zeros(n, dtype=np.uint64)
    margin = max(p["zone"], p.get("rescue_zone", 0)) + p["disp"] + 6.0 + p.get("jump", 0.0) + p.get("shear", 0.0) * 0.5
    if p.get("disto"):
        margin += 40.0
    gap = p.get("gap", 2.0 * p["disp"] + 6.0 + (2.0 * p.get("jump", 0.0) if p.get("jump") else 0.0))
    got = L.ptk_synth_place(C.c_int(p["dimx"]), C.c_int(p["dimy"]), C.c_int(n), C.c_int(len(mix)), _dp(w),
                            _dp(rlo), _dp(rhi), C.c_double(p["sig"][0]), C.c_double(p["sig"][1]),
                            C.c_double(margin), C.c_double(gap), C.c_uint64(seed), _dp(cx), _dp(cy), _dp(r),
                            _dp(sig), _dp(gseed))
    return dict(cx=cx[:got], cy=cy[:got], r=r[:got], sig=sig[:got], gseed=gseed[:got])


def render(p: dict, grains: dict, dx, dy, th, noise_seed: int, disto=None) -> np.ndarray:
    L = _synth_lib()
    n = grains["cx"].shape[0]
    out = np.zeros((p["dimy"], p["dimx"]), dtype=np.uint16)
    dx = np.ascontiguousarray(dx, dtype=np.float64)
    dy = np.ascontiguousarray(dy, dtype=np.float64)
    th = np.ascontiguousarray(th, dtype=np.float64)
    dp = _dp(np.ascontiguousarray(disto, dtype=np.float64)) if disto is not None else None
    keep = np.ascontiguousarray(disto, dtype=np.float64) if disto is not None else None  # noqa: F841
    L.ptk_synth_render(C.c_int(p["dimx"]), C.c_int(p["dimy"]), C.c_int(p["maxval"]), C.c_double(p["bg"]),
                       C.c_double(p["noise"]), C.c_double(p["density"]), C.c_double(p["amp"][0]),
                       C.c_double(p["amp"][1]), C.c_int(n), _dp(grains["cx"]), _dp(grains["cy"]),
                       _dp(grains["r"]), _dp(grains["sig"]), _dp(grains["gseed"]), _dp(dx), _dp(dy), _dp(th),
                       dp, C.c_uint64(noise_seed), C.c_int(_threads()), _dp(out))
    return out


def start_records(grains: dict) -> np.ndarray:
    """13-column records of the 4-column start form (refrot 0)."""
    n = grains["cx"].shape[0]
    rec = np.zeros((n, 13))
    fx, fy = np.floor(grains["cx"]), np.floor(grains["cy"])
    rec[:, 0], rec[:, 1] = fx, fy
    rec[:, 3] = grains["r"]
    rec[:, 4] = rec[:, 7] = grains["cx"] - fx
    rec[:, 5] = rec[:, 8] = grains["cy"] - fy
    return rec


def anchor_truth(grains: dict, rec: np.ndarray, dx, dy, th) -> np.ndarray:
    """Expected (dx, dy, drot) columns after tracking the pair: the pattern
    anchor refcoord moves to c + d + R(theta)(refcoord - c)."""
    c, s = np.cos(th), np.sin(th)
    vx = rec[:, 0] - grains["cx"]
    vy = rec[:, 1] - grains["cy"]
    tx = grains["cx"] + dx + c * vx + s * vy
    ty = grains["cy"] + dy - s * vx + c * vy
    return np.stack([tx - rec[:, 0], ty - rec[:, 1], np.asarray(th, dtype=np.float64)], axis=1)


def make_pair(name_or_params, seed: int = 1, n: int | None = None) -> dict:
    """Reference/current frames of one preset, the start records and the truth."""
    p = PRESETS[name_or_params] if isinstance(name_or_params, str) else name_or_params
    grains = place(p, seed, n)
    ng = grains["cx"].shape[0]
    rng = np.random.default_rng(seed + 7919)
    dx = rng.uniform(-p["disp"], p["disp"], ng)
    dy = rng.uniform(-p["disp"], p["disp"], ng)
    th = rng.uniform(-p["rot"], p["rot"], ng)
    zeros = np.zeros(ng)
    ref = render(p, grains, zeros, zeros, zeros, noise_seed=seed * 2 + 1)
    cur = render(p, grains, dx, dy, th, noise_seed=seed * 2 + 2)
    if p["maxval"] <= 255:
        ref, cur = ref.astype(np.uint8), cur.astype(np.uint8)
    rec = start_records(grains)
    return dict(params=p, ref=ref, cur=cur, rec=rec, grains=grains, motion=np.stack([dx, dy, th], 1),
                truth=anchor_truth(grains, rec, dx, dy, th))


def tracker_options(p: dict) -> dict:
    """Options of the tracking context for a preset (command-file tokens)."""
    z = p["zone"]
    zones = [(z, z, z, z, p["num_rot"], p["inc_rot"])]
    rz = p.get("rescue_zone", 0)
    if rz:
        zones.append((rz, rz, rz, rz, p["num_rot"], p["inc_rot"]))
        level = 1
    else:
        zones.append(None)
        level = 0
    zones.append(None)
    return dict(zones=zones, rescue_level=level, NCC_min=0.7)


def distortion_params(p: dict) -> np.ndarray:
    """14 undistor parameters (src/p-tracker.hpp:151-165) of a preset."""
    k1, k2 = p["disto"]
    X = np.zeros(14)
    X[0], X[1] = 0.5 * p["dimx"], 0.5 * p["dimy"]
    X[2], X[3] = k1, k2
    X[8], X[9] = 0.5 * p["dimx"], 0.5 * p["dimy"]
    return X


def sequence_motion(p: dict, grains: dict, seed: int):
    """Cumulative per-frame motion of the cfg5 sequence: a smooth shear field
    growing linearly to p['shear'] px at the frame edges, a rotation random
    walk, and a one-off jump for a fraction of the grains."""
    ng = grains["cx"].shape[0]
    nf = p["frames"]
    rng = np.random.default_rng(seed + 104729)
    yc = 0.5 * p["dimy"]
    rot = np.cumsum(rng.normal(0.0, p["rot_walk"], (nf, ng)), axis=0)
    rot[0] = 0.0
    jumpers = rng.random(ng) < p["jump_frac"]
    jump_frame = rng.integers(1, nf, ng)
    ang = rng.uniform(0, 2 * math.pi, ng)
    out = []
    for k in range(nf):
        gamma = p["shear"] * k / max(1, nf - 1) / yc
        dxk = gamma * (grains["cy"] - yc)
        dyk = np.zeros(ng)
        j = jumpers & (jump_frame <= k)
        dxk = dxk + np.where(j, p["jump"] * np.cos(ang), 0.0)
        dyk = dyk + np.where(j, p["jump"] * np.sin(ang), 0.0)
        out.append((dxk, dyk, rot[k]))
    return out, jumpers, jump_frame


def make_sequence(name_or_params, seed: int = 1, frames: int | None = None) -> dict:
    """Frames of a cfg5-style sequence: the preset's grains moved by
    sequence_motion (shear field, rotation walk, jumps), rendered through the
    preset's radial distortion when it has one.  Returns the uint16 frames, the
    start records, the 14 undistor parameters (or None), the motion and the
    jumpers."""
    p = dict(PRESETS[name_or_params] if isinstance(name_or_params, str) else name_or_params)
    if frames is not None:
        p["frames"] = frames
    grains = place(p, seed)
    motion, jumpers, jump_frame = sequence_motion(p, grains, seed)
    disto = distortion_params(p) if p.get("disto") else None
    out = [render(p, grains, dx, dy, th, noise_seed=seed * 1000 + k, disto=disto)
           for k, (dx, dy, th) in enumerate(motion)]
    return dict(params=p, frames=out, rec=start_records(grains), grains=grains, disto=disto, motion=motion,
                jumpers=jumpers, jump_frame=jump_frame)


def make_disto_case(seed: int = 1, n: int = 2000, n_tracked: int = 3, dimx: int = 5616, dimy: int = 3744,
                    k1: float = -2e-9, k2: float = 1e-16, noise: float = 0.01, low_ncc: float = 0.03) -> dict:
    """Inputs of the distortion-parameter fit (correction_distortion): n grains
    at integer reference positions of a dimx x dimy frame seen through the
    radial lens (k1, k2) about the frame centre, and the displacements a
    tracker reports in n_tracked images where the scene moved by one
    translation each (+-20 px, equiprojective), plus Gaussian tracking noise
    (px) and a fraction of failed grains (NCC_subpix 0.3; the others 0.98).
    The distorted positions invert the radial model by fixed-point iteration."""
    rng = np.random.default_rng(seed)
    X = distortion_params(dict(dimx=dimx, dimy=dimy, disto=(k1, k2)))
    xc, yc = X[0], X[1]
    w = dimx - 200
    cell = rng.choice(w * (dimy - 200), size=n, replace=False)  # distinct positions: no pair of length 0
    refx = (100 + cell % w).astype(np.int32)
    refy = (100 + cell // w).astype(np.int32)

    def radial(x, y):
        r2 = (x - xc) ** 2 + (y - yc) ** 2
        return k1 * r2 + k2 * r2 * r2

    f = radial(refx.astype(np.float64), refy.astype(np.float64))
    ux = refx + (refx - xc) * f
    uy = refy + (refy - yc) * f
    dx = np.zeros((n_tracked, n))
    dy = np.zeros((n_tracked, n))
    for im in range(n_tracked):
        t = rng.uniform(-20.0, 20.0, 2)
        tx, ty = ux + t[0], uy + t[1]
        xd, yd = tx.copy(), ty.copy()
        for _ in range(30):  # xu = xd + (xd - xc) f(xd): contraction, |f| < 0.03 on the frame
            g = radial(xd, yd)
            xd = xc + (tx - xc) / (1.0 + g)
            yd = yc + (ty - yc) / (1.0 + g)
        dx[im] = xd - refx + rng.normal(0.0, noise, n)
        dy[im] = yd - refy + rng.normal(0.0, noise, n)
    ncc = np.where(rng.random((n_tracked, n)) < low_ncc, 0.3, 0.98)
    return dict(X=X, refx=refx, refy=refy, dx=dx, dy=dy, ncc=ncc, dimx=dimx, dimy=dimy)
