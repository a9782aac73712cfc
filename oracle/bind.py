"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes access to the two CPU checkers:
  * `Port`      -- oracle/port/ptk_oracle.cpp, the project's restatement
                   (oracle/_build/libptk_oracle.so, always buildable);
  * `Reference` -- the reference's own sources compiled by oracle/Makefile
                   (oracle/_ref/libptk_ref.so; built where the reference
                   sources exist, shipped as a built file elsewhere).
Both expose the same methods so a test can run one scenario on either.  Only
tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_SO = HERE / "_build" / "libptk_oracle.so"
REF_SO = HERE / "_ref" / "libptk_ref.so"
# the reference checkout sits beside this repository (sibling directory
# reference/) unless PTK_REFERENCE_SRC names its src/ directory
REF_SRC = Path(os.environ.get("PTK_REFERENCE_SRC", str(HERE.parent.parent / "reference" / "src")))


def build(ref: bool = True) -> dict:
    """Builds the port, and the reference library when its sources exist."""
    subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    built_ref = False
    if ref and (REF_SRC / "p-tracker.cpp").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REFSRC={REF_SRC}"], check=True)
        built_ref = True
    return {"port": str(PORT_SO), "ref": str(REF_SO) if REF_SO.exists() else None, "ref_rebuilt": built_ref}


def have_reference() -> bool:
    return REF_SO.exists()


_D = C.c_double
_I = C.c_int
_P = C.c_void_p


def _p(a):
    return C.c_void_p(a.ctypes.data)


class _Base:
    prefix = ""
    so = None

    def __init__(self, dimx: int, dimy: int, threads: int = 1):
        L = C.CDLL(str(self.so))
        self.L = L
        pre = self.prefix
        self._f = lambda name: getattr(L, pre + name)
        self._f("create").restype = _P
        self._f("create").argtypes = [_I, _I]
        for nm in ("objective", "interp"):
            self._f(nm).restype = _D
        self.h = C.c_void_p(self._f("create")(dimx, dimy))
        self.dimx, self.dimy = dimx, dimy
        self.n = 0
        self.set_threads(threads)

    def close(self):
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, n: int):
        self._f("set_threads")(self.h, _I(int(n)))

    @staticmethod
    def _u16(img):
        return np.ascontiguousarray(img, dtype=np.uint16)

    def load_first(self, img):
        a = self._u16(img)
        self._f("load_first")(self.h, _p(a))

    def load_reference(self, img):
        a = self._u16(img)
        self._f("load_reference")(self.h, _p(a))

    def load_current(self, img):
        a = self._u16(img)
        self._f("load_current")(self.h, _p(a))

    def set_grains(self, rec13, masked=None):
        rec = np.ascontiguousarray(rec13, dtype=np.float64).reshape(-1, 13)
        self.n = rec.shape[0]
        m = np.ascontiguousarray(masked, dtype=np.uint8) if masked is not None else None
        self._f("set_grains")(self.h, _I(self.n), _p(rec), _p(m) if m is not None else None)

    def get_grains(self) -> np.ndarray:
        out = np.zeros((self.n, 13))
        self._f("get_grains")(self.h, _p(out))
        return out

    def get_precomp(self):
        m, c = np.zeros(self.n), np.zeros(self.n)
        self._f("get_precomp")(self.h, _p(m), _p(c))
        return m, c

    def set_pattern(self, g: int, xy):
        a = np.ascontiguousarray(xy, dtype=np.int32).reshape(-1, 2)
        self._f("set_pattern")(self.h, _I(g), _I(a.shape[0]), _p(a))

    def make_pattern(self, g: int, kind: int, a: int, b: int = 0):
        self._f("make_pattern")(self.h, _I(g), _I(kind), _I(int(a)), _I(int(b)))

    def grain_diameter_patterns(self, rec13, reduction: float = 1.0, min_radius: float = 1.0):
        """`pattern grain_diameter f rmin` (src/p-tracker.cpp:1656-1666)."""
        for g in range(self.n):
            radius = int(rec13[g, 3] * reduction)
            if radius < min_radius:
                radius = int(min_radius)
            self.make_pattern(g, 0, radius)

    def pattern(self, g: int, which: int = 0) -> np.ndarray:
        n = self._f("pattern_size")(self.h, _I(g))
        out = np.zeros((n, 2), dtype=np.int32)
        self._f("get_pattern")(self.h, _I(g), _I(which), _p(out))
        return out

    def set_zone(self, level, left, right, up, down, num_rot, inc_rot):
        self._f("set_zone")(self.h, _I(level), _I(left), _I(right), _I(up), _I(down), _I(num_rot), _D(inc_rot))

    def set_param(self, key: str, v: float):
        rc = self._f("set_param")(self.h, key.encode(), _D(float(v)))
        if rc != 0:
            raise KeyError(key)

    def precompute(self):
        self._f("precompute")(self.h)

    def pixel_all(self) -> int:
        return self._f("pixel_all")(self.h)

    def rescue_all(self) -> int:
        return self._f("rescue_all")(self.h)

    def super_rescue_all(self):
        self._f("super_rescue_all")(self.h)

    def subpixel_all(self):
        self._f("subpixel_all")(self.h)

    def end_frame(self, num_image: int):
        self._f("end_frame")(self.h, _I(num_image))

    def track_frame(self, num_image: int):
        self._f("track_frame")(self.h, _I(num_image))

    def lists(self):
        a = np.zeros(max(self.n, 1), dtype=np.int32)
        b = np.zeros(max(self.n, 1), dtype=np.int32)
        ns = C.c_int()
        nr = self._f("get_lists")(self.h, _p(a), _p(b), C.byref(ns))
        return sorted(a[:nr].tolist()), sorted(b[:ns.value].tolist())

    def objective(self, g: int, X) -> float:
        x = np.ascontiguousarray(X, dtype=np.float64)
        return float(self._f("objective")(self.h, _I(g), _p(x)))

    def interp(self, kind: int, slot: int, x: float, y: float) -> float:
        return float(self._f("interp")(self.h, _I(kind), _I(slot), _D(x), _D(y)))

    def indices(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        self._f("get_indices")(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value


class Port(_Base):
    prefix = "orc_"
    so = PORT_SO

    def __init__(self, dimx, dimy, threads=1):
        super().__init__(dimx, dimy, threads)
        self._f("gradient").restype = _D

    def top2(self) -> np.ndarray:
        out = np.zeros((self.n, 2))
        self._f("get_top2")(self.h, _p(out))
        return out

    def gradient(self, g: int, X):
        x = np.ascontiguousarray(X, dtype=np.float64)
        gr = np.zeros(3)
        f = self._f("gradient")(self.h, _I(g), _p(x), _p(gr))
        return float(f), gr

    def save_grains(self, path: str, from_name: str, to_name: str):
        self._f("save_grains")(self.h, str(path).encode(), from_name.encode(), to_name.encode())


class Reference(_Base):
    prefix = "ref_"
    so = REF_SO

    def save_grains(self, path: str, num: int):
        self._f("save_grains")(self.h, str(path).encode(), _I(num))

    def undistor(self, params14, xd: float, yd: float):
        p = np.ascontiguousarray(params14, dtype=np.float64)
        xu, yu = C.c_double(), C.c_double()
        self._f("undistor")(self.h, _p(p), _D(xd), _D(yd), C.byref(xu), C.byref(yu))
        return xu.value, yu.value


def rotation_steps(inc_rot: float, num_rot: int) -> np.ndarray:
    L = C.CDLL(str(PORT_SO))
    out = np.zeros(8192)
    n = L.orc_rotation_steps(_D(inc_rot), _I(num_rot), _p(out), _I(8192))
    return out[:n].copy()


def undistor(params14, xd: float, yd: float):
    L = C.CDLL(str(PORT_SO))
    p = np.ascontiguousarray(params14, dtype=np.float64)
    xu, yu = C.c_double(), C.c_double()
    L.orc_undistor(_p(p), _D(xd), _D(yd), C.byref(xu), C.byref(yu))
    return xu.value, yu.value


def _disto_lib(reference: bool):
    return C.CDLL(str(REF_SO if reference else PORT_SO))


def disto_pairs(refx, refy, dmin: float, dmax: float, reference: bool = False) -> np.ndarray:
    """precompute_paires: the port's restatement, or the reference's member
    function run on grains placed at refx, refy."""
    L = _disto_lib(reference)
    rx = np.ascontiguousarray(refx, dtype=np.int32)
    ry = np.ascontiguousarray(refy, dtype=np.int32)
    n = rx.shape[0]
    cap = n * (n - 1) // 2 + 1
    out = np.zeros((cap, 2), dtype=np.int32)
    if reference:
        L.ref_create.restype = _P
        L.ref_disto_pairs.restype = C.c_int64
        h = C.c_void_p(L.ref_create(8, 8))
        np_ = L.ref_disto_pairs(h, _p(rx), _p(ry), _I(n), _D(dmin), _D(dmax), _p(out), C.c_int64(cap))
        L.ref_destroy(h)
    else:
        L.orc_disto_pairs.restype = C.c_int64
        np_ = L.orc_disto_pairs(_p(rx), _p(ry), _I(n), _D(dmin), _D(dmax), _p(out), C.c_int64(cap))
    return out[:np_].copy()


def disto_objective(params14, refx, refy, dx, dy, ncc, NCC_min: float, pairs, origx=None, origy=None,
                    reference: bool = False, with_residuals: bool = False):
    """The equiprojectivity criterion (POWELL functor; with origx/origy the
    POWELL_ITER functor): the port's restatement, or the loop around the
    reference's own undistor."""
    L = _disto_lib(reference)
    X = np.ascontiguousarray(params14, dtype=np.float64)
    rx = np.ascontiguousarray(refx, dtype=np.int32)
    ry = np.ascontiguousarray(refy, dtype=np.int32)
    ddx = np.ascontiguousarray(dx, dtype=np.float64)
    ddy = np.ascontiguousarray(dy, dtype=np.float64)
    nc = np.ascontiguousarray(ncc, dtype=np.float64)
    pr = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    n, nimg1 = rx.shape[0], ddx.shape[0]
    use_orig = origx is not None
    ox = np.ascontiguousarray(origx if use_orig else rx, dtype=np.float64)
    oy = np.ascontiguousarray(origy if use_orig else ry, dtype=np.float64)
    if reference:
        L.ref_create.restype = _P
        L.ref_disto_objective.restype = _D
        h = C.c_void_p(L.ref_create(8, 8))
        v = L.ref_disto_objective(h, _p(X), _p(rx), _p(ry), _p(ox), _p(oy), _I(n), _I(nimg1), _p(ddx), _p(ddy), _p(nc),
                                  _D(NCC_min), _p(pr), C.c_int64(pr.shape[0]), _I(int(use_orig)))
        L.ref_destroy(h)
        return v
    L.orc_disto_objective.restype = _D
    f = np.zeros(nimg1 * pr.shape[0])
    v = L.orc_disto_objective(_p(X), _p(rx), _p(ry), _p(ox), _p(oy), _I(n), _I(nimg1), _p(ddx), _p(ddy), _p(nc),
                              _D(NCC_min), _p(pr), C.c_int64(pr.shape[0]), _I(int(use_orig)),
                              _p(f) if with_residuals else None)
    return (v, f) if with_residuals else v


def disto_fit(params14, perturb14, algo: int, num_iter: int, dimx: int, dimy: int, refx, refy, dx, dy, ncc,
              NCC_min: float, pairs):
    """The port's minimisation of correction_distortion (POWELL = 0,
    POWELL_ITER = 1) with the oracle Powell; returns (params, index_ini,
    index_end, history, dx, dy)."""
    L = _disto_lib(False)
    X = np.array(params14, dtype=np.float64)
    DX = np.ascontiguousarray(perturb14, dtype=np.float64)
    rx = np.ascontiguousarray(refx, dtype=np.int32)
    ry = np.ascontiguousarray(refy, dtype=np.int32)
    ddx = np.array(dx, dtype=np.float64)
    ddy = np.array(dy, dtype=np.float64)
    nc = np.ascontiguousarray(ncc, dtype=np.float64)
    pr = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    ini, end = C.c_double(), C.c_double()
    hist = np.zeros((max(num_iter, 1), 15))
    L.orc_disto_fit(_p(X), _p(DX), _I(algo), _I(num_iter), _I(dimx), _I(dimy), _p(rx), _p(ry), _I(rx.shape[0]),
                    _I(ddx.shape[0]), _p(ddx), _p(ddy), _p(nc), _D(NCC_min), _p(pr), C.c_int64(pr.shape[0]),
                    C.byref(ini), C.byref(end), _p(hist))
    return X, ini.value, end.value, (hist[:num_iter] if algo == 1 else hist[:0]), ddx, ddy


def remap(params14, src: np.ndarray, threads: int = 1) -> np.ndarray:
    L = C.CDLL(str(PORT_SO))
    p = np.ascontiguousarray(params14, dtype=np.float64)
    s = np.ascontiguousarray(src, dtype=np.uint16)
    out = np.zeros_like(s)
    L.orc_remap(_p(p), _p(s), _I(s.shape[1]), _I(s.shape[0]), _p(out), _I(threads))
    return out


def raw_demosaic(raw: np.ndarray, width: int, height: int, left: int, top: int, mode: int, rescale: bool,
                 reference: bool = False):
    """Grey frame (height, width) from an unpacked RAW mosaic (raw_height,
    raw_width) with DemosaicModel `mode` (-1, -2, -20): the port's
    restatement (returns (frame, (MinGray, MaxGray)), or None when a stencil
    leaves the array), or the reference's own read_raw_image on the mosaic
    (returns (frame, None))."""
    r = np.ascontiguousarray(raw, dtype=np.uint16)
    out = np.zeros((height, width), dtype=np.uint16)
    if reference:
        L = C.CDLL(str(REF_SO))
        L.ref_create.restype = _P
        h = C.c_void_p(L.ref_create(8, 8))
        L.ref_raw_demosaic(h, _p(r), _I(r.shape[1]), _I(r.shape[0]), _I(width), _I(height), _I(left), _I(top),
                           _I(mode), _I(int(rescale)), _p(out))
        L.ref_destroy(h)
        return out, None
    L = C.CDLL(str(PORT_SO))
    mm = np.zeros(2, dtype=np.uint16)
    rc = L.orc_raw_demosaic(_p(r), _I(r.shape[1]), _I(r.shape[0]), _I(width), _I(height), _I(left), _I(top),
                            _I(mode), _I(int(rescale)), _p(out), _p(mm))
    return None if rc != 0 else (out, (int(mm[0]), int(mm[1])))


def setup(cls, pair: dict, threads: int = 1, zones=None, params: dict | None = None, pattern=("grain_diameter", 1.0, 1.0)):
    """Builds a checker (Port or Reference) for a workload pair."""
    p = pair["params"]
    t = cls(p["dimx"], p["dimy"], threads)
    t.load_first(pair["ref"])
    t.load_current(pair["cur"])
    t.set_grains(pair["rec"])
    kind = pattern[0]
    if kind == "grain_diameter":
        t.grain_diameter_patterns(pair["rec"], pattern[1], pattern[2])
    else:
        k = {"circ": 0, "ring": 1, "rect": 2}[kind]
        for g in range(t.n):
            t.make_pattern(g, k, pattern[1], pattern[2] if len(pattern) > 2 else 0)
    for lvl, z in enumerate(zones or []):
        if z is not None:
            t.set_zone(lvl, *z)
    for k, v in (params or {}).items():
        t.set_param(k, v)
    return t
