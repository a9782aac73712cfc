"""ctypes binding of the sm_100a tracking path (include/ptk.h).

The product is the C ABI in libptk.so; this module exposes it to Python for
the tests and the benchmark.  `Tracker` mirrors the part of the reference's
`ptracker` class that particle tracking uses (src/p-tracker.hpp:66-238):
search zones, grains, patterns, the two frames, and the stages
do_precomputations / follow_pattern_* / follow_pattern_subpixel_xyR, batched
over all grains.  Grains travel as (n, 13) float64 arrays in dic_out column
order (src/p-tracker.cpp:1330-1343).

There is no CPU fallback: importing this module without the built library
raises, and a Tracker cannot be created without a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

COLUMNS = ("refcoord_xpix", "refcoord_ypix", "refrot", "radius_pix", "dx", "dy", "drot",
           "upix", "vpix", "rot_inc", "NCC", "NCC_rescue", "NCC_subpix")

PTK_OK, PTK_ERR_ARG, PTK_ERR_STATE, PTK_ERR_CUDA, PTK_ERR_IO, PTK_ERR_LIMIT, PTK_ERR_TIMEOUT = range(7)
ST_RESCUED, ST_SUPER_RESCUED, ST_FAILED, ST_OUT_OF_BOUNDS, ST_MASKED, ST_SUBPIX_CLAMPED = 1, 2, 4, 8, 16, 32
INTERP = {"linear": 0, "cubic": 1, "quintic": 2}
SUBPIX_POWELL, SUBPIX_ADJOINT_LM = 0, 1
SEARCH_EXACT, SEARCH_BF16 = 0, 1
DEMOSAIC_BOX2, DEMOSAIC_BINOMIAL3, DEMOSAIC_GREY = -1, -2, -20
PATTERN = {"circ": 0, "ring": 1, "rect": 2, "grain_diameter": 3}


class Zone(C.Structure):
    _fields_ = [("left", C.c_int32), ("right", C.c_int32), ("up", C.c_int32), ("down", C.c_int32),
                ("num_rot", C.c_int32), ("inc_rot", C.c_double)]


class Grain(C.Structure):
    _fields_ = [("refcoord_xpix", C.c_int32), ("refcoord_ypix", C.c_int32)] + \
               [(k, C.c_double) for k in COLUMNS[2:]] + \
               [("masked", C.c_uint8), ("status", C.c_uint8), ("pad_", C.c_uint8 * 6)]


class Config(C.Structure):
    _fields_ = [("dimx", C.c_int32), ("dimy", C.c_int32), ("rescue_level", C.c_int32),
                ("NCC_min", C.c_double), ("NCC_min_super", C.c_double), ("subpixel", C.c_int32),
                ("subpix_tol", C.c_double), ("initial_direction", C.c_double * 3),
                ("image_interpolator", C.c_int32), ("overflow_stiffness", C.c_double),
                ("subpix_displacement_max", C.c_double), ("rotations", C.c_int32), ("zone", Zone * 3),
                ("iraz", C.c_int32), ("subpix_method", C.c_int32), ("search_method", C.c_int32),
                ("topk", C.c_int32), ("lm_max_iter", C.c_int32), ("lm_tol", C.c_double),
                ("autotune", C.c_int32), ("lm_cell_px", C.c_double), ("lm_cell_rot", C.c_double)]


class TuneReport(C.Structure):
    _fields_ = [("method", C.c_int32), ("choice", C.c_int32), ("n", C.c_int32), ("values", C.c_int32 * 8),
                ("ms", C.c_float * 8)]


GRAIN_DTYPE = np.dtype({"names": ["refx", "refy"] + list(COLUMNS[2:]) + ["masked", "status", "pad"],
                        "formats": ["<i4", "<i4"] + ["<f8"] * 11 + ["u1", "u1", ("u1", 6)],
                        "offsets": [0, 4] + [8 + 8 * k for k in range(11)] + [96, 97, 98],
                        "itemsize": 104})

_P = C.c_void_p
_SIGS = {
    "ptk_config_default": (C.c_int, [C.POINTER(Config)]),
    "ptk_create": (C.c_int, [C.POINTER(_P), C.POINTER(Config)]),
    "ptk_destroy": (C.c_int, [_P]),
    "ptk_set_config": (C.c_int, [_P, C.POINTER(Config)]),
    "ptk_set_search_zone": (C.c_int, [_P, C.c_int, C.POINTER(Zone)]),
    "ptk_set_grains": (C.c_int, [_P, _P, C.c_int]),
    "ptk_get_grains": (C.c_int, [_P, _P, C.c_int]),
    "ptk_snapshot_grains": (C.c_int, [_P]),
    "ptk_restore_grains": (C.c_int, [_P]),
    "ptk_set_patterns": (C.c_int, [_P, _P, _P, C.c_int]),
    "ptk_make_patterns": (C.c_int, [_P, C.c_int, C.c_double, C.c_double, C.c_double]),
    "ptk_pattern_size": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "ptk_load_frame": (C.c_int, [_P, C.c_int, _P, C.c_int, C.c_int, C.c_int, C.c_size_t]),
    "ptk_load_frame_device": (C.c_int, [_P, C.c_int, _P, C.c_size_t]),
    "ptk_host_alloc": (C.c_int, [C.POINTER(_P), C.c_size_t]),
    "ptk_host_free": (C.c_int, [_P]),
    "ptk_autotune": (C.c_int, [_P, C.POINTER(TuneReport)]),
    "ptk_load_frame_raw": (C.c_int, [_P, C.c_int, _P] + [C.c_int] * 6 + [_P]),
    "ptk_load_frame_raw_device": (C.c_int, [_P, C.c_int, _P] + [C.c_int] * 6 + [_P]),
    "ptk_read_frame": (C.c_int, [_P, C.c_int, _P]),
    "ptk_precompute": (C.c_int, [_P]),
    "ptk_search": (C.c_int, [_P, C.c_int]),
    "ptk_search_timed": (C.c_int, [_P, C.c_int, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_int)]),
    "ptk_read_image_file": (C.c_int, [C.c_char_p, _P, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p,
                                      C.c_int]),
    "ptk_image_error": (C.c_char_p, []),
    "ptk_subpixel": (C.c_int, [_P, C.c_int]),
    "ptk_end_frame": (C.c_int, [_P, C.c_int]),
    "ptk_track_frame": (C.c_int, [_P, C.c_int]),
    "ptk_swap_reference": (C.c_int, [_P, C.c_int]),
    "ptk_set_iref": (C.c_int, [_P, C.c_int]),
    "ptk_get_rescue_counts": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "ptk_objective": (C.c_int, [_P, _P, _P]),
    "ptk_grad": (C.c_int, [_P, _P, _P, _P]),
    "ptk_set_distortion": (C.c_int, [_P, _P]),
    "ptk_remap_frame": (C.c_int, [_P, C.c_int]),
    "ptk_set_stream": (C.c_int, [_P, _P]),
    "ptk_get_stream": (_P, [_P]),
    "ptk_synchronize": (C.c_int, [_P]),
    "ptk_kernel_launches": (C.c_int64, [_P]),
    "ptk_test_bf16_wait_timeout": (C.c_int, [_P, C.c_int]),
    "ptk_set_tune_cache": (C.c_int, [_P, C.c_char_p]),
    "ptk_tune_signature": (C.c_int, [_P, C.c_char_p, C.c_int32]),
    "ptk_tune_cache_lookup": (C.c_int, [C.c_char_p, C.c_char_p] + [C.POINTER(C.c_int32)] * 3),
    "ptk_tune_cache_store": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int32, C.c_int32, C.c_int32,
                                       C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "ptk_abi_sizes": (C.c_int, [C.POINTER(C.c_size_t)] * 3),
    "ptk_search_pixel_noalloc": (C.c_int, [_P, _P, C.c_size_t, C.c_int, C.c_int, C.c_int] + [_P] * 8 +
                                 [C.c_int, C.c_int, C.POINTER(Zone), C.c_int] + [_P] * 5),
    "ptk_last_error": (C.c_char_p, [_P]),
    "ptk_read_grains_file": (C.c_int, [C.c_char_p, C.c_int, _P, C.c_int, C.POINTER(C.c_int)]),
    "ptk_save_grains_file": (C.c_int, [C.c_char_p, _P, C.c_int, C.c_char_p, C.c_char_p, C.c_char_p,
                                       C.c_char_p]),
    "ptk_disto_pairs": (C.c_int, [_P, _P, C.c_int, C.c_double, C.c_double, _P, C.c_int64, C.POINTER(C.c_int64)]),
    "ptk_disto_create": (C.c_int, [C.POINTER(_P), C.c_int, C.c_int, _P, _P, C.c_int, C.c_int, _P, _P, _P,
                                   C.c_double, _P, C.c_int64]),
    "ptk_disto_destroy": (C.c_int, [_P]),
    "ptk_disto_last_error": (C.c_char_p, [_P]),
    "ptk_disto_objective": (C.c_int, [_P, _P, C.POINTER(C.c_double)]),
    "ptk_disto_residuals": (C.c_int, [_P, _P, C.POINTER(C.c_double), _P]),
    "ptk_disto_fit": (C.c_int, [_P, _P, _P, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), _P]),
    "ptk_disto_tracked": (C.c_int, [_P, _P, _P]),
    "ptk_disto_levmar_info": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_char_p)]),
    "ptk_disto_objective_timed": (C.c_int, [_P, _P, C.c_int, _P]),
}

_lib = None
_synth = None


def lib_path() -> Path:
    return HERE / "libptk.so"


def lib() -> C.CDLL:
    """Loads libptk.so (built in-tree by build.py); raises if it is missing."""
    global _lib
    if _lib is None:
        p = lib_path()
        if not p.exists():
            raise RuntimeError(f"{p} is missing: run p-tracker_b200/build.py (no CPU fallback exists)")
        L = C.CDLL(str(p))
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def synth() -> C.CDLL:
    global _synth
    if _synth is None:
        p = HERE / "libptk_synth.so"
        if not p.exists():
            raise RuntimeError(f"{p} is missing: run p-tracker_b200/build.py")
        L = C.CDLL(str(p))
        L.ptk_synth_place.restype = C.c_int
        L.ptk_synth_render.restype = C.c_int
        _synth = L
    return _synth


class PtkError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ptk error {code}: {msg}")
        self.code = code


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def default_config(dimx: int, dimy: int) -> Config:
    cfg = Config()
    lib().ptk_config_default(C.byref(cfg))
    cfg.dimx, cfg.dimy = dimx, dimy
    return cfg


def records_to_structs(rec: np.ndarray, masked: np.ndarray | None = None) -> np.ndarray:
    rec = np.asarray(rec, dtype=np.float64).reshape(-1, 13)
    out = np.zeros(rec.shape[0], dtype=GRAIN_DTYPE)
    out["refx"] = rec[:, 0].astype(np.int32)
    out["refy"] = rec[:, 1].astype(np.int32)
    for k, name in enumerate(COLUMNS[2:], start=2):
        out[name] = rec[:, k]
    if masked is not None:
        out["masked"] = np.asarray(masked, dtype=np.uint8)
    return out


def structs_to_records(s: np.ndarray) -> np.ndarray:
    rec = np.zeros((s.shape[0], 13))
    rec[:, 0] = s["refx"]
    rec[:, 1] = s["refy"]
    for k, name in enumerate(COLUMNS[2:], start=2):
        rec[:, k] = s[name]
    return rec


class Tracker:
    """One tracking context on the current CUDA device."""

    def __init__(self, dimx: int, dimy: int, **options):
        self._L = lib()
        self.cfg = default_config(dimx, dimy)
        for k, v in options.items():
            self._set_option(k, v)
        h = C.c_void_p()
        self._check(self._L.ptk_create(C.byref(h), C.byref(self.cfg)), None)
        self.h = h
        self.n = 0

    def _set_option(self, k, v):
        if k == "image_interpolator" and isinstance(v, str):
            v = INTERP[v]
        if k == "initial_direction":
            for i in range(3):
                self.cfg.initial_direction[i] = v[i]
        elif k == "zones":
            for lvl, z in enumerate(v):
                if z is not None:
                    self.cfg.zone[lvl] = Zone(*z)
        else:
            setattr(self.cfg, k, v)

    def _check(self, rc: int, h=None):
        if rc != PTK_OK:
            msg = self._L.ptk_last_error(h if h is not None else getattr(self, "h", None))
            raise PtkError(rc, (msg or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            self._L.ptk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- configuration -------------------------------------------------------
    def configure(self, **options):
        for k, v in options.items():
            self._set_option(k, v)
        self._check(self._L.ptk_set_config(self.h, C.byref(self.cfg)), self.h)

    def set_zone(self, level: int, left: int, right: int, up: int, down: int, num_rot: int, inc_rot: float):
        z = Zone(left, right, up, down, num_rot, inc_rot)
        self._check(self._L.ptk_set_search_zone(self.h, level, C.byref(z)), self.h)
        self.cfg.zone[level] = z

    # -- grains and patterns -------------------------------------------------
    def set_grains(self, rec13: np.ndarray, masked=None):
        s = records_to_structs(rec13, masked)
        self.n = s.shape[0]
        self._check(self._L.ptk_set_grains(self.h, _ptr(s), self.n), self.h)

    def get_grains_structs(self) -> np.ndarray:
        s = np.zeros(self.n, dtype=GRAIN_DTYPE)
        self._check(self._L.ptk_get_grains(self.h, _ptr(s), self.n), self.h)
        return s

    def get_grains(self) -> np.ndarray:
        return structs_to_records(self.get_grains_structs())

    def snapshot_grains(self):
        self._check(self._L.ptk_snapshot_grains(self.h), self.h)

    def restore_grains(self):
        self._check(self._L.ptk_restore_grains(self.h), self.h)

    def status(self) -> np.ndarray:
        return self.get_grains_structs()["status"].copy()

    def make_patterns(self, kind: str, a: float, b: float = 0.0, target_radius: float = -1.0):
        self._check(self._L.ptk_make_patterns(self.h, PATTERN[kind], a, b, target_radius), self.h)

    def set_patterns(self, patterns: list):
        starts = np.zeros(len(patterns) + 1, dtype=np.int64)
        starts[1:] = np.cumsum([len(p) for p in patterns])
        xy = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.int32).reshape(-1, 2) for p in patterns])
                                  if patterns else np.zeros((0, 2), np.int32))
        self._check(self._L.ptk_set_patterns(self.h, _ptr(xy), _ptr(starts), len(patterns)), self.h)

    def pattern_size(self, g: int) -> int:
        n = C.c_int()
        self._check(self._L.ptk_pattern_size(self.h, g, C.byref(n)), self.h)
        return n.value

    # -- frames --------------------------------------------------------------
    def load_frame(self, slot: int, img: np.ndarray):
        img = np.ascontiguousarray(img)
        bpp = img.dtype.itemsize
        if img.dtype not in (np.uint8, np.uint16):
            raise ValueError("frames are uint8 or uint16")
        self._check(self._L.ptk_load_frame(self.h, slot, _ptr(img), img.shape[1], img.shape[0], bpp,
                                           img.strides[0]), self.h)

    def load_frame_device(self, slot: int, dev_ptr: int, pitch_bytes: int):
        self._check(self._L.ptk_load_frame_device(self.h, slot, C.c_void_p(dev_ptr), pitch_bytes), self.h)

    def load_frame_raw(self, slot: int, raw: np.ndarray, left_margin: int, top_margin: int, mode: int,
                       rescale: bool = False) -> tuple[int, int]:
        """A frame from an unpacked RAW mosaic (raw_height, raw_width) uint16,
        demosaiced on the GPU with DemosaicModel `mode` (-1, -2, -20);
        returns (MinGray, MaxGray)."""
        r = np.ascontiguousarray(raw, dtype=np.uint16)
        mm = np.zeros(2, dtype=np.uint16)
        self._check(self._L.ptk_load_frame_raw(self.h, slot, _ptr(r), r.shape[1], r.shape[0], left_margin,
                                               top_margin, mode, int(rescale), _ptr(mm)), self.h)
        return int(mm[0]), int(mm[1])

    def load_frame_raw_device(self, slot: int, dev_ptr: int, raw_width: int, raw_height: int, left_margin: int,
                              top_margin: int, mode: int, rescale: bool = False):
        """Same with the mosaic in device memory; does not wait for the GPU."""
        self._check(self._L.ptk_load_frame_raw_device(self.h, slot, C.c_void_p(dev_ptr), raw_width, raw_height,
                                                      left_margin, top_margin, mode, int(rescale), None), self.h)

    def read_frame(self, slot: int) -> np.ndarray:
        out = np.zeros((self.cfg.dimy, self.cfg.dimx), dtype=np.uint16)
        self._check(self._L.ptk_read_frame(self.h, slot, _ptr(out)), self.h)
        return out

    # -- stages ----------------------------------------------------------------
    def precompute(self):
        self._check(self._L.ptk_precompute(self.h), self.h)

    def search(self, level: int = 0):
        self._check(self._L.ptk_search(self.h, level), self.h)

    def autotune(self) -> dict:
        """Times the level-0 search shapes on the loaded frames and keeps the
        fastest (ptk_autotune): {"method": "bf16"|"exact", "choice": value,
        "candidates": {value: best ms}, "cached": bool} - with a tune cache
        set and an entry for this workload, nothing is timed ("cached": True,
        no candidates)."""
        r = TuneReport()
        self._check(self._L.ptk_autotune(self.h, C.byref(r)), self.h)
        return {"method": "bf16" if r.method else "exact", "choice": int(r.choice),
                "candidates": {int(r.values[k]): float(r.ms[k]) for k in range(r.n)}, "cached": r.n == 0}

    def set_tune_cache(self, path):
        """JSON file of autotune choices per (GPU, workload) signature
        (ptk_set_tune_cache); None turns the cache off."""
        self._check(self._L.ptk_set_tune_cache(self.h, None if path is None else str(path).encode()), self.h)

    def tune_signature(self) -> str:
        """The autotune cache key of this context's GPU and workload."""
        buf = C.create_string_buffer(1024)
        self._check(self._L.ptk_tune_signature(self.h, buf, len(buf)), self.h)
        return buf.value.decode()

    def search_timed(self, level: int = 0) -> list:
        """The level's search with CUDA events between its kernels: per-kernel
        milliseconds in launch order (see ptk_search_timed)."""
        ms = (C.c_float * 8)()
        n = C.c_int(0)
        self._check(self._L.ptk_search_timed(self.h, level, ms, 8, C.byref(n)), self.h)
        return [float(ms[k]) for k in range(n.value)]

    def subpixel(self, method: int = SUBPIX_POWELL):
        self._check(self._L.ptk_subpixel(self.h, method), self.h)

    def end_frame(self, num_image: int):
        self._check(self._L.ptk_end_frame(self.h, num_image), self.h)

    def track_frame(self, num_image: int):
        self._check(self._L.ptk_track_frame(self.h, num_image), self.h)

    def swap_reference(self, num_image: int):
        self._check(self._L.ptk_swap_reference(self.h, num_image), self.h)

    def set_iref(self, iref: int):
        self._check(self._L.ptk_set_iref(self.h, iref), self.h)

    def rescue_counts(self) -> tuple[int, int]:
        a, b = C.c_int(), C.c_int()
        self._check(self._L.ptk_get_rescue_counts(self.h, C.byref(a), C.byref(b)), self.h)
        return a.value, b.value

    def objective(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(self.n, 3)
        f = np.zeros(self.n)
        self._check(self._L.ptk_objective(self.h, _ptr(X), _ptr(f)), self.h)
        return f

    def grad(self, X: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float64).reshape(self.n, 3)
        f = np.zeros(self.n)
        g = np.zeros((self.n, 3))
        self._check(self._L.ptk_grad(self.h, _ptr(X), _ptr(f), _ptr(g)), self.h)
        return f, g

    def set_distortion(self, params14):
        p = np.ascontiguousarray(params14, dtype=np.float64)
        self._check(self._L.ptk_set_distortion(self.h, _ptr(p)), self.h)

    def remap(self, slot: int):
        self._check(self._L.ptk_remap_frame(self.h, slot), self.h)

    def set_stream(self, stream_ptr: int | None):
        self._check(self._L.ptk_set_stream(self.h, C.c_void_p(stream_ptr or 0)), self.h)

    def stream(self) -> int:
        return self._L.ptk_get_stream(self.h) or 0

    def synchronize(self):
        self._check(self._L.ptk_synchronize(self.h), self.h)

    def launches(self) -> int:
        return int(self._L.ptk_kernel_launches(self.h))


def abi_sizes() -> tuple[int, int, int]:
    a, b, c = C.c_size_t(), C.c_size_t(), C.c_size_t()
    lib().ptk_abi_sizes(C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


class _PinnedBuffer:
    """Page-locked host memory from ptk_host_alloc, freed with the last array
    that views it (numpy keeps this object as the array's base)."""

    def __init__(self, shape, dtype):
        dt = np.dtype(dtype)
        nbytes = max(int(np.prod(shape)) * dt.itemsize, 1)
        self.ptr = C.c_void_p()
        self._free = lib().ptk_host_free  # kept: module globals may be gone when the last array dies
        rc = lib().ptk_host_alloc(C.byref(self.ptr), nbytes)
        if rc != PTK_OK:
            raise PtkError(rc, "ptk_host_alloc")
        self.__array_interface__ = {"shape": tuple(shape), "typestr": dt.str, "data": (self.ptr.value, False),
                                    "version": 3}

    def __del__(self):
        if getattr(self, "ptr", None) and self.ptr.value:
            self._free(self.ptr)
            self.ptr = None


def pinned_copy(a: np.ndarray) -> np.ndarray:
    """A copy of `a` in page-locked host memory, so that Tracker.load_frame
    uploads it asynchronously (from pageable memory an upload is synchronous)."""
    a = np.ascontiguousarray(a)
    out = np.asarray(_PinnedBuffer(a.shape, a.dtype))
    out[...] = a
    return out


def tune_cache_lookup(path: str, signature: str):
    """(method, choice) stored for signature in the autotune cache at path,
    or None (ptk_tune_cache_lookup)."""
    found, method, choice = C.c_int32(), C.c_int32(), C.c_int32()
    rc = lib().ptk_tune_cache_lookup(str(path).encode(), signature.encode(), C.byref(found), C.byref(method),
                                     C.byref(choice))
    if rc != PTK_OK:
        raise PtkError(rc, f"cannot read the autotune cache {path}")
    return (method.value, choice.value) if found.value else None


def tune_cache_store(path: str, signature: str, method: int, choice: int, values=(), ms=()):
    """Writes one entry of the autotune cache at path (ptk_tune_cache_store)."""
    n = len(values)
    if len(ms) != n:
        raise ValueError("values and ms differ in length")
    v = (C.c_int32 * max(n, 1))(*[int(x) for x in values])
    t = (C.c_float * max(n, 1))(*[float(x) for x in ms])
    rc = lib().ptk_tune_cache_store(str(path).encode(), signature.encode(), int(method), int(choice), n, v, t)
    if rc != PTK_OK:
        raise PtkError(rc, f"cannot write the autotune cache {path}")


def read_grains_file(path: str, format13: bool = True) -> np.ndarray:
    L = lib()
    n = C.c_int()
    rc = L.ptk_read_grains_file(str(path).encode(), int(format13), None, 0, C.byref(n))
    if rc != PTK_OK:
        raise PtkError(rc, f"cannot read {path}")
    s = np.zeros(n.value, dtype=GRAIN_DTYPE)
    rc = L.ptk_read_grains_file(str(path).encode(), int(format13), _ptr(s), n.value, C.byref(n))
    if rc != PTK_OK:
        raise PtkError(rc, f"cannot parse {path}")
    return structs_to_records(s)


def save_grains_file(path: str, rec13: np.ndarray, from_image: str = "", to_image: str = "",
                     from_datetime: str = "dateTime unknown", to_datetime: str = "dateTime unknown"):
    s = records_to_structs(rec13)
    rc = lib().ptk_save_grains_file(str(path).encode(), _ptr(s), s.shape[0], from_image.encode(),
                                    from_datetime.encode(), to_image.encode(), to_datetime.encode())
    if rc != PTK_OK:
        raise PtkError(rc, f"cannot write {path}")


def read_image_file(path: str) -> tuple[np.ndarray, str]:
    """Grey levels of an image file as the tracking path reads it
    (ptk_read_image_file): a (rows, columns) uint16 array and the TIFF DateTime
    (or "dateTime unknown")."""
    L = lib()
    w, h = C.c_int(), C.c_int()
    rc = L.ptk_read_image_file(str(path).encode(), None, 0, C.byref(w), C.byref(h), None, 0)
    if rc != PTK_OK:
        raise PtkError(rc, L.ptk_image_error().decode())
    out = np.zeros((h.value, w.value), dtype=np.uint16)
    when = C.create_string_buffer(256)
    rc = L.ptk_read_image_file(str(path).encode(), _ptr(out), out.size, C.byref(w), C.byref(h), when, 256)
    if rc != PTK_OK:
        raise PtkError(rc, L.ptk_image_error().decode())
    return out, when.value.decode()


DISTO_POWELL, DISTO_POWELL_ITER, DISTO_LEVMAR = 0, 1, 2


def disto_pairs(refx: np.ndarray, refy: np.ndarray, dmin: float, dmax: float) -> np.ndarray:
    """precompute_paires (src/distortion_correction.cpp:63-81): (npairs, 2)
    int32 pairs i < j, i-major, of grains dmin .. dmax apart."""
    L = lib()
    rx = np.ascontiguousarray(refx, dtype=np.int32)
    ry = np.ascontiguousarray(refy, dtype=np.int32)
    n = C.c_int64()
    rc = L.ptk_disto_pairs(_ptr(rx), _ptr(ry), rx.shape[0], float(dmin), float(dmax), None, 0, C.byref(n))
    out = np.zeros((max(n.value, 1), 2), dtype=np.int32)
    rc = L.ptk_disto_pairs(_ptr(rx), _ptr(ry), rx.shape[0], float(dmin), float(dmax), _ptr(out), n.value,
                           C.byref(n))
    if rc != 0:
        raise PtkError(rc, "ptk_disto_pairs")
    return out[:n.value]


class DistoFit:
    """The distortion-parameter fit of correction_distortion on the GPU
    (ptk_disto_*): grains' integer reference positions, their tracked
    displacements and subpixel NCC per image after the reference
    ([image, grain]), and the grain pairs."""

    def __init__(self, dimx: int, dimy: int, refx, refy, dx, dy, ncc_subpix, NCC_min: float, pairs):
        L = lib()
        self._L = L
        self._keep = [np.ascontiguousarray(refx, dtype=np.int32), np.ascontiguousarray(refy, dtype=np.int32),
                      np.ascontiguousarray(dx, dtype=np.float64), np.ascontiguousarray(dy, dtype=np.float64),
                      np.ascontiguousarray(ncc_subpix, dtype=np.float64),
                      np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)]
        rx, ry, ddx, ddy, nc, pr = self._keep
        self.n, self.nimg1, self.npairs = rx.shape[0], ddx.shape[0], pr.shape[0]
        h = C.c_void_p()
        rc = L.ptk_disto_create(C.byref(h), dimx, dimy, _ptr(rx), _ptr(ry), self.n, self.nimg1, _ptr(ddx), _ptr(ddy),
                                _ptr(nc), float(NCC_min), _ptr(pr), self.npairs)
        if rc != 0:
            raise PtkError(rc, "ptk_disto_create")
        self.h = h

    def _check(self, rc: int):
        if rc != 0:
            raise PtkError(rc, self._L.ptk_disto_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self._L.ptk_disto_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def objective(self, params14) -> float:
        x = np.ascontiguousarray(params14, dtype=np.float64)
        v = C.c_double()
        self._check(self._L.ptk_disto_objective(self.h, _ptr(x), C.byref(v)))
        return v.value

    def residuals(self, params14) -> tuple[float, np.ndarray]:
        x = np.ascontiguousarray(params14, dtype=np.float64)
        v = C.c_double()
        f = np.zeros(self.nimg1 * self.npairs)
        self._check(self._L.ptk_disto_residuals(self.h, _ptr(x), C.byref(v), _ptr(f)))
        return v.value, f

    def fit(self, params14, perturb14, algo: int = DISTO_POWELL, num_iter: int = 5):
        x = np.array(params14, dtype=np.float64)
        dx = np.ascontiguousarray(perturb14, dtype=np.float64)
        ini, end = C.c_double(), C.c_double()
        hist = np.zeros((max(num_iter, 1), 15))
        self._check(self._L.ptk_disto_fit(self.h, _ptr(x), _ptr(dx), algo, num_iter, C.byref(ini), C.byref(end),
                                          _ptr(hist)))
        keep = num_iter if algo == DISTO_POWELL_ITER else (1 if algo == DISTO_LEVMAR else 0)
        return x, ini.value, end.value, hist[:keep]

    def levmar_info(self) -> tuple[int, int, str]:
        """Exit state of the last LEVMAR fit: lmdif's info code, residual
        evaluations, and the text for the code."""
        info, nfev, text = C.c_int(), C.c_int(), C.c_char_p()
        self._check(self._L.ptk_disto_levmar_info(self.h, C.byref(info), C.byref(nfev), C.byref(text)))
        return info.value, nfev.value, (text.value or b"").decode()

    def tracked(self) -> tuple[np.ndarray, np.ndarray]:
        dx = np.zeros((self.nimg1, self.n))
        dy = np.zeros((self.nimg1, self.n))
        self._check(self._L.ptk_disto_tracked(self.h, _ptr(dx), _ptr(dy)))
        return dx, dy

    def objective_timed(self, params14, reps: int) -> float:
        """Average device time (ms) of one objective evaluation's kernels."""
        x = np.ascontiguousarray(params14, dtype=np.float64)
        ms = C.c_double()
        self._check(self._L.ptk_disto_objective_timed(self.h, _ptr(x), int(reps), C.byref(ms)))
        return ms.value


def cli_path() -> Path:
    """The command-file driver (ptracker_b200), built next to libptk.so."""
    return Path(__file__).resolve().parent / "ptracker_b200"


__all__ = ["Tracker", "Config", "Zone", "Grain", "GRAIN_DTYPE", "COLUMNS", "lib", "synth", "PtkError",
           "read_grains_file", "save_grains_file", "read_image_file", "cli_path", "abi_sizes", "exported_symbols"]
