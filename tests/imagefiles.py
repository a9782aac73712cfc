"""Writers of the image files the tracking path reads (test helpers):
uncompressed baseline TIFF and binary PGM, plus the grey levels the reference
computes from a TIFF through libtiff's RGBA reader (src/p-tracker.cpp:147-180),
restated in numpy with the same double operations."""
from __future__ import annotations

import struct
import zlib

import numpy as np


def write_tiff(path, data: np.ndarray, photometric: int | None = None, big_endian: bool = False,
               rows_per_strip: int | None = None, compression: int = 1, datetime: str | None = None,
               predictor: int | None = None, truncate: int = 0):
    """data: (h, w) grey or (h, w, spp) colour, uint8 or uint16, stored as
    given (compression 8 deflates each strip with zlib; other values only set
    the tag); predictor sets tag 317 (the caller stores differences)."""
    a = np.asarray(data)
    h, w = a.shape[:2]
    spp = 1 if a.ndim == 2 else a.shape[2]
    bps = 8 if a.dtype == np.uint8 else 16
    if photometric is None:
        photometric = 1 if spp == 1 else 2
    e = ">" if big_endian else "<"
    raw = a.astype(np.dtype(a.dtype).newbyteorder(e)).tobytes()
    rps = rows_per_strip or h
    row_bytes = w * spp * bps // 8
    strips = [raw[r * row_bytes:min(h, r + rps) * row_bytes] for r in range(0, h, rps)]
    if compression == 8:
        strips = [zlib.compress(s) for s in strips]
    if truncate:  # damaged files: every strip loses its last `truncate` bytes
        strips = [s[:-truncate] for s in strips]
    header = 8
    data_off = header
    offsets = []
    for s in strips:
        offsets.append(data_off)
        data_off += len(s)
    extra = b""
    extra_off = data_off

    def put_extra(b: bytes) -> int:
        nonlocal extra
        off = extra_off + len(extra)
        extra += b + (b"\0" if len(b) % 2 else b"")
        return off

    entries = []

    def add(tag, typ, values):
        n = len(values)
        fmt = {3: "H", 4: "I", 2: "B"}[typ]
        size = {3: 2, 4: 4, 2: 1}[typ] * n
        payload = struct.pack(e + fmt * n, *values)
        if size <= 4:
            entries.append((tag, typ, n, payload.ljust(4, b"\0")))
        else:
            entries.append((tag, typ, n, struct.pack(e + "I", put_extra(payload))))

    add(256, 4, [w])
    add(257, 4, [h])
    add(258, 3, [bps] * spp)
    add(259, 3, [compression])
    add(262, 3, [photometric])
    add(273, 4, offsets)
    add(277, 3, [spp])
    add(278, 4, [rps])
    add(279, 4, [len(s) for s in strips])
    add(284, 3, [1])
    if predictor is not None:
        add(317, 3, [predictor])
    if datetime is not None:
        add(306, 2, list(datetime.encode() + b"\0"))
    entries.sort()
    ifd_off = extra_off + len(extra)
    ifd = struct.pack(e + "H", len(entries))
    for tag, typ, n, payload in entries:
        ifd += struct.pack(e + "HHI", tag, typ, n) + payload
    ifd += struct.pack(e + "I", 0)
    with open(path, "wb") as f:
        f.write((b"MM" if big_endian else b"II") + struct.pack(e + "HI", 42, ifd_off))
        for s in strips:
            f.write(s)
        f.write(extra)
        f.write(ifd)


def write_pgm(path, data: np.ndarray):
    a = np.asarray(data)
    h, w = a.shape
    maxval = 255 if a.dtype == np.uint8 else 65535
    with open(path, "wb") as f:
        f.write(f"P5\n# test frame\n{w} {h}\n{maxval}\n".encode())
        f.write(a.astype(">u2" if maxval > 255 else np.uint8).tobytes())


def reference_grey(r8: np.ndarray, g8: np.ndarray, b8: np.ndarray) -> np.ndarray:
    """(uint16)(65535 (0.299 r + 0.587 g + 0.114 b)) with r = R * (1 / 255),
    evaluated left to right in double as the reference does."""
    fact = 1.0 / 255.0
    r = r8.astype(np.float64) * fact
    g = g8.astype(np.float64) * fact
    b = b8.astype(np.float64) * fact
    return (65535.0 * (0.299 * r + 0.587 * g + 0.114 * b)).astype(np.uint16)
