"""Linear HDR image files: OpenEXR (read) and PFM (read).

`read_exr` decodes single-part scanline OpenEXR files without compression —
what the host's writer (host/exr.cpp) and `nori_render out.exr` produce —
with HALF, FLOAT or UINT channels, in pure numpy.  Other compressions
(ZIP, PIZ, ... as written by Mitsuba) are read through OpenCV when it is
installed, as the reference's comparison tool does
(validation_tests/compare_exr.py: cv2.imread with IMREAD_ANYDEPTH).
Images come back as float32 arrays of shape (H, W, 3), RGB, top row first.
"""

from __future__ import annotations

import os
import struct

import numpy as np

_MAGIC = 20000630
_PIXEL = {0: (np.uint32, 4), 1: (np.float16, 2), 2: (np.float32, 4)}


def _cstr(b: bytes, at: int) -> tuple[str, int]:
    end = b.index(b"\0", at)
    return b[at:end].decode("ascii"), end + 1


def _parse_header(b: bytes):
    magic, version = struct.unpack_from("<ii", b, 0)
    if magic != _MAGIC:
        raise ValueError("not an OpenEXR file")
    if version & 0x1200:  # tiled or multi-part
        raise ValueError("tiled or multi-part OpenEXR files are not supported")
    at, attrs = 8, {}
    while b[at] != 0:
        name, at = _cstr(b, at)
        typ, at = _cstr(b, at)
        (size,) = struct.unpack_from("<i", b, at)
        at += 4
        attrs[name] = (typ, b[at:at + size])
        at += size
    return attrs, at + 1


def _channels(raw: bytes):
    out, at = [], 0
    while raw[at] != 0:
        name, at = _cstr(raw, at)
        ptype, _, xs, ys = struct.unpack_from("<iiii", raw, at)
        at += 16
        if xs != 1 or ys != 1:
            raise ValueError("subsampled channels are not supported")
        out.append((name, ptype))
    return out


def read_exr(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        b = f.read()
    attrs, at = _parse_header(b)
    if attrs["compression"][1][0] != 0:
        return _read_with_opencv(path)
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    W, H = x1 - x0 + 1, y1 - y0 + 1
    chans = _channels(attrs["channels"][1])
    offsets = np.frombuffer(b, np.uint64, H, at)
    planes = {name: np.empty((H, W), np.float32) for name, _ in chans}
    for off in offsets:
        y, _size = struct.unpack_from("<ii", b, int(off))
        p = int(off) + 8
        for name, ptype in chans:  # channels in header (alphabetical) order
            dt, sz = _PIXEL[ptype]
            planes[name][y - y0] = np.frombuffer(b, dt, W, p).astype(np.float32)
            p += W * sz
    if not all(c in planes for c in "RGB"):
        raise ValueError(f"expected R, G, B channels, found {sorted(planes)}")
    return np.stack([planes["R"], planes["G"], planes["B"]], -1)


def _read_with_opencv(path: str) -> np.ndarray:
    os.environ.setdefault("OPENCV_IO_ENABLE_OPENEXR", "1")
    try:
        import cv2
    except ImportError as e:
        raise ValueError(f"{path}: compressed OpenEXR needs OpenCV") from e
    raw = cv2.imread(path, cv2.IMREAD_UNCHANGED | cv2.IMREAD_ANYDEPTH)
    if raw is None or raw.ndim != 3 or raw.shape[2] < 3:
        raise ValueError(f"{path}: OpenCV could not read a 3-channel image")
    return raw[..., :3][..., ::-1].astype(np.float32)


def read_pfm(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        kind = f.readline().strip()
        W, H = (int(v) for v in f.readline().split())
        scale = float(f.readline())
        data = np.frombuffer(f.read(), "<f4" if scale < 0 else ">f4")
    if kind != b"PF":
        raise ValueError("only colour PFM files are supported")
    return data.reshape(H, W, 3)[::-1].astype(np.float32)


def read_image(path: str) -> np.ndarray:
    return read_pfm(path) if path.lower().endswith(".pfm") else read_exr(path)
