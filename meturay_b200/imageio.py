"""Headless image files: OpenEXR (uncompressed scanline) and PFM.

The stand-in for the reference's FreeImage/OpenEXR image writer
(ImageIO/ImageIO.cpp) where there is no display.  Arrays are (height,
width[, channels]) float32 with row 0 at the bottom of the image, as the
tracers produce them; EXR files store the top row first, so rows are
flipped on write and read.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from ._lib import check, lib

__all__ = ["write_exr", "write_pfm", "read_image"]


def _prep(pixels: np.ndarray):
    a = np.ascontiguousarray(pixels, np.float32)
    if a.ndim == 2:
        return a, a.shape[1], a.shape[0], 1
    if a.ndim != 3 or a.shape[2] not in (1, 3, 4):
        raise ValueError("pixels must be (h, w) or (h, w, 1|3|4)")
    return a, a.shape[1], a.shape[0], a.shape[2]


def write_exr(path, pixels: np.ndarray, half: bool = False):
    a, w, h, c = _prep(pixels)
    check(lib.mrb_write_exr(str(path).encode(), a.ctypes.data, w, h, c, 1 if half else 0))


def write_pfm(path, pixels: np.ndarray):
    a, w, h, c = _prep(pixels)
    check(lib.mrb_write_pfm(str(path).encode(), a.ctypes.data, w, h, c))


def read_image(path) -> np.ndarray:
    """(h, w, channels) float32 from a .exr or .pfm file."""
    p = str(Path(path)).encode()
    w, h, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
    check(lib.mrb_read_image(p, None, 0, C.byref(w), C.byref(h), C.byref(c)))
    out = np.zeros((h.value, w.value, c.value), np.float32)
    check(lib.mrb_read_image(p, out.ctypes.data, out.size, C.byref(w), C.byref(h), C.byref(c)))
    return out
