"""Reconstruction filters and image memory (GPUReconFilterI, ImageMemory).

``ReconFilter`` mirrors GPUReconFilterI (GPUReconFilterI.h:6-33): a filter
type ("Box", "Tent", "Gaussian", "Mitchell"), a radius in pixels and the
type's options ("alpha"; "b", "c"), and ``filter_to_img`` splatting device
samples into an ``ImageMemory`` (ImageMemory.h:14-78).  Device buffers are
passed as torch CUDA tensors or raw device pointers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import MrbError, check, lib

__all__ = ["ReconFilter", "ImageMemory", "filter_pixel_wh"]


def filter_pixel_wh(radius: float) -> int:
    """FilterRadiusToPixelWH: side of the pixel window one sample reaches."""
    return int(lib.mrb_recon_filter_pixel_wh(float(radius)))


def _dev_ptr(x) -> int:
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise MrbError(-1, "recon filter: tensors must live on the GPU")
        if not x.is_contiguous():
            raise MrbError(-1, "recon filter: tensors must be contiguous")
        return int(x.data_ptr())
    raise MrbError(-1, f"recon filter: expected a CUDA tensor or a device pointer, got {type(x)}")


class ReconFilter:
    """GPUReconFilterI, built as TracerSystemI::GenerateReconFilter builds it
    from filter options {"type", "radius", ...}."""

    def __init__(self, filter_type: str, radius: float, options: dict | None = None):
        opts = {k: float(v) for k, v in (options or {}).items()}
        names = (C.c_char_p * max(1, len(opts)))(*[k.encode() for k in opts])
        vals = (C.c_float * max(1, len(opts)))(*opts.values())
        h = C.c_void_p()
        check(lib.mrb_recon_filter_create(filter_type.encode(), float(radius), len(opts), names,
                                          vals, C.byref(h)))
        self._h = h
        self.radius = float(radius)

    @classmethod
    def from_options(cls, options: dict) -> "ReconFilter":
        """TracerSystemCUDA::GenerateReconFilter (TracerSystemCUDA.cpp:109-137)."""
        if "type" not in options:
            raise MrbError(-1, 'Filter Options has to have "type" field')
        if "radius" not in options:
            raise MrbError(-1, 'Filter Options has to have "radius" field')
        rest = {k: v for k, v in options.items() if k not in ("type", "radius")}
        return cls(str(options["type"]), float(options["radius"]), rest)

    def close(self):
        if getattr(self, "_h", None):
            lib.mrb_recon_filter_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def type(self) -> str:
        return lib.mrb_recon_filter_type(self._h).decode()

    def used_gpu_memory(self) -> int:
        return int(lib.mrb_recon_filter_used_bytes(self._h))

    def weight(self, pixel_xy, sample_xy) -> float:
        """The filter functor on the host (pixel centre, sample position)."""
        return float(lib.mrb_recon_filter_weight(self._h, float(pixel_xy[0]), float(pixel_xy[1]),
                                                 float(sample_xy[0]), float(sample_xy[1])))

    def filter_to_img(self, image: "ImageMemory", values, img_coords, sample_count: int,
                      scalar_multiplier: float = 1.0, stream: int | None = None):
        """FilterToImg: values (n, channels) float32 and img_coords (n, 2)
        float32 on the device, added into the image's pixels and counts."""
        if hasattr(values, "dim"):
            channels = 1 if values.dim() == 1 else int(values.shape[-1])
        else:
            channels = image.channels
        check(lib.mrb_recon_filter_to_img(self._h, image._h, _dev_ptr(values), channels,
                                          _dev_ptr(img_coords), int(sample_count),
                                          float(scalar_multiplier), stream))


class ImageMemory:
    """ImageMemory: pixels (channels 1 = R_FLOAT or 4 = RGBA_FLOAT) and the
    per-pixel sample counts of one image portion."""

    def __init__(self, width: int, height: int, channels: int = 4):
        h = C.c_void_p()
        check(lib.mrb_image_create(int(width), int(height), int(channels), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.mrb_image_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        v = np.zeros(7, np.int32)
        check(lib.mrb_image_info(self._h, v.ctypes.data))
        return {"segment_offset": (int(v[0]), int(v[1])), "segment_size": (int(v[2]), int(v[3])),
                "resolution": (int(v[4]), int(v[5])), "channels": int(v[6])}

    @property
    def channels(self) -> int:
        return self.info()["channels"]

    def reportion(self, start, end):
        check(lib.mrb_image_reportion(self._h, int(start[0]), int(start[1]), int(end[0]),
                                      int(end[1])))

    def resize(self, width: int, height: int):
        check(lib.mrb_image_resize(self._h, int(width), int(height)))

    def reset(self, stream: int | None = None):
        check(lib.mrb_image_reset(self._h, stream))

    def device_pointers(self) -> tuple[int, int]:
        p, c = C.c_void_p(), C.c_void_p()
        check(lib.mrb_image_device(self._h, C.byref(p), C.byref(c)))
        return int(p.value or 0), int(c.value or 0)

    def write(self, path):
        """Pixels / sample counts as .exr (FLOAT) or .pfm."""
        check(lib.mrb_image_write(self._h, str(path).encode()))

    def get_image(self, stream: int | None = None) -> tuple[np.ndarray, np.ndarray]:
        """GetImageToCPU: (pixels (h, w[, 4]), counts (h, w)); resets the image."""
        i = self.info()
        w, h = i["segment_size"]
        ch = i["channels"]
        pixels = np.zeros((h, w, ch) if ch > 1 else (h, w), np.float32)
        counts = np.zeros((h, w), np.float32)
        check(lib.mrb_image_get(self._h, pixels.ctypes.data, counts.ctypes.data, stream))
        return pixels, counts
