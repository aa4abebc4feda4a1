"""meturay_b200: a B200-native (sm_100a) wavefront path-tracing core that
drops in for MRay's (yalcinerbora/meturay) LBVH accelerator group, the plain
wavefront PathTracer and the path-guiding WFPGTracer with their
reconstruction filters and image memory, and reads MRay scene files.

The compute path is ``libmrb200.so`` (hand-written CUDA, C ABI in
``include/mrb200.h``); this package is the host-side mirror of the
reference's plugin interfaces over that ABI.
"""
from ._lib import MrbError, lib  # noqa: F401  (fails loudly if the library is missing)
from .tracer import GPUScene, PathTracer, TracerSystem, WFPGTracer, camera_frame  # noqa: F401
from . import scenes  # noqa: F401
from .scene_json import load_scene, load_scene_text, load_tracer_config  # noqa: F401
from .recon import ImageMemory, ReconFilter, filter_pixel_wh  # noqa: F401
from . import imageio  # noqa: F401
from .pool import Job, WavefrontPool  # noqa: F401

__all__ = ["TracerSystem", "GPUScene", "PathTracer", "WFPGTracer", "MrbError", "scenes",
           "camera_frame", "load_scene", "load_scene_text", "load_tracer_config",
           "ReconFilter", "ImageMemory", "filter_pixel_wh", "imageio",
           "WavefrontPool", "Job"]
