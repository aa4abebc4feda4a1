"""MRay scene files (TracerSystemI::GenerateScene's JSON) as Scene objects.

The parse runs in the native library (``mrb_json_scene_load``); this module
copies the resulting description into a :class:`meturay_b200.scenes.Scene`
so that it can go through ``GPUScene`` like any generated scene.  A scene
file carries no image size (MRay takes it from the visor configuration or
the command line), so ``width`` and ``height`` are arguments.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from ._lib import Camera, MrbError, SceneDesc, check, lib
from .scenes import LAMBERT, LAMBERTC, LIGHT, METAL, REFRACT, UNREAL, Scene

__all__ = ["load_scene", "load_scene_text", "load_tracer_config"]


def _copy(ptr, count: int, dtype, shape) -> np.ndarray:
    if count == 0:
        return np.zeros(shape, dtype)
    n = int(np.prod(shape))
    ctype = {np.float32: C.c_float, np.uint32: C.c_uint32, np.uint8: C.c_uint8}[dtype]
    buf = C.cast(ptr, C.POINTER(ctype * n)).contents
    return np.frombuffer(buf, dtype=dtype, count=n).reshape(shape).copy()


def _material_dict(m) -> dict:
    t = int(m.type)
    d = {"type": t}
    if t in (LAMBERT, LAMBERTC, REFRACT, UNREAL):
        d["albedo"] = np.array(m.albedo[:], np.float32)
    if t == METAL:
        d["eta"] = np.array(m.eta[:], np.float32)
        d["k"] = np.array(m.k[:], np.float32)
        d["specular"] = np.array(m.specular[:], np.float32)
        d["roughness"] = float(m.roughness)
    if t == UNREAL:
        d["roughness"] = float(m.roughness)
        d["metallic"] = float(m.metallic)
        d["specular_scalar"] = float(m.specular[0])
    if t == REFRACT:
        d["medium"] = int(m.medium)
    if t == LIGHT:
        d["radiance"] = np.array(m.radiance[:], np.float32)
    return d


def load_scene_text(text: str, width: int = 128, height: int = 128, camera: int = 0,
                    name: str = "json") -> Scene:
    """Parse an MRay scene (JSON text with // comments allowed)."""
    raw = text.encode()
    h = C.c_void_p()
    check(lib.mrb_json_scene_load(raw, len(raw), C.byref(h)))
    try:
        d = SceneDesc()
        ncam = C.c_uint32()
        check(lib.mrb_json_scene_get(h, C.byref(d), C.byref(ncam)))
        V, T = int(d.vertex_count), int(d.triangle_count)
        pos = _copy(d.positions, V, np.float32, (V, 3))
        nrm = _copy(d.normals, V, np.float32, (V, 3))
        uvs = _copy(d.uvs, V, np.float32, (V, 2))
        idx = _copy(d.indices, T, np.uint32, (T, 3))
        tri_mat = _copy(d.tri_material, T, np.uint32, (T,))
        cull = _copy(d.tri_cull, T, np.uint8, (T,))
        mats = [_material_dict(d.materials[i]) for i in range(int(d.material_count))]
        media = _copy(d.medium_ior, int(d.medium_count), np.float32, (int(d.medium_count),))
        if int(ncam.value) == 0:
            raise MrbError(-1, "scene JSON: no CameraSurfaces entry")
        cam = Camera()
        check(lib.mrb_json_scene_camera(h, int(camera), C.byref(cam)))
        cdict = {"position": list(cam.position), "gaze": list(cam.gaze), "up": list(cam.up),
                 "near_far": list(cam.near_far), "fov": list(cam.fov)}
        return Scene(name, pos, nrm, uvs, idx, tri_mat, mats, media, int(d.base_medium), cdict,
                     int(width), int(height), tri_cull=cull,
                     meta={"cameras": int(ncam.value), "camera": int(camera)})
    finally:
        lib.mrb_json_scene_destroy(h)


def load_scene(path, width: int = 128, height: int = 128, camera: int = 0) -> Scene:
    """Load an MRay scene file (``GenerateScene(path)``)."""
    p = Path(path)
    return load_scene_text(p.read_text(), width, height, camera, name=p.stem)


def _strip_comments(text: str) -> str:
    out, i, n, in_str = [], 0, len(text), False
    while i < n:
        c = text[i]
        if in_str:
            out.append(c)
            if c == "\\" and i + 1 < n:
                out.append(text[i + 1])
                i += 2
                continue
            if c == '"':
                in_str = False
            i += 1
        elif c == '"':
            in_str = True
            out.append(c)
            i += 1
        elif text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    return "".join(out)


def load_tracer_config(path_or_text) -> tuple[str, dict]:
    """Tracer type and options of an MRay tracer configuration (tConf_*.json):
    "TracerTypeName", "TracerOptions" and "TracerParameters"/"seed" (as
    "Seed").  Booleans become 0/1; keys the core does not know are kept so
    the caller can decide."""
    import json
    import re
    text = str(path_or_text)
    if not text.lstrip().startswith("{"):
        text = Path(path_or_text).read_text()
    text = _strip_comments(text)
    text = re.sub(r",(\s*[}\]])", r"\1", text)
    cfg = json.loads(text)
    opts = {}
    for k, v in cfg.get("TracerOptions", {}).items():
        opts[k] = int(v) if isinstance(v, bool) else v
    seed = cfg.get("TracerParameters", {}).get("seed")
    if seed is not None:
        opts["Seed"] = int(seed)
    return cfg.get("TracerTypeName", "PathTracer"), opts
