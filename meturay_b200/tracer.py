"""Python mirror of the MRay plugin interfaces on the hot path.

``TracerSystem``   <- TracerSystemI (RayLib/TracerSystemI.h:34-50):
                      ``generate_scene``, ``generate_tracer``
``GPUScene``       <- GPUSceneI + the "LBVH" GPUAcceleratorGroupI
                      (GPUAcceleratorI.h:46-134): ``construct_accelerators``,
                      ``hit``
``PathTracer``     <- GPUTracerI "PathTracer" (RayLib/GPUTracerI.h:24-71,
                      PathTracer.cu:120-326): ``set_options``,
                      ``generate_work``, ``render``, ``finalize``

Every call goes through the C ABI of libmrb200.so; errors raise
``MrbError`` carrying the library's status and message, as the reference
returns ``TracerError`` values.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import Camera, Material, MrbError, SceneDesc, check, lib
from .scenes import Scene

# traversal kernels of the 8-wide layout (MRB_WIDE_SORTED ..
# MRB_WIDE_OCTANT_REFILL), and the automatic choice (MRB_WIDE_AUTO)
WIDE_ORDERS = ("sorted", "octant", "sorted_refill", "octant_refill")
WIDE_AUTO = 4

__all__ = ["TracerSystem", "GPUScene", "PathTracer", "WFPGTracer", "MrbError"]


def _ptr(a: np.ndarray | None):
    return None if a is None else C.c_void_p(a.ctypes.data)


def make_camera(cam: dict) -> Camera:
    c = Camera()
    c.position[:] = [float(v) for v in cam["position"]]
    c.gaze[:] = [float(v) for v in cam["gaze"]]
    c.up[:] = [float(v) for v in cam["up"]]
    c.near_far[:] = [float(v) for v in cam["near_far"]]
    c.fov[:] = [float(v) for v in cam["fov"]]
    return c


def camera_frame(cam: dict) -> np.ndarray:
    """The 14-float pinhole frame the device uses (GPUCameraPinhole.cuh:135-162)."""
    out = np.zeros(14, np.float32)
    c = make_camera(cam)
    check(lib.mrb_camera_frame(C.byref(c), _ptr(out)))
    return out


class TracerSystem:
    """TracerSystemI: owns the device context and generates scenes and tracers."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.mrb_system_create(int(device), C.byref(h)))
        self._h = h

    def close(self):
        if self._h:
            lib.mrb_system_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def generate_scene(self, scene: Scene) -> "GPUScene":
        return GPUScene(self, scene)

    def generate_recon_filter(self, filter_options: dict):
        """GenerateReconFilter (TracerSystemCUDA.cpp:109-137): {"type", "radius", ...}."""
        from .recon import ReconFilter
        return ReconFilter.from_options(filter_options)

    def generate_tracer(self, scene: "GPUScene", tracer_type: str = "PathTracer",
                        options: dict | None = None) -> "PathTracer":
        """GenerateTracer (TracerSystemI): "PathTracer" or "WFPGTracer"."""
        t = WFPGTracer(self, scene) if tracer_type == "WFPGTracer" else \
            PathTracer(self, scene, tracer_type)
        if options:
            t.set_options(options)
        return t


class GPUScene:
    """A scene on the device with its "LBVH" accelerator group."""

    def __init__(self, system: TracerSystem, scene: Scene):
        self.system = system
        self.scene = scene
        self._keep = []
        mats = (Material * max(1, len(scene.materials)))()
        for i, m in enumerate(scene.materials):
            mats[i].type = int(m["type"])
            for key in ("albedo", "eta", "k", "specular", "radiance"):
                if key in m:
                    getattr(mats[i], key)[:] = [float(v) for v in m[key]]
            mats[i].roughness = float(m.get("roughness", 0.0))
            mats[i].metallic = float(m.get("metallic", 0.0))
            if "specular_scalar" in m:
                mats[i].specular[0] = float(m["specular_scalar"])
            mats[i].medium = int(m.get("medium", 0))
        arrs = {
            "positions": np.ascontiguousarray(scene.positions, np.float32),
            "normals": np.ascontiguousarray(scene.normals, np.float32),
            "uvs": np.ascontiguousarray(scene.uvs, np.float32) if scene.uvs is not None else None,
            "indices": np.ascontiguousarray(scene.indices, np.uint32),
            "tri_material": np.ascontiguousarray(scene.tri_material, np.uint32),
            "tri_cull": (np.ascontiguousarray(scene.tri_cull, np.uint8)
                         if scene.tri_cull is not None else None),
            "medium_ior": np.ascontiguousarray(scene.medium_ior, np.float32),
        }
        d = SceneDesc()
        d.vertex_count = arrs["positions"].shape[0]
        d.triangle_count = arrs["indices"].shape[0]
        for k in ("positions", "normals", "uvs", "indices", "tri_material", "tri_cull",
                  "medium_ior"):
            setattr(d, k, _ptr(arrs[k]))
        d.material_count = len(scene.materials)
        d.materials = C.cast(mats, C.POINTER(Material))
        d.medium_count = arrs["medium_ior"].shape[0]
        d.base_medium = scene.base_medium
        h = C.c_void_p()
        check(lib.mrb_scene_create(system._h, C.byref(d), C.byref(h)))
        self._h = h
        self.counts = np.zeros(8, np.uint32)
        check(lib.mrb_scene_counts(self._h, _ptr(self.counts)))

    def close(self):
        if getattr(self, "_h", None):
            lib.mrb_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def triangle_count(self) -> int:
        return int(self.counts[0])

    @property
    def id_bits(self) -> int:
        return int(self.counts[7])

    def construct_accelerators(self, stream: int | None = None):
        """GPUAcceleratorGroupI::ConstructAccelerators for the LBVH group."""
        check(lib.mrb_accel_construct(self._h, stream))

    def set_traversal(self, mode: int):
        """1: 8-wide quantised nodes (default), 0: binary LBVH nodes."""
        check(lib.mrb_accel_set_traversal(self._h, int(mode)))

    def accel_info(self) -> dict:
        info = np.zeros(4, np.uint32)
        check(lib.mrb_accel_info(self._h, _ptr(info)))
        ext = np.zeros(2, np.uint32)
        areas = np.zeros(2, np.float64)
        check(lib.mrb_accel_info_ext(self._h, _ptr(ext), _ptr(areas)))
        return {"triangles": int(info[0]), "binary_nodes": int(info[1]),
                "wide_nodes": int(info[2]), "traversal": int(info[3]),
                "wide_tree": "ploc" if ext[0] == 1 else "lbvh", "ploc_steps": int(ext[1]),
                "inner_area_lbvh": float(areas[0]), "inner_area_ploc": float(areas[1])}

    def set_wide_order(self, order):
        """Traversal kernel of the 8-wide layout: "sorted", "octant",
        "sorted_refill", "octant_refill" (or 0-3), or "auto" (4, default):
        the fastest, timed on seeded probe rays at construction and then per
        depth on a tracer's own rays in the frame before it captures its
        graph."""
        if isinstance(order, str):
            order = WIDE_AUTO if order == "auto" else WIDE_ORDERS.index(order)
        check(lib.mrb_accel_set_wide_order(self._h, int(order)))

    def wide_order(self) -> dict:
        """The kernel in use where no tracer tuned its own, and the last
        measured ms per kernel."""
        o = C.c_int(0)
        ms = np.zeros(len(WIDE_ORDERS), np.float32)
        check(lib.mrb_accel_wide_order(self._h, C.byref(o), _ptr(ms)))
        return {"order": WIDE_ORDERS[o.value],
                "ms": {k: float(v) for k, v in zip(WIDE_ORDERS, ms)}}

    def set_wide_tree(self, tree: int):
        """Before construct_accelerators: the tree collapsed into the 8-wide
        layout: 0 the LBVH, 1 PLOC, 2 (default) the one with less box area."""
        check(lib.mrb_accel_set_wide_tree(self._h, int(tree)))

    def set_wide_collapse(self, collapse: int):
        """Before construct_accelerators: how each 8-wide node picks its
        children: 0 the largest-area internal child first, 1 the surface-area
        dynamic program, 2 (default) both, keeping the layout the seeded
        probe rays read fewer bytes of."""
        check(lib.mrb_accel_set_wide_collapse(self._h, int(collapse)))

    def wide_collapse(self) -> dict:
        """The collapse in use and, after an automatic choice, the probe
        bytes of each."""
        used = C.c_int32()
        b = np.zeros(2, np.float64)
        check(lib.mrb_accel_wide_collapse(self._h, C.byref(used), _ptr(b)))
        names = ("largest_area", "surface_area")
        return {"used": names[used.value], "probe_bytes": {k: float(v) for k, v in zip(names, b)}}

    def build_svo(self, resolution: int):
        """Sparse voxel octree of the scene at `resolution` leaf voxels per axis."""
        check(lib.mrb_svo_build(self._h, int(resolution), None))

    def export_svo(self) -> dict:
        """Octree structure and radiance-cache payload (host copies)."""
        info = np.zeros(6, np.uint32)
        params = np.zeros(7, np.float32)
        check(lib.mrb_svo_info(self._h, _ptr(info), _ptr(params)))
        out = _svo_arrays(info, params)
        check(lib.mrb_svo_export(self._h, *[_ptr(out[k]) for k in _SVO_KEYS]))
        check(lib.mrb_svo_export_payload(self._h, *[_ptr(out[k]) for k in _PAYLOAD_KEYS]))
        return out

    def export(self) -> dict:
        """Host copies of the device scene arrays, as the hot path consumes them."""
        c = self.counts
        out = {
            "tbn": np.zeros((int(c[1]), 4), np.float32),
            "tri_key": np.zeros(int(c[0]), np.uint32),
            "lambert": np.zeros((int(c[3]), 3), np.float32),
            "metal": np.zeros((int(c[4]), 10), np.float32),
            "refract": np.zeros((int(c[5]), 3), np.float32),
            "refract_medium": np.zeros(int(c[5]), np.uint32),
            "light_radiance": np.zeros((int(c[2]), 3), np.float32),
            "light_prim": np.zeros(int(c[2]), np.uint32),
        }
        check(lib.mrb_scene_export(self._h, *[_ptr(out[k]) for k in (
            "tbn", "tri_key", "lambert", "metal", "refract", "refract_medium",
            "light_radiance", "light_prim")]))
        n2 = np.zeros(2, np.uint32)
        check(lib.mrb_scene_export_ext(self._h, None, None, _ptr(n2)))
        out["lambertc"] = np.zeros((int(n2[0]), 3), np.float32)
        out["unreal"] = np.zeros((int(n2[1]), 6), np.float32)
        check(lib.mrb_scene_export_ext(self._h, _ptr(out["lambertc"]), _ptr(out["unreal"]), None))
        return out

    def export_accel(self) -> dict:
        n = self.triangle_count
        ni = max(n - 1, 0)
        out = {"codes": np.zeros(n, np.uint64), "sorted_idx": np.zeros(n, np.uint32),
               "left": np.zeros(ni, np.uint32), "right": np.zeros(ni, np.uint32),
               "parent": np.zeros(2 * n - 1, np.uint32), "inner": np.zeros((ni, 6), np.float32),
               "root": np.zeros(1, np.uint32), "tri_aabbs": np.zeros((n, 6), np.float32),
               "extent": np.zeros(7, np.float32)}
        check(lib.mrb_accel_export(self._h, *[_ptr(out[k]) for k in (
            "codes", "sorted_idx", "left", "right", "parent", "inner", "root", "tri_aabbs",
            "extent")]))
        return out

    def hit(self, ray_o_ptr: int, ray_d_ptr: int, n: int, key_ptr: int, prim_ptr: int,
            t_ptr: int, bary_ptr: int, stream: int | None = None):
        """GPUAcceleratorGroupI::Hit on device buffers (raw pointers)."""
        check(lib.mrb_accel_hit(self._h, ray_o_ptr, ray_d_ptr, int(n), key_ptr, prim_ptr,
                                t_ptr, bary_ptr, stream))


_SVO_KEYS = ("nodes", "leaf_parents", "leaf_codes", "leaf_normals", "leaf_lights",
             "level_offsets")
_PAYLOAD_KEYS = ("node_normals", "leaf_irr", "leaf_cnt", "leaf_avg", "node_avg")


def _svo_arrays(info, params) -> dict:
    U, N = int(info[1]), int(info[2])
    return {"voxels": int(info[0]), "leaves": U, "nodes_count": N, "depth": int(info[3]),
            "resolution": int(info[4]), "lo": params[0:3].copy(), "hi": params[3:6].copy(),
            "leaf_size": float(params[6]),
            "nodes": np.zeros(N, np.uint64), "leaf_parents": np.zeros(U, np.uint32),
            "leaf_codes": np.zeros(U, np.uint64), "leaf_normals": np.zeros(U, np.uint32),
            "leaf_lights": np.zeros(U, np.uint32),
            "level_offsets": np.zeros(int(info[5]), np.uint32),
            "node_normals": np.zeros(N, np.uint32), "leaf_irr": np.zeros((U, 2), np.uint64),
            "leaf_cnt": np.zeros((U, 2), np.uint32), "leaf_avg": np.zeros(U, np.uint32),
            "node_avg": np.zeros(N, np.uint32)}


class PathTracer:
    """GPUTracerI "PathTracer": wavefront path tracing with NEE and Russian roulette."""

    OPTION_KEYS = ("Samples", "MaxDepth", "NextEventEstimation", "RussianRouletteStart",
                   "DirectLightMIS", "Seed", "Frame")

    def __init__(self, system: TracerSystem, scene: GPUScene, tracer_type: str = "PathTracer"):
        self.system = system
        self.gscene = scene
        h = C.c_void_p()
        check(lib.mrb_tracer_create(system._h, scene._h, tracer_type.encode(), C.byref(h)))
        self._h = h
        self.samples = 1
        self.width = self.height = 0
        sc = scene.scene
        self.set_resolution(sc.width, sc.height)
        self.set_camera(sc.camera)

    def close(self):
        if getattr(self, "_h", None):
            lib.mrb_tracer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_options(self, opts: dict):
        for k, v in opts.items():
            if k not in self.OPTION_KEYS:
                raise MrbError(-1, f"unknown option '{k}'")
            if k == "Samples":
                self.samples = int(v)
            check(lib.mrb_tracer_set_option(self._h, k.encode(), int(v)))

    def set_resolution(self, w: int, h: int):
        check(lib.mrb_tracer_set_resolution(self._h, int(w), int(h)))
        self.width, self.height = int(w), int(h)

    def set_camera(self, cam: dict):
        c = make_camera(cam)
        check(lib.mrb_tracer_set_camera(self._h, C.byref(c)))

    def write_image(self, path):
        """The image's estimate (rgb / w) as .exr or .pfm."""
        check(lib.mrb_tracer_write_image(self._h, str(path).encode()))

    def attach_recon_filter(self, recon_filter):
        """AttachReconFilter: Finalize splats through the filter (None detaches).
        The image restarts; afterwards .w holds the weight sums."""
        check(lib.mrb_tracer_set_filter(self._h, recon_filter._h if recon_filter else None))
        self.recon_filter = recon_filter

    def generate_work(self, camera_index: int = 0):
        check(lib.mrb_tracer_generate_work(self._h, int(camera_index)))

    def render(self) -> bool:
        return check(lib.mrb_tracer_render(self._h)) == 1

    def finalize(self):
        check(lib.mrb_tracer_finalize(self._h))

    def render_frame(self):
        """GenerateWork + Render* + Finalize replayed from one CUDA graph."""
        check(lib.mrb_tracer_render_frame(self._h))

    def image(self) -> np.ndarray:
        out = np.zeros((self.height, self.width, 4), np.float32)
        check(lib.mrb_tracer_get_image(self._h, _ptr(out)))
        return out

    def image_into(self, host_ptr: int):
        check(lib.mrb_tracer_get_image(self._h, host_ptr))

    def image_into_async(self, host_ptr: int):
        """Snapshot the image and copy it into pinned host memory while later
        frames render; valid after wait_image()."""
        check(lib.mrb_tracer_get_image_async(self._h, host_ptr))

    def wait_image(self):
        check(lib.mrb_tracer_wait_image(self._h))

    def sample_radiance(self) -> np.ndarray:
        s = self.samples
        out = np.zeros((self.height * s, self.width * s, 4), np.float32)
        check(lib.mrb_tracer_get_samples(self._h, _ptr(out)))
        return out

    def reset_image(self):
        check(lib.mrb_tracer_reset_image(self._h))

    def stats(self) -> tuple[int, int]:
        r = C.c_uint64()
        f = C.c_uint32()
        check(lib.mrb_tracer_stats(self._h, C.byref(r), C.byref(f)))
        return int(r.value), int(f.value)

    def launches_per_frame(self) -> int:
        return check(lib.mrb_tracer_launches_per_frame(self._h))

    def wide_orders(self) -> list:
        """The 8-wide traversal kernel of each depth (names, with "+alt" where
        it runs over the scene's alternate layout; None with the binary
        traversal)."""
        buf = (C.c_int * 256)()
        n = lib.mrb_tracer_wide_orders(self._h, buf, 256)
        if n < 0:
            check(n)
        alt = 16  # MRB_WIDE_ALT_LAYOUT
        return [None if buf[i] < 0 else
                WIDE_ORDERS[buf[i] & ~alt] + ("+alt" if buf[i] & alt else "") for i in range(n)]

    def profile_frame(self) -> dict:
        """One stepwise frame with per-stage CUDA-event timings and work counts."""
        ms = np.zeros(5, np.float32)
        work = np.zeros(4, np.uint64)
        check(lib.mrb_tracer_profile_frame(self._h, _ptr(ms), _ptr(work)))
        return {"camera_ms": float(ms[0]), "trace_ms": float(ms[1]),
                "partition_ms": float(ms[2]), "shade_ms": float(ms[3]),
                "resolve_ms": float(ms[4]), "rays": int(work[0]),
                "node_visits": int(work[1]), "tri_tests": int(work[2]),
                "trace_launches": int(work[3])}

    STAGES = ("camera", "trace", "partition", "shade", "reconstruct", "guide_clear",
              "guide_bin", "guide_sort", "guide_kernel", "deposit", "normalize_filter",
              "learned_collect")

    def profile_stages(self) -> dict:
        """One stepwise frame timed stage by stage, the guided stages apart
        (milliseconds per stage, summed over depths) and its work counts."""
        ms = np.zeros(len(self.STAGES), np.float32)
        work = np.zeros(4, np.uint64)
        check(lib.mrb_tracer_profile_stages(self._h, _ptr(ms), len(self.STAGES), _ptr(work)))
        out = {f"{k}_ms": float(v) for k, v in zip(self.STAGES, ms)}
        out.update(rays=int(work[0]), node_visits=int(work[1]), tri_tests=int(work[2]))
        return out

    @property
    def stream(self) -> int:
        return lib.mrb_tracer_stream(self._h) or 0


class WFPGTracer(PathTracer):
    """GPUTracerI "WFPGTracer": the wavefront path tracer with product path
    guiding from the tracer's sparse voxel octree radiance cache."""

    OPTION_KEYS = PathTracer.OPTION_KEYS + (
        "OctreeLevel", "MinRayBinLevel", "BinRayCount", "DoProductPathGuiding", "PurePG",
        "SkipPG", "GuideBounceAmount", "OmitDirectRadiance", "PGDumpDataStruct",
        "PGDataStructDumpIntervalExp", "LearnedGuiding", "LearnedWarmupFrames",
        "LearnedTrainSteps", "LearnedSamples", "LearnedSeed", "LearnedProductTarget",
        "LearnedWarmupOctree")
    FLOAT_KEYS = ("BXDF-GuideMISRatio", "RFieldFilterAlpha", "LearnedRate", "LearnedWeightMax",
                  "LearnedEMA")
    STRING_KEYS = ("InitialSVO", "PGDataStructDumpName")

    def __init__(self, system: TracerSystem, scene: GPUScene):
        super().__init__(system, scene, "WFPGTracer")

    def set_options(self, opts: dict):
        ints = {k: v for k, v in opts.items()
                if k not in self.FLOAT_KEYS and k not in self.STRING_KEYS}
        super().set_options(ints)
        for k, v in opts.items():
            if k in self.FLOAT_KEYS:
                check(lib.mrb_tracer_set_option_float(self._h, k.encode(), float(v)))
            elif k in self.STRING_KEYS:
                check(lib.mrb_tracer_set_option_string(self._h, k.encode(), str(v).encode()))

    def learned_params(self) -> np.ndarray:
        """The learned guiding network's parameters (LearnedGuiding)."""
        p = np.zeros(int(lib.mrb_mlp_param_count()), np.float32)
        check(lib.mrb_tracer_learned_params(self._h, _ptr(p)))
        return p

    def learned_loss(self) -> float:
        """Weighted mean -log q of the last frame's training batches."""
        out = np.zeros(2, np.float32)
        check(lib.mrb_tracer_learned_loss(self._h, _ptr(out)))
        return float(out[0] / out[1]) if out[1] > 0 else float("nan")

    def dump_svo(self) -> bytes:
        """DumpSVOAsBinary: the octree and its radiance state as bytes."""
        n = C.c_size_t()
        check(lib.mrb_tracer_svo_dump(self._h, None, 0, C.byref(n)))
        buf = (C.c_uint8 * n.value)()
        check(lib.mrb_tracer_svo_dump(self._h, buf, n.value, C.byref(n)))
        return bytes(buf)

    def load_svo(self, data: bytes):
        """Constrcut(data): replace the octree with a dump."""
        check(lib.mrb_tracer_svo_load(self._h, data, len(data)))

    def export_svo(self) -> dict:
        """The tracer's octree with its current radiance state."""
        info = np.zeros(6, np.uint32)
        params = np.zeros(7, np.float32)
        check(lib.mrb_tracer_svo_info(self._h, _ptr(info), _ptr(params)))
        out = _svo_arrays(info, params)
        check(lib.mrb_tracer_svo_export(self._h, *[_ptr(out[k]) for k in _SVO_KEYS + _PAYLOAD_KEYS]))
        out["leaf_shadow"] = np.zeros((out["leaves"], 2), np.uint32)
        out["node_factor"] = np.zeros(out["nodes_count"], np.uint16)
        check(lib.mrb_tracer_svo_guiding(self._h, _ptr(out["leaf_shadow"]), _ptr(out["node_factor"])))
        return out

    def guide_state(self) -> dict:
        """Per-ray guide words of the wavefront the last Render() step shaded."""
        n = C.c_uint32()
        check(lib.mrb_tracer_guide_export(self._h, C.byref(n), None, None, None, None))
        k = int(n.value)
        out = {"samples": np.zeros(k, np.uint32), "guide": np.zeros((k, 2), np.uint32),
               "sorted_bin": np.zeros(k, np.uint32), "sorted_rid": np.zeros(k, np.uint32)}
        check(lib.mrb_tracer_guide_export(self._h, C.byref(n), _ptr(out["samples"]),
                                          _ptr(out["guide"]), _ptr(out["sorted_bin"]),
                                          _ptr(out["sorted_rid"])))
        return out
