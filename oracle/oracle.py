"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference leg, always as the checker.  The C++
restatement it loads cites the MRay reference file:line for every step.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libmrayref.so"


def build(ref_root: str | None = None) -> None:
    """Compile the oracle; with ``ref_root`` (or the REF_ROOT environment
    variable) naming an MRay source tree, also the reference shim and the
    product-sampler harness (the latter needs nvcc)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    ref_root = ref_root or os.environ.get("REF_ROOT")
    if not ref_root:
        return
    root = Path(ref_root)
    if not (root / "Source" / "RayLib" / "Ray.hpp").exists():
        raise FileNotFoundError(f"REF_ROOT={root} is not an MRay source tree")
    subprocess.run(["make", "-s", "-C", str(HERE), "ref", "psamp", f"REF_ROOT={root}"], check=True)


class Scene(C.Structure):
    _fields_ = [("vertex_count", C.c_uint32), ("tri_count", C.c_uint32),
                ("pos", C.c_void_p), ("tbn", C.c_void_p), ("idx", C.c_void_p),
                ("tri_key", C.c_void_p), ("tri_cull", C.c_void_p),
                ("lambert_count", C.c_uint32), ("lambert_albedo", C.c_void_p),
                ("metal_count", C.c_uint32), ("metal_params", C.c_void_p),
                ("refract_count", C.c_uint32), ("refract_albedo", C.c_void_p),
                ("refract_medium", C.c_void_p),
                ("light_count", C.c_uint32), ("light_radiance", C.c_void_p),
                ("light_prim", C.c_void_p),
                ("medium_count", C.c_uint32), ("medium_ior", C.c_void_p),
                ("base_medium", C.c_uint32),
                ("lambertc_count", C.c_uint32), ("lambertc_albedo", C.c_void_p),
                ("unreal_count", C.c_uint32), ("unreal_params", C.c_void_p)]


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("bottom_left", C.c_float * 3),
                ("right", C.c_float * 3), ("up", C.c_float * 3), ("plane_size", C.c_float * 2),
                ("near_far", C.c_float * 2)]


class Options(C.Structure):
    _fields_ = [(k, C.c_uint32) for k in ("width", "height", "samples", "max_depth", "rr_start",
                                          "nee", "mis", "seed_lo", "seed_hi", "frame", "threads",
                                          "row_begin", "row_end", "row_step")]


def _load():
    if not LIB.exists():
        build()
    lib = C.CDLL(str(LIB))
    vp, u32 = C.c_void_p, C.c_uint32
    lib.oracle_morton3d.restype = C.c_uint64
    lib.oracle_morton3d.argtypes = [u32, u32, u32]
    lib.oracle_acosf.restype = C.c_float
    lib.oracle_acosf.argtypes = [C.c_float]
    lib.oracle_bvh_create.restype = vp
    lib.oracle_bvh_create.argtypes = [C.POINTER(Scene), C.POINTER(C.c_int)]
    lib.oracle_bvh_destroy.argtypes = [vp]
    lib.oracle_bvh_root.restype = u32
    lib.oracle_bvh_root.argtypes = [vp]
    lib.oracle_trace.argtypes = [C.POINTER(Scene), vp, vp, u32, vp, vp, vp, vp, u32]
    lib.oracle_trace_linear.argtypes = [C.POINTER(Scene), vp, u32, vp, vp, vp, vp, u32]
    lib.oracle_trace_counters.argtypes = [vp, C.c_int]
    lib.oracle_product_pin.argtypes = [vp, u32, u32, vp, vp, u32, C.c_float, C.c_float, vp, vp,
                                       vp, vp, vp]
    lib.oracle_render.restype = C.c_uint64
    lib.oracle_render.argtypes = [C.POINTER(Scene), vp, C.POINTER(Camera), C.POINTER(Options), vp]
    lib.oracle_render_f64.restype = C.c_uint64
    lib.oracle_render_f64.argtypes = [C.POINTER(Scene), vp, C.POINTER(Camera),
                                      C.POINTER(Options), vp]
    lib.oracle_partition.restype = u32
    return lib


lib = _load()


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def morton_codes(pos: np.ndarray, idx: np.ndarray):
    pos = np.ascontiguousarray(pos, np.float32)
    idx = np.ascontiguousarray(idx, np.uint32)
    n = idx.shape[0]
    aabbs = np.zeros((n, 6), np.float32)
    ext = np.zeros(6, np.float32)
    delta = np.zeros(1, np.float32)
    codes = np.zeros(n, np.uint64)
    lib.oracle_morton_codes(_p(pos), _p(idx), C.c_uint32(n), _p(aabbs), _p(ext), _p(delta),
                            _p(codes))
    return aabbs, ext, float(delta[0]), codes


def sort_pairs(keys: np.ndarray, vals: np.ndarray, begin: int, end: int, descending: bool):
    keys = np.ascontiguousarray(keys).copy()
    vals = np.ascontiguousarray(vals, np.uint32).copy()
    fn = lib.oracle_sort_pairs_u64 if keys.dtype == np.uint64 else lib.oracle_sort_pairs_u32
    fn(_p(keys), _p(vals), C.c_uint32(keys.shape[0]), C.c_int(begin), C.c_int(end),
       C.c_int(1 if descending else 0))
    return keys, vals


def lbvh(sorted_codes: np.ndarray, sorted_idx: np.ndarray, leaf_aabbs: np.ndarray):
    n = sorted_codes.shape[0]
    ni = max(n - 1, 0)
    out = {"left": np.zeros(ni, np.uint32), "right": np.zeros(ni, np.uint32),
           "parent": np.zeros(2 * n - 1, np.uint32), "inner": np.zeros((ni, 6), np.float32),
           "root": np.zeros(1, np.uint32)}
    st = lib.oracle_lbvh_build(_p(np.ascontiguousarray(sorted_codes, np.uint64)),
                               _p(np.ascontiguousarray(sorted_idx, np.uint32)),
                               _p(np.ascontiguousarray(leaf_aabbs, np.float32)), C.c_uint32(n),
                               _p(out["left"]), _p(out["right"]), _p(out["parent"]),
                               _p(out["inner"]), _p(out["root"]))
    out["status"] = st
    return out


def trace_counters(reset: bool = False) -> tuple[int, int]:
    """Inner LBVH nodes entered and triangles tested by the oracle's
    traversal (OracleScene.trace / render, all threads) since the last reset;
    reset=True zeroes them after reading."""
    out = np.zeros(2, np.uint64)
    lib.oracle_trace_counters(_p(out), 1 if reset else 0)
    return int(out[0]), int(out[1])


def product_pin(fields: np.ndarray, rays_per_bin: int, surfaces: np.ndarray,
                streams: np.ndarray, mis_ratio: float, mult: float) -> dict:
    """The oracle's product sampler on table inputs (fields (bins, 64, 64);
    surfaces (rays, 198); streams (rays, 32, n) uniforms per lane), as the
    reference sampler's harness runs it."""
    fields = np.ascontiguousarray(fields, np.float32)
    surfaces = np.ascontiguousarray(surfaces, np.float32)
    streams = np.ascontiguousarray(streams, np.float32)
    bins, rays = fields.shape[0], surfaces.shape[0]
    out = {"uv": np.zeros((rays, 2), np.float32), "pdf": np.zeros(rays, np.float32),
           "sel": np.zeros(rays, np.uint32), "small": np.zeros((bins, 64), np.float32),
           "norm": np.zeros((bins, 64), np.float32)}
    lib.oracle_product_pin(_p(fields), bins, rays_per_bin, _p(surfaces), _p(streams),
                           streams.shape[2], float(mis_ratio), float(mult), _p(out["uv"]),
                           _p(out["pdf"]), _p(out["sel"]), _p(out["small"]), _p(out["norm"]))
    return out


def partition(keys: np.ndarray, batch_bits: int, id_bits: int):
    keys = np.ascontiguousarray(keys, np.uint32)
    n = keys.shape[0]
    sk = np.zeros(n, np.uint32)
    si = np.zeros(n, np.uint32)
    pb = np.zeros(256, np.uint32)
    po = np.zeros(256, np.uint32)
    pc = np.zeros(256, np.uint32)
    k = lib.oracle_partition(_p(keys), C.c_uint32(n), C.c_uint32(batch_bits), C.c_uint32(id_bits),
                             _p(sk), _p(si), _p(pb), _p(po), _p(pc))
    return sk, si, [(int(pb[i]), int(po[i]), int(pc[i])) for i in range(k)]


class OracleScene:
    """The scene as the hot path consumes it, plus the oracle's own LBVH."""

    def __init__(self, scene, exported: dict):
        self.arrays = {
            "pos": np.ascontiguousarray(scene.positions, np.float32),
            "tbn": np.ascontiguousarray(exported["tbn"], np.float32),
            "idx": np.ascontiguousarray(scene.indices, np.uint32),
            "tri_key": np.ascontiguousarray(exported["tri_key"], np.uint32),
            "tri_cull": (np.ascontiguousarray(scene.tri_cull, np.uint8)
                         if scene.tri_cull is not None else None),
            "lambert": np.ascontiguousarray(exported["lambert"], np.float32),
            "metal": np.ascontiguousarray(exported["metal"], np.float32),
            "refract": np.ascontiguousarray(exported["refract"], np.float32),
            "refract_medium": np.ascontiguousarray(exported["refract_medium"], np.uint32),
            "light_radiance": np.ascontiguousarray(exported["light_radiance"], np.float32),
            "light_prim": np.ascontiguousarray(exported["light_prim"], np.uint32),
            "medium_ior": np.ascontiguousarray(scene.medium_ior, np.float32),
            "lambertc": np.ascontiguousarray(exported.get("lambertc", np.zeros((0, 3))),
                                             np.float32),
            "unreal": np.ascontiguousarray(exported.get("unreal", np.zeros((0, 6))), np.float32),
        }
        a = self.arrays
        s = Scene()
        s.vertex_count = a["pos"].shape[0]
        s.tri_count = a["idx"].shape[0]
        s.pos, s.tbn, s.idx, s.tri_key = _p(a["pos"]), _p(a["tbn"]), _p(a["idx"]), _p(a["tri_key"])
        s.tri_cull = _p(a["tri_cull"])
        s.lambert_count, s.lambert_albedo = a["lambert"].shape[0], _p(a["lambert"])
        s.metal_count, s.metal_params = a["metal"].shape[0], _p(a["metal"])
        s.refract_count, s.refract_albedo = a["refract"].shape[0], _p(a["refract"])
        s.refract_medium = _p(a["refract_medium"])
        s.light_count = a["light_prim"].shape[0]
        s.light_radiance, s.light_prim = _p(a["light_radiance"]), _p(a["light_prim"])
        s.medium_count, s.medium_ior = a["medium_ior"].shape[0], _p(a["medium_ior"])
        s.base_medium = scene.base_medium
        s.lambertc_count, s.lambertc_albedo = a["lambertc"].shape[0], _p(a["lambertc"])
        s.unreal_count, s.unreal_params = a["unreal"].shape[0], _p(a["unreal"])
        self.c = s
        st = C.c_int(0)
        self.bvh = lib.oracle_bvh_create(C.byref(s), C.byref(st))
        self.bvh_status = st.value

    @classmethod
    def from_scene(cls, scene) -> "OracleScene":
        """The scene with every table (HitKeys, material and light tables,
        tangent-space rotations) built by the oracle itself, so that nothing
        the checker uses comes from the device it checks."""
        ex = scene_tables(scene)
        ex["tbn"] = build_tbn(scene)
        return cls(scene, ex)

    def __del__(self):
        if getattr(self, "bvh", None):
            lib.oracle_bvh_destroy(self.bvh)
            self.bvh = None

    def trace(self, rays: np.ndarray, threads: int = 0, linear: bool = False):
        """rays: (n, 8) float32 = origin, tMin, direction, tMax."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        key = np.zeros(n, np.uint32)
        prim = np.zeros(n, np.uint32)
        t = np.zeros(n, np.float32)
        bary = np.zeros((n, 2), np.float32)
        if linear:
            lib.oracle_trace_linear(C.byref(self.c), _p(rays), n, _p(key), _p(prim), _p(t),
                                    _p(bary), threads)
        else:
            lib.oracle_trace(C.byref(self.c), self.bvh, _p(rays), n, _p(key), _p(prim), _p(t),
                             _p(bary), threads)
        return key, prim, t, bary

    def render(self, camera_frame: np.ndarray, width: int, height: int, samples: int,
               max_depth: int, rr_start: int, nee: bool, seed: int, frame: int = 0,
               threads: int = 0, rows: tuple[int, int] = (0, 0), fp64: bool = False,
               mis: bool = False, row_step: int = 1):
        """Per-sample radiance ((h*s), (w*s), 3) and the rays traced.  ``rows``
        (begin, end) and ``row_step`` select the sample rows rendered (every
        row_step-th row from begin); the others stay zero."""
        cam = Camera()
        f = camera_frame
        cam.position[:] = [float(v) for v in f[0:3]]
        cam.bottom_left[:] = [float(v) for v in f[3:6]]
        cam.right[:] = [float(v) for v in f[6:9]]
        cam.up[:] = [float(v) for v in f[9:12]]
        cam.plane_size[:] = [float(v) for v in f[12:14]]
        cam.near_far[:] = [float(v) for v in f[14:16]]
        o = Options(width, height, samples, max_depth, rr_start, 1 if nee else 0, 1 if mis else 0,
                    seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, frame, threads, rows[0], rows[1],
                    row_step)
        out = np.zeros((height * samples, width * samples, 3), np.float64 if fp64 else np.float32)
        fn = lib.oracle_render_f64 if fp64 else lib.oracle_render
        rays = fn(C.byref(self.c), self.bvh, C.byref(cam), C.byref(o), _p(out))
        return out, int(rays)

    def render_wfpg(self, camera_frame: np.ndarray, width: int, height: int, samples: int,
                    max_depth: int, rr_start: int, nee: bool, seed: int, svo: "OracleSvo",
                    frame: int = 0, mis: bool = False, min_bin_level: int = 5,
                    bin_ray_count: int = 512, pure_pg: bool = False, skip_pg: bool = False,
                    guide_bounce: int = 512, mis_ratio: float = 0.5, filter_alpha: float = 1.0,
                    dump_iteration: int | None = None, threads: int = 0, product: bool = True):
        """One WFPG frame; returns per-sample radiance, rays traced and the
        guide words / bin ids (per path) of step dump_iteration."""
        cam = Camera()
        f = camera_frame
        cam.position[:] = [float(v) for v in f[0:3]]
        cam.bottom_left[:] = [float(v) for v in f[3:6]]
        cam.right[:] = [float(v) for v in f[6:9]]
        cam.up[:] = [float(v) for v in f[9:12]]
        cam.plane_size[:] = [float(v) for v in f[12:14]]
        cam.near_far[:] = [float(v) for v in f[14:16]]
        o = Options(width, height, samples, max_depth, rr_start, 1 if nee else 0, 1 if mis else 0,
                    seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, frame, threads, 0, 0)
        w = WfpgOptions()
        w.min_bin_level = min_bin_level
        w.bin_ray_count = bin_ray_count
        w.pure_pg = 1 if pure_pg else 0
        w.skip_pg = 1 if skip_pg else 0
        w.guide_bounce = guide_bounce
        w.mis_ratio = float(mis_ratio)
        w.filter[:] = [float(v) for v in gauss_taps(filter_alpha)]
        w.product = 1 if product else 0
        w.dump_iteration = 0xFFFFFFFF if dump_iteration is None else int(dump_iteration)
        paths = width * samples * height * samples
        out = np.zeros((height * samples, width * samples, 3), np.float32)
        dg = np.zeros((paths, 2), np.uint32)
        dg[:, 1] = 0x7E00
        db = np.full(paths, 0xFFFFFFFF, np.uint32)
        lib.oracle_render_wfpg.restype = C.c_uint64
        rays = lib.oracle_render_wfpg(C.byref(self.c), self.bvh, C.byref(cam), C.byref(o),
                                      C.byref(w), svo.h, _p(out), _p(dg), _p(db))
        return out, int(rays), dg, db


def scene_tables(scene) -> dict:
    """HitKeys and material tables of a scene, assigned as the product's loader
    does: batch per material type (1 Lambert, 2 Metal, 3 Refract, 4 light),
    ids in material order, one primitive light per light triangle in triangle
    order (GPULightPrimitive: one GPULight per primitive)."""
    mats = scene.materials
    key = np.zeros(len(mats), np.uint32)
    lam, met, ref, refm, lamc, unr = [], [], [], [], [], []
    for i, m in enumerate(mats):
        t = int(m["type"])
        if t == 5:
            key[i] = (5 << 24) | len(lamc)
            lamc.append(np.asarray(m["albedo"], np.float32))
        elif t == 6:
            key[i] = (6 << 24) | len(unr)
            unr.append(np.array(list(m["albedo"]) + [m["roughness"], m.get("metallic", 0.0),
                                                     m.get("specular_scalar", 0.0)], np.float32))
        if t == 1:
            key[i] = (1 << 24) | len(lam)
            lam.append(np.asarray(m["albedo"], np.float32))
        elif t == 2:
            key[i] = (2 << 24) | len(met)
            met.append(np.concatenate([m["eta"], m["k"], m["specular"], [m["roughness"]]])
                       .astype(np.float32))
        elif t == 3:
            key[i] = (3 << 24) | len(ref)
            ref.append(np.asarray(m["albedo"], np.float32))
            refm.append(int(m["medium"]))
    tm = np.asarray(scene.tri_material, np.uint32)
    tri_key = key[tm].copy()
    light_tris = np.nonzero(np.array([int(mats[i]["type"]) == 4 for i in tm]))[0] \
        if len(tm) < 200000 else np.nonzero(np.isin(tm, [i for i, m in enumerate(mats)
                                                         if int(m["type"]) == 4]))[0]
    light_rad = np.array([mats[tm[t]]["radiance"] for t in light_tris], np.float32).reshape(-1, 3)
    tri_key[light_tris] = (4 << 24) | np.arange(len(light_tris), dtype=np.uint32)
    z3 = np.zeros((0, 3), np.float32)
    return {"tri_key": tri_key,
            "lambert": np.array(lam, np.float32).reshape(-1, 3) if lam else z3,
            "metal": np.array(met, np.float32).reshape(-1, 10) if met else np.zeros((0, 10),
                                                                                  np.float32),
            "refract": np.array(ref, np.float32).reshape(-1, 3) if ref else z3,
            "refract_medium": np.array(refm, np.uint32),
            "light_radiance": light_rad,
            "light_prim": light_tris.astype(np.uint32),
            "lambertc": np.array(lamc, np.float32).reshape(-1, 3) if lamc else z3,
            "unreal": np.array(unr, np.float32).reshape(-1, 6) if unr else np.zeros((0, 6),
                                                                                  np.float32)}


def build_tbn(scene) -> np.ndarray:
    pos = np.ascontiguousarray(scene.positions, np.float32)
    nrm = np.ascontiguousarray(scene.normals, np.float32)
    uvs = None if scene.uvs is None else np.ascontiguousarray(scene.uvs, np.float32)
    idx = np.ascontiguousarray(scene.indices, np.uint32)
    out = np.zeros((pos.shape[0], 4), np.float32)
    lib.oracle_build_tbn(_p(pos), _p(nrm), _p(uvs), _p(idx), C.c_uint32(pos.shape[0]),
                         C.c_uint32(idx.shape[0]), _p(out))
    return out


class WfpgOptions(C.Structure):
    _fields_ = [("min_bin_level", C.c_uint32), ("bin_ray_count", C.c_uint32),
                ("pure_pg", C.c_uint32), ("skip_pg", C.c_uint32), ("guide_bounce", C.c_uint32),
                ("mis_ratio", C.c_float), ("filter", C.c_float * 11),
                ("dump_iteration", C.c_uint32), ("product", C.c_uint32)]


def gauss_taps(alpha: float) -> np.ndarray:
    """StaticGaussianFilter1D<11> taps, exp(-t^2 / (2 alpha)) normalised,
    evaluated in double from the float option value and rounded once."""
    a = float(np.float32(alpha))
    w = [math.exp(-(float(i - 5) * float(i - 5)) * 0.5 / a) for i in range(11)]
    tot = 0.0
    for v in w:
        tot += v
    return np.array([v / tot for v in w], np.float32)


class OracleSvo:
    """The oracle's octree with its radiance-cache payload; a WFPG frame
    rendered by OracleScene.render_wfpg updates it."""

    def __init__(self, scene, tri_key: np.ndarray, extent: np.ndarray, resolution: int,
                 light_radiance: np.ndarray, omit_direct: bool = False):
        self._pos = np.ascontiguousarray(scene.positions, np.float32)
        self._idx = np.ascontiguousarray(scene.indices, np.uint32)
        self._key = np.ascontiguousarray(tri_key, np.uint32)
        ext = np.ascontiguousarray(extent[:6], np.float32)
        lib.oracle_svo_build.restype = C.c_void_p
        st = C.c_int(0)
        self.h = C.c_void_p(lib.oracle_svo_build(_p(self._pos), _p(self._idx), _p(self._key),
                                                 C.c_uint32(self._idx.shape[0]), _p(ext),
                                                 C.c_uint32(resolution), C.byref(st)))
        self.status = st.value
        self._rad = np.ascontiguousarray(np.asarray(light_radiance, np.float32).reshape(-1, 3))
        lights = self._key[(self._key >> 24) == 4] & 0xFFFFFF
        if lights.size and int(lights.max()) >= self._rad.shape[0]:
            raise ValueError(f"light radiance has {self._rad.shape[0]} entries; the triangle "
                             f"keys index light {int(lights.max())}")
        if self.status == 0:
            lib.oracle_svo_payload_init(self.h, _p(self._rad), C.c_uint32(1 if omit_direct else 0))

    def __del__(self):
        if getattr(self, "h", None):
            lib.oracle_svo_destroy(self.h)
            self.h = None

    def bin_rays(self, org: np.ndarray, dirs: np.ndarray, t: np.ndarray, valid: np.ndarray,
                 min_level: int, bin_ray_count: int) -> np.ndarray:
        """Bin ids of rays hitting at org + t * dirs (valid: rays the binning
        takes): 0xFFFFFFFF, leaf | 1 << 31 or the node index of the bin."""
        org = np.ascontiguousarray(org, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        valid = np.ascontiguousarray(valid, np.uint8)
        out = np.zeros(t.shape[0], np.uint32)
        lib.oracle_svo_bin_rays(self.h, _p(org), _p(dirs), _p(t), _p(valid),
                                C.c_uint32(t.shape[0]), C.c_uint32(min_level),
                                C.c_uint32(bin_ray_count), _p(out))
        return out

    def set_radiance(self, leaf_irr: np.ndarray, leaf_cnt: np.ndarray, normalize: bool = True):
        """Set the leaf radiance sums (2^-24 fixed point) and counts, then
        NormalizeAndFilterRadiance."""
        irr = np.ascontiguousarray(leaf_irr, np.uint64)
        cnt = np.ascontiguousarray(leaf_cnt, np.uint32)
        lib.oracle_svo_set_radiance(self.h, _p(irr), _p(cnt))
        if normalize:
            lib.oracle_svo_normalize(self.h)

    def set_shadow(self, leaf_shadow: np.ndarray, normalize: bool = True):
        """Set the per-leaf shadow-ray counters (hits, misses), then
        NormalizeAndFilterRadiance (which derives the node guiding factors)."""
        sh = np.ascontiguousarray(leaf_shadow, np.uint32)
        lib.oracle_svo_set_shadow(self.h, _p(sh))
        if normalize:
            lib.oracle_svo_normalize(self.h)

    def deposit_nee(self, pos: np.ndarray, is_hit: np.ndarray):
        """DepositNEEHitMiss of vertices over zeroed shadow-ray counters."""
        pos = np.ascontiguousarray(pos, np.float32)
        hit = np.ascontiguousarray(is_hit, np.uint8)
        lib.oracle_svo_deposit_nee(self.h, _p(pos), _p(hit), C.c_uint32(hit.shape[0]))

    def deposit(self, pos: np.ndarray, wo: np.ndarray, lum: np.ndarray):
        """DepositRadiance of path vertices over zeroed leaf sums."""
        pos = np.ascontiguousarray(pos, np.float32)
        wo = np.ascontiguousarray(wo, np.float32)
        lum = np.ascontiguousarray(lum, np.float32)
        lib.oracle_svo_deposit(self.h, _p(pos), _p(wo), _p(lum), C.c_uint32(lum.shape[0]))

    def cone_trace(self, org: np.ndarray, dirs: np.ndarray, tmin: np.ndarray,
                   aperture: np.ndarray, max_query_offset: int = 0) -> dict:
        """ConeTraceRay + ReadRadiance per cone: t, id, is_leaf, radiance."""
        org = np.ascontiguousarray(org, np.float32)
        dirs = np.ascontiguousarray(dirs, np.float32)
        tmin = np.ascontiguousarray(tmin, np.float32)
        aperture = np.ascontiguousarray(aperture, np.float32)
        n = tmin.shape[0]
        out = {"t": np.zeros(n, np.float32), "id": np.zeros(n, np.uint32),
               "leaf": np.zeros(n, np.uint8), "radiance": np.zeros(n, np.float32)}
        lib.oracle_svo_cone_trace(self.h, _p(org), _p(dirs), _p(tmin), _p(aperture),
                                  C.c_uint32(max_query_offset), C.c_uint32(n), _p(out["t"]),
                                  _p(out["id"]), _p(out["leaf"]), _p(out["radiance"]))
        return out

    def export(self) -> dict:
        sz = np.zeros(6, np.uint32)
        lib.oracle_svo_sizes(self.h, _p(sz))
        U, N = int(sz[1]), int(sz[2])
        out = {"status": self.status, "voxels": int(sz[0]), "depth": int(sz[3]),
               "nodes": np.zeros(N, np.uint64), "leaf_parents": np.zeros(U, np.uint32),
               "leaf_codes": np.zeros(U, np.uint64), "leaf_lights": np.zeros(U, np.uint32),
               "level_offsets": np.zeros(int(sz[4]), np.uint32),
               "tri_voxels": np.zeros(int(sz[5]), np.uint32), "params": np.zeros(7, np.float32),
               "leaf_normals": np.zeros(U, np.uint32), "node_normals": np.zeros(N, np.uint32),
               "leaf_irr": np.zeros((U, 2), np.uint64), "leaf_cnt": np.zeros((U, 2), np.uint32),
               "leaf_avg": np.zeros(U, np.uint32), "node_avg": np.zeros(N, np.uint32)}
        lib.oracle_svo_get(self.h, _p(out["nodes"]), _p(out["leaf_parents"]),
                           _p(out["leaf_codes"]), _p(out["leaf_lights"]), _p(out["level_offsets"]),
                           _p(out["tri_voxels"]), _p(out["params"]))
        if self.status == 0:
            lib.oracle_svo_payload_get(self.h, _p(out["leaf_normals"]), _p(out["node_normals"]),
                                       _p(out["leaf_irr"]), _p(out["leaf_cnt"]),
                                       _p(out["leaf_avg"]), _p(out["node_avg"]))
            out["leaf_shadow"] = np.zeros((U, 2), np.uint32)
            out["node_factor"] = np.zeros(N, np.uint16)
            lib.oracle_svo_guiding_get(self.h, _p(out["leaf_shadow"]), _p(out["node_factor"]))
        return out


def scene_extent(scene) -> np.ndarray:
    """Scene AABB (min xyz, max xyz) as the LBVH build reduces it: over the
    per-triangle boxes of KCGenerateAABBs."""
    aabbs, ext, _, _ = morton_codes(scene.positions, scene.indices)
    return ext


def voxelize(positions: np.ndarray, indices: np.ndarray, extent: np.ndarray, resolution: int):
    """TriFunctions::Voxelize over every triangle: (per-triangle voxel counts,
    Morton codes, packed spherical normals u16 | u16 << 16), triangle order."""
    pos = np.ascontiguousarray(positions, np.float32)
    idx = np.ascontiguousarray(indices, np.uint32)
    ext = np.ascontiguousarray(extent[:6], np.float32)
    T = idx.shape[0]
    counts = np.zeros(T, np.uint64)
    lib.oracle_voxelize.restype = C.c_int64
    n = lib.oracle_voxelize(_p(pos), _p(idx), C.c_uint32(T), _p(ext), C.c_uint32(resolution),
                            _p(counts), None, None, C.c_uint64(0))
    codes = np.zeros(n, np.uint64)
    normals = np.zeros(n, np.uint32)
    lib.oracle_voxelize(_p(pos), _p(idx), C.c_uint32(T), _p(ext), C.c_uint32(resolution),
                        _p(counts), _p(codes), _p(normals), C.c_uint64(n))
    return counts, codes, normals


def svo_build(scene, tri_key: np.ndarray, extent: np.ndarray, resolution: int) -> dict:
    """The oracle's sparse voxel octree of a scene (reference build order)."""
    pos = np.ascontiguousarray(scene.positions, np.float32)
    idx = np.ascontiguousarray(scene.indices, np.uint32)
    key = np.ascontiguousarray(tri_key, np.uint32)
    ext = np.ascontiguousarray(extent[:6], np.float32)
    lib.oracle_svo_build.restype = C.c_void_p
    st = C.c_int(0)
    h = lib.oracle_svo_build(_p(pos), _p(idx), _p(key), C.c_uint32(idx.shape[0]), _p(ext),
                             C.c_uint32(resolution), C.byref(st))
    sz = np.zeros(6, np.uint32)
    lib.oracle_svo_sizes(C.c_void_p(h), _p(sz))
    out = {"status": st.value, "voxels": int(sz[0]), "depth": int(sz[3]),
           "nodes": np.zeros(int(sz[2]), np.uint64), "leaf_parents": np.zeros(int(sz[1]), np.uint32),
           "leaf_codes": np.zeros(int(sz[1]), np.uint64), "leaf_lights": np.zeros(int(sz[1]), np.uint32),
           "level_offsets": np.zeros(int(sz[4]), np.uint32),
           "tri_voxels": np.zeros(int(sz[5]), np.uint32), "params": np.zeros(7, np.float32)}
    lib.oracle_svo_get(C.c_void_p(h), _p(out["nodes"]), _p(out["leaf_parents"]),
                       _p(out["leaf_codes"]), _p(out["leaf_lights"]), _p(out["level_offsets"]),
                       _p(out["tri_voxels"]), _p(out["params"]))
    lib.oracle_svo_destroy(C.c_void_p(h))
    return out


# ---- reconstruction filters (oracle/recon.cpp) ----------------------------
FILTER_TYPES = {"Box": 0, "Tent": 1, "Gaussian": 2, "Mitchell": 3}


class Filter(C.Structure):
    _fields_ = [("type", C.c_uint32), ("radius", C.c_float), ("alpha", C.c_float),
                ("b", C.c_float), ("c", C.c_float)]


def _filter(ftype: str, radius: float, alpha: float = 0.0, b: float = 0.0, c: float = 0.0):
    return Filter(FILTER_TYPES[ftype], radius, alpha, b, c)


lib.oracle_filter_pixel_wh.restype = C.c_uint32
lib.oracle_filter_pixel_wh.argtypes = [C.c_float]
lib.oracle_filter_weight.restype = C.c_float
lib.oracle_filter_weight.argtypes = [C.POINTER(Filter)] + [C.c_float] * 4
lib.oracle_filter_to_img.argtypes = [C.POINTER(Filter), C.c_void_p, C.c_uint32, C.c_void_p,
                                     C.c_uint32] + [C.c_int32] * 6 + [C.c_float, C.c_void_p,
                                                                      C.c_void_p]
lib.oracle_filter_direct.argtypes = [C.POINTER(Filter), C.c_void_p, C.c_void_p, C.c_uint32,
                                     C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
lib.oracle_mt19937_coords.argtypes = [C.c_uint32, C.c_int32, C.c_int32, C.c_uint32, C.c_void_p]
lib.oracle_camera_img_coords.argtypes = [C.POINTER(Options), C.c_void_p]
lib.oracle_exp.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]


def pexp(x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    lib.oracle_exp(_p(x), x.size, _p(out))
    return out


def filter_pixel_wh(radius: float) -> int:
    return int(lib.oracle_filter_pixel_wh(radius))


def filter_weight(ftype: str, radius: float, px, py, sx, sy, **params) -> float:
    f = _filter(ftype, radius, **params)
    return float(lib.oracle_filter_weight(C.byref(f), px, py, sx, sy))


def filter_to_img(ftype: str, radius: float, values: np.ndarray, coords: np.ndarray,
                  resolution, segment=None, multiplier: float = 1.0, pixels=None, counts=None,
                  **params):
    """FilterToImg on the CPU.  values: (n,) or (n, 4); coords: (n, 2).
    segment: (offX, offY, w, h), default the whole image.  Returns the
    image portion's (pixels, counts), added onto the given arrays if any."""
    f = _filter(ftype, radius, **params)
    values = np.ascontiguousarray(values, np.float32)
    coords = np.ascontiguousarray(coords, np.float32)
    ch = 1 if values.ndim == 1 else values.shape[1]
    W, H = resolution
    ox, oy, sw, sh = segment if segment is not None else (0, 0, W, H)
    if pixels is None:
        pixels = np.zeros((sh, sw, ch) if ch > 1 else (sh, sw), np.float32)
    if counts is None:
        counts = np.zeros((sh, sw), np.float32)
    lib.oracle_filter_to_img(C.byref(f), _p(values), ch, _p(coords), coords.shape[0], W, H, ox, oy,
                             sw, sh, multiplier, _p(pixels), _p(counts))
    return pixels, counts


def filter_direct(ftype: str, radius: float, values: np.ndarray, coords: np.ndarray, resolution,
                  **params):
    """The reference test's own direct CPU splat (RGBA, whole image)."""
    f = _filter(ftype, radius, **params)
    values = np.ascontiguousarray(values, np.float32)
    coords = np.ascontiguousarray(coords, np.float32)
    W, H = resolution
    pixels = np.zeros((H, W, 4), np.float32)
    counts = np.zeros((H, W), np.float32)
    lib.oracle_filter_direct(C.byref(f), _p(values), _p(coords), coords.shape[0], W, H,
                             _p(pixels), _p(counts))
    return pixels, counts


def mt19937_coords(n: int, width: int, height: int, seed: int = 0) -> np.ndarray:
    out = np.zeros((n, 2), np.float32)
    lib.oracle_mt19937_coords(n, width, height, seed, _p(out))
    return out


def camera_img_coords(width: int, height: int, samples: int, seed: int, frame: int) -> np.ndarray:
    o = Options()
    o.width, o.height, o.samples = width, height, samples
    o.seed_lo, o.seed_hi, o.frame = seed & 0xFFFFFFFF, seed >> 32, frame
    out = np.zeros((width * samples * height * samples, 2), np.float32)
    lib.oracle_camera_img_coords(C.byref(o), _p(out))
    return out


# ---- octree dump layout (DumpSVOAsBinary, AnisoSVO.cu:1555-1697) ----------
def _u64_to_f32_rne(v: int) -> np.float32:
    """uint64 -> float32 with one round-to-nearest-even step."""
    if v < (1 << 24):
        return np.float32(v)
    shift = v.bit_length() - 24
    m, rem = v >> shift, v & ((1 << shift) - 1)
    half = 1 << (shift - 1)
    if rem > half or (rem == half and (m & 1)):
        m += 1
    return np.float32(np.ldexp(np.float64(m), shift))


def svo_dump_bytes(ex: dict, node_bin16=None, leaf_bin16=None) -> bytes:
    """The dump of an exported octree (tracer.export_svo()), restated from
    the reference's layout: 48-byte header, tree arrays, then the payload
    with FP32 sums (2^-24 fixed point here), FP32 averages (half pairs here),
    the first N bytes of the binary16 node guiding factors (the reference
    copies N bytes of its half array) and zero leaf guiding factors."""
    N, U = ex["nodes_count"], ex["leaves"]
    lv = ex["level_offsets"].astype(np.uint32)
    nb = np.zeros(N, np.uint16) if node_bin16 is None else np.asarray(node_bin16, np.uint16)
    lb = np.zeros(U, np.uint16) if leaf_bin16 is None else np.asarray(leaf_bin16, np.uint16)

    def halves(words):
        w = np.asarray(words, np.uint32)
        pairs = np.stack([w & 0xFFFF, w >> 16], 1).astype(np.uint16)
        return pairs.view(np.float16).astype(np.float32)

    nf = ex.get("node_factor")
    factor_bytes = (np.zeros(N, np.uint8) if nf is None else
                    np.frombuffer(np.ascontiguousarray(nf, np.uint16).tobytes()[:N], np.uint8))
    irr = np.array([_u64_to_f32_rne(int(v)) for v in ex["leaf_irr"].ravel()],
                   np.float32) * np.float32(2.0 ** -24)
    parts = [np.asarray(ex["lo"], np.float32), np.asarray(ex["hi"], np.float32),
             np.array([ex["resolution"], ex["depth"], N, U], np.uint32),
             np.array([ex["leaf_size"]], np.float32), np.array([lv.size], np.uint32),
             ex["nodes"].astype(np.uint64), nb, ex["leaf_parents"].astype(np.uint32), lb, lv,
             halves(ex["node_avg"]), ex["node_normals"].astype(np.uint32), factor_bytes,
             irr.astype(np.float32), ex["leaf_cnt"].astype(np.uint32), halves(ex["leaf_avg"]),
             ex["leaf_normals"].astype(np.uint32), np.zeros(U, np.uint8)]
    return b"".join(np.ascontiguousarray(p).tobytes() for p in parts)


class OracleGroup:
    """The oracle's accelerator group: one LBVH per surface in local space
    under a local-to-world 3x4 matrix, closest hit over the surfaces."""

    def __init__(self, positions, indices, keys, surfaces, local_to_world, cull=None):
        self._pos = np.ascontiguousarray(positions, np.float32)
        self._idx = np.ascontiguousarray(indices, np.uint32)
        self._key = np.ascontiguousarray(keys, np.uint32)
        self._cull = None if cull is None else np.ascontiguousarray(cull, np.uint8)
        self._surf = np.ascontiguousarray(surfaces, np.uint32).reshape(-1, 3)
        self._l2w = np.ascontiguousarray(local_to_world, np.float32).reshape(-1, 12)
        lib.oracle_group_create.restype = C.c_void_p
        st = C.c_int(0)
        self.h = C.c_void_p(lib.oracle_group_create(
            _p(self._pos), C.c_uint32(self._pos.shape[0]), _p(self._idx), _p(self._key),
            _p(self._cull), C.c_uint32(self._idx.shape[0]), _p(self._surf),
            C.c_uint32(self._surf.shape[0]), _p(self._l2w), C.c_uint32(self._l2w.shape[0]),
            C.byref(st)))
        self.status = st.value

    def __del__(self):
        if getattr(self, "h", None):
            lib.oracle_group_destroy(self.h)
            self.h = None

    def trace(self, rays: np.ndarray) -> dict:
        """rays: (n, 8) origin, tMin, direction, tMax."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        out = {"key": np.zeros(n, np.uint32), "transform": np.zeros(n, np.uint32),
               "prim": np.zeros(n, np.uint64), "t": np.zeros(n, np.float32),
               "bary": np.zeros((n, 2), np.float32)}
        lib.oracle_group_trace(self.h, _p(rays), C.c_uint32(n), _p(out["key"]),
                               _p(out["transform"]), _p(out["prim"]), _p(out["t"]),
                               _p(out["bary"]))
        return out

    def aabbs(self) -> np.ndarray:
        out = np.zeros((self._surf.shape[0], 6), np.float32)
        lib.oracle_group_aabbs(self.h, _p(out))
        return out
