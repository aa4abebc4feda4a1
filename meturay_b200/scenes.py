"""Seeded synthetic scenes standing in for the benchmark inputs.

* ``cornell(seed)``: the small plain-tracer scene -- a Cornell-style box of
  five 2-triangle walls, a 1x1 primitive-backed quad light (radiance
  17,12,4) just below the ceiling and eight 32x16 UV spheres of radius
  U[0.1,0.25] at uniform positions inside the box (about 7.7k triangles),
  all Lambert with albedo U[0.2,0.8]; pinhole camera at (0.5,0.5,-1)
  looking +z with a 40 degree field of view.
* ``clusters(seed)``: the 1M-triangle scene -- 1000 Gaussian clusters
  (sigma U[0.5,3]) of 1000 triangles each in a 100^3 box, edge lengths
  LogNormal(-3, 0.5) with uniform directions; per cluster 40% Lambert
  (albedo U[0.2,0.8]), 40% GGX conductor (roughness U[0.05,0.8], F0
  U[0.5,1] mapped to a real index of refraction with k = 0), 20% dielectric
  in an IOR 1.5 medium; four 40x40 quad emitters on the walls.

Both use numpy's PCG64 generator seeded with ``seed``; the same seed gives
the same arrays on every machine.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

LAMBERT, METAL, REFRACT, LIGHT, LAMBERTC, UNREAL = 1, 2, 3, 4, 5, 6


@dataclass
class Scene:
    name: str
    positions: np.ndarray      # (V, 3) float32
    normals: np.ndarray        # (V, 3) float32
    uvs: np.ndarray            # (V, 2) float32
    indices: np.ndarray        # (T, 3) uint32
    tri_material: np.ndarray   # (T,) uint32
    materials: list            # dicts with "type" and parameters
    medium_ior: np.ndarray     # (M,) float32
    base_medium: int
    camera: dict               # position, gaze, up, near_far, fov (radians)
    width: int
    height: int
    tri_cull: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    @property
    def triangle_count(self) -> int:
        return int(self.indices.shape[0])


def _quad(p0, p1, p2, p3, normal):
    pos = np.array([p0, p1, p2, p3], np.float32)
    nrm = np.repeat(np.array([normal], np.float32), 4, axis=0)
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    idx = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    return pos, nrm, uv, idx


def uv_sphere(center, radius, segments=32, rings=16):
    """UV sphere with smooth normals; pole rings emit one triangle per quad."""
    th = np.linspace(0.0, math.pi, rings + 1)
    ph = np.linspace(0.0, 2.0 * math.pi, segments + 1)
    tt, pp = np.meshgrid(th, ph, indexing="ij")
    n = np.stack([np.sin(tt) * np.cos(pp), np.cos(tt), np.sin(tt) * np.sin(pp)], -1).reshape(-1, 3)
    uv = np.stack([pp / (2 * math.pi), tt / math.pi], -1).reshape(-1, 2)
    pos = np.asarray(center, np.float64) + radius * n
    # per quad (ring r, segment s), in r-major then s order: (a, d, b) unless
    # r is the top ring, then (d, c, b) unless r is the bottom ring
    w = segments + 1
    rr, ss = np.meshgrid(np.arange(rings), np.arange(segments), indexing="ij")
    a, b = rr * w + ss, (rr + 1) * w + ss
    c, d = (rr + 1) * w + ss + 1, rr * w + ss + 1
    t1 = np.stack([a, d, b], -1)
    t2 = np.stack([d, c, b], -1)
    both = np.stack([t1, t2], 2)                     # rings x segments x 2 x 3
    keep = np.stack([rr != 0, rr != rings - 1], -1)  # rings x segments x 2
    tris = both[keep]
    return (pos.astype(np.float32), n.astype(np.float32), uv.astype(np.float32),
            tris.astype(np.uint32))


class _Builder:
    def __init__(self):
        self.pos, self.nrm, self.uv, self.idx, self.mat = [], [], [], [], []
        self.nv = 0

    def add(self, pos, nrm, uv, idx, material):
        self.pos.append(pos)
        self.nrm.append(nrm)
        self.uv.append(uv)
        self.idx.append(idx + self.nv)
        self.mat.append(np.full(len(idx), material, np.uint32))
        self.nv += len(pos)

    def arrays(self):
        return (np.concatenate(self.pos).astype(np.float32),
                np.concatenate(self.nrm).astype(np.float32),
                np.concatenate(self.uv).astype(np.float32),
                np.concatenate(self.idx).astype(np.uint32),
                np.concatenate(self.mat).astype(np.uint32))


def cornell(seed: int = 1, width: int = 128, height: int = 128, mixed: bool = False,
            triangles: int | None = None, shielded: bool = False) -> Scene:
    """mixed=True gives the spheres, in turn, Lambert, LambertC, Metal (GGX
    conductor), Unreal and Refract materials (a test input for every BxDF).
    triangles: scale the spheres' tessellation (segments = 2 x rings) so the
    scene has about that many triangles (default 32 x 16 per sphere).
    shielded=True replaces the ceiling-wide light by a 0.2 x 0.2 light 0.1
    below the ceiling's centre, facing it, over an opaque 0.3 x 0.3 panel:
    the room sees the light only by way of the lit ceiling, the
    indirect-lighting case path guiding is for."""
    rng = np.random.default_rng(seed)
    segments, rings = 32, 16
    if triangles is not None:
        # a sphere of S segments and S/2 rings has S^2 - 2S triangles
        per = max(8.0, (triangles - 12) / 8.0)
        segments = max(4, 2 * int(round((1.0 + math.sqrt(1.0 + per)) / 2.0)))
        rings = segments // 2
    b = _Builder()
    mats = []

    def lambert():
        mats.append({"type": LAMBERT, "albedo": rng.uniform(0.2, 0.8, 3).astype(np.float32)})
        return len(mats) - 1

    walls = [
        ((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1), (0, 1, 0)),    # floor
        ((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0), (0, -1, 0)),   # ceiling
        ((0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1), (0, 0, -1)),   # back
        ((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0), (1, 0, 0)),    # left
        ((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1), (-1, 0, 0)),   # right
    ]
    for p0, p1, p2, p3, n in walls:
        # counter-clockwise seen from inside: the winding agrees with n
        b.add(*_quad(p0, p3, p2, p1, n), lambert())
    mats.append({"type": LIGHT, "radiance": np.array([17, 12, 4], np.float32)})
    light = len(mats) - 1
    y = 0.999
    if not shielded:
        b.add(*_quad((0, y, 0), (1, y, 0), (1, y, 1), (0, y, 1), (0, -1, 0)), light)
    else:
        # the light faces the ceiling from 0.1 below it; an opaque panel
        # just under the light hides it from the room
        ly, lo, hi = 0.9, 0.4, 0.6
        b.add(*_quad((lo, ly, lo), (lo, ly, hi), (hi, ly, hi), (hi, ly, lo), (0, 1, 0)), light)
        py, plo, phi = 0.895, 0.35, 0.65
        # one quad: triangles are two-sided, the panel shades from both
        b.add(*_quad((plo, py, plo), (phi, py, plo), (phi, py, phi), (plo, py, phi), (0, -1, 0)),
              lambert())
    kinds = [LAMBERT, LAMBERTC, METAL, UNREAL, REFRACT]
    for k in range(8):
        r = float(rng.uniform(0.1, 0.25))
        c = rng.uniform(r, 1.0 - r, 3)
        if not mixed or kinds[k % 5] == LAMBERT:
            b.add(*uv_sphere(c, r, segments, rings), lambert())
            continue
        kind = kinds[k % 5]
        if kind == LAMBERTC:
            mats.append({"type": LAMBERTC, "albedo": rng.uniform(0.2, 0.8, 3).astype(np.float32)})
        elif kind == METAL:
            f0 = rng.uniform(0.5, 0.95, 3)
            mats.append({"type": METAL, "eta": ((1 + np.sqrt(f0)) / (1 - np.sqrt(f0))).astype(
                np.float32), "k": np.zeros(3, np.float32), "specular": np.ones(3, np.float32),
                "roughness": float(rng.uniform(0.1, 0.6))})
        elif kind == UNREAL:
            mats.append({"type": UNREAL, "albedo": rng.uniform(0.2, 0.8, 3).astype(np.float32),
                         "roughness": float(rng.uniform(0.2, 0.8)),
                         "metallic": float(rng.uniform(0.0, 1.0)), "specular_scalar": 0.5})
        else:
            mats.append({"type": REFRACT, "albedo": np.ones(3, np.float32), "medium": 1})
        b.add(*uv_sphere(c, r, segments, rings), len(mats) - 1)
    pos, nrm, uv, idx, mat = b.arrays()
    fov = math.radians(40.0)
    cam = {"position": [0.5, 0.5, -1.0], "gaze": [0.5, 0.5, 0.5], "up": [0.0, 1.0, 0.0],
           "near_far": [0.1, 100.0], "fov": [fov, fov]}
    return Scene("cornell", pos, nrm, uv, idx, mat, mats, np.array([1.0, 1.5], np.float32), 0,
                 cam, width, height, meta={"seed": seed, "mixed": mixed, "shielded": shielded,
                                           "sphere_tessellation": (segments, rings)})


def clusters(seed: int = 1, width: int = 1920, height: int = 1080, n_clusters: int = 1000,
             tris_per_cluster: int = 1000) -> Scene:
    rng = np.random.default_rng(seed)
    n = n_clusters * tris_per_cluster
    centers = rng.uniform(0.0, 100.0, (n_clusters, 3))
    sigma = rng.uniform(0.5, 3.0, n_clusters)
    cid = np.repeat(np.arange(n_clusters), tris_per_cluster)
    v0 = centers[cid] + rng.normal(size=(n, 3)) * sigma[cid, None]

    def rand_dir(k):
        d = rng.normal(size=(k, 3))
        return d / np.linalg.norm(d, axis=1, keepdims=True)

    e1 = rand_dir(n) * rng.lognormal(-3.0, 0.5, (n, 1))
    e2 = rand_dir(n) * rng.lognormal(-3.0, 0.5, (n, 1))
    pos = np.stack([v0, v0 + e1, v0 + e2], 1).astype(np.float32)          # (n, 3, 3)
    fn = np.cross(pos[:, 1] - pos[:, 0], pos[:, 2] - pos[:, 0]).astype(np.float64)
    ln = np.linalg.norm(fn, axis=1, keepdims=True)
    fn = np.where(ln > 0, fn / np.maximum(ln, 1e-30), np.array([0.0, 0.0, 1.0]))
    nrm = np.repeat(fn[:, None, :], 3, axis=1).astype(np.float32)
    uv = np.tile(np.array([[0, 0], [1, 0], [0, 1]], np.float32), (n, 1, 1))
    # per-cluster materials: 40% Lambert, 40% GGX conductor, 20% dielectric
    kind = rng.choice([LAMBERT, METAL, REFRACT], size=n_clusters, p=[0.4, 0.4, 0.2])
    mats = []
    for k in kind:
        if k == LAMBERT:
            mats.append({"type": LAMBERT, "albedo": rng.uniform(0.2, 0.8, 3).astype(np.float32)})
        elif k == METAL:
            f0 = np.minimum(rng.uniform(0.5, 1.0, 3), 0.99)
            sq = np.sqrt(f0)
            eta = ((1.0 + sq) / (1.0 - sq)).astype(np.float32)
            mats.append({"type": METAL, "eta": eta, "k": np.zeros(3, np.float32),
                         "specular": np.ones(3, np.float32),
                         "roughness": float(rng.uniform(0.05, 0.8)), "f0": f0.astype(np.float32)})
        else:
            mats.append({"type": REFRACT, "albedo": np.ones(3, np.float32), "medium": 1})
    tri_mat = cid.astype(np.uint32)
    positions = pos.reshape(-1, 3)
    normals = nrm.reshape(-1, 3)
    uvs = uv.reshape(-1, 2)
    indices = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    # four 40x40 quad emitters on the walls, facing inwards
    mats.append({"type": LIGHT, "radiance": np.array([6, 6, 6], np.float32)})
    light = len(mats) - 1
    L = [((0, 30, 30), (0, 70, 30), (0, 70, 70), (0, 30, 70), (1, 0, 0)),
         ((100, 30, 30), (100, 30, 70), (100, 70, 70), (100, 70, 30), (-1, 0, 0)),
         ((30, 100, 30), (70, 100, 30), (70, 100, 70), (30, 100, 70), (0, -1, 0)),
         ((30, 30, 100), (30, 70, 100), (70, 70, 100), (70, 30, 100), (0, 0, -1))]
    b = _Builder()
    b.add(positions, normals, uvs, indices, 0)
    b.mat[0] = tri_mat
    for q in L:
        b.add(*_quad(*q), light)
    positions, normals, uvs, indices, tri_mat = b.arrays()
    fx = math.radians(65.0)
    fy = 2.0 * math.atan(math.tan(fx / 2.0) * height / width)
    cam = {"position": [50.0, 50.0, -60.0], "gaze": [50.0, 50.0, 50.0], "up": [0.0, 1.0, 0.0],
           "near_far": [0.1, 1000.0], "fov": [fx, fy]}
    return Scene("clusters", positions, normals, uvs, indices, tri_mat, mats,
                 np.array([1.0, 1.5], np.float32), 0, cam, width, height,
                 meta={"seed": seed, "clusters": n_clusters, "tris_per_cluster": tris_per_cluster})


def random_triangles(seed: int, n: int, extent: float = 10.0, size: float = 0.3) -> Scene:
    """Uniform random triangles in a cube, one Lambert material; test input."""
    rng = np.random.default_rng(seed)
    v0 = rng.uniform(0.0, extent, (n, 3))
    pos = np.stack([v0, v0 + rng.normal(size=(n, 3)) * size, v0 + rng.normal(size=(n, 3)) * size],
                   1).astype(np.float32)
    fn = np.cross(pos[:, 1] - pos[:, 0], pos[:, 2] - pos[:, 0]).astype(np.float64)
    fn /= np.maximum(np.linalg.norm(fn, axis=1, keepdims=True), 1e-30)
    nrm = np.repeat(fn[:, None, :], 3, axis=1).astype(np.float32)
    uv = np.tile(np.array([[0, 0], [1, 0], [0, 1]], np.float32), (n, 1, 1))
    mats = [{"type": LAMBERT, "albedo": np.array([0.5, 0.5, 0.5], np.float32)}]
    cam = {"position": [extent / 2, extent / 2, -extent], "gaze": [extent / 2] * 3,
           "up": [0.0, 1.0, 0.0], "near_far": [0.01, 1000.0], "fov": [1.0, 1.0]}
    return Scene("random", pos.reshape(-1, 3), nrm.reshape(-1, 3), uv.reshape(-1, 2),
                 np.arange(3 * n, dtype=np.uint32).reshape(n, 3), np.zeros(n, np.uint32), mats,
                 np.array([1.0], np.float32), 0, cam, 64, 64, meta={"seed": seed})
