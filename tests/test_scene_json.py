"""MRay scene-file loader (mrb_json_scene_*): host-side checks.

tests/scenes/box_mixed.json is an MRay-format scene written for these
tests: comments, multi-id nodes, row- and column-major matrices, trs
transforms, indexed and plain in-node triangles, a transformed primitive
light, every material type and a second camera with a transform.
"""
import math
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
BOX = HERE / "scenes" / "box_mixed.json"


def _load(text_or_path=BOX, **kw):
    import meturay_b200 as m
    if isinstance(text_or_path, Path):
        return m.load_scene(text_or_path, **kw)
    return m.load_scene_text(text_or_path, **kw)


def _trs(t, r_deg, s):
    def rot(axis, a):
        a = math.radians(a)
        c, sn = math.cos(a), math.sin(a)
        R = np.eye(4)
        i, j = (axis + 1) % 3, (axis + 2) % 3
        R[i, i], R[i, j], R[j, i], R[j, j] = c, -sn, sn, c
        return R
    S, T = np.diag([s[0], s[1], s[2], 1.0]), np.eye(4)
    T[:3, 3] = t
    return T @ rot(2, r_deg[2]) @ rot(1, r_deg[1]) @ rot(0, r_deg[0]) @ S


QUAD = np.array([[-0.5, -0.5, 0], [0.5, -0.5, 0], [0.5, 0.5, 0], [-0.5, 0.5, 0]])


def test_box_structure():
    s = _load(width=64, height=48)
    # 5 walls + slab + light = 7 quads (14 tris), 2 tetrahedra (8 tris)
    assert s.triangle_count == 22
    assert (s.width, s.height) == (64, 48)
    # floor: row-major matrix
    M = np.array([[2, 0, 0, 0], [0, 0, 1, 0], [0, -2, 0, 0], [0, 0, 0, 1]], float)
    exp = (M @ np.c_[QUAD, np.ones(4)].T).T[:, :3]
    assert np.allclose(s.positions[:4], exp, atol=1e-6)
    assert np.allclose(s.normals[:4], [0, 1, 0], atol=1e-6)
    # walls of the box face inwards after the inverse-transpose of normals
    left = s.normals[8:12]
    assert np.allclose(left, [1, 0, 0], atol=1e-6)
    # cull flags: quads default to culling, the tetrahedra disable it
    assert s.tri_cull.tolist() == [1] * 10 + [0] * 4 + [1, 1] + [0] * 4 + [1, 1]


def test_materials_media_and_lights():
    from meturay_b200 import scenes as sc
    s = _load()
    types = [m["type"] for m in s.materials]
    # material order = first use: floor white, back Lambert, left red, right
    # green, tetrahedron Unreal(25), slab Refract, Metal, light
    assert types == [sc.LAMBERTC, sc.LAMBERT, sc.LAMBERTC, sc.LAMBERTC, sc.UNREAL, sc.REFRACT,
                     sc.METAL, sc.LIGHT]
    assert np.allclose(s.materials[0]["albedo"], [0.725, 0.71, 0.68])
    assert np.allclose(s.materials[2]["albedo"], [0.63, 0.065, 0.05])
    u = s.materials[4]
    assert np.allclose(u["albedo"], [0.9, 0.6, 0.2]) and u["roughness"] == pytest.approx(0.4)
    assert u["metallic"] == 1.0 and u["specular_scalar"] == 0.5
    assert s.materials[5]["medium"] == 1 and s.medium_ior[1] == pytest.approx(1.45)
    assert s.base_medium == 0 and s.medium_ior[0] == 1.0
    assert np.allclose(s.materials[7]["radiance"], [12, 10, 8])
    # the light quad: trs (rotate 90 about x) puts it just below the ceiling facing down
    light = np.nonzero(np.asarray(s.tri_material) == 7)[0]
    v = s.positions[s.indices[light].ravel()]
    exp = (_trs([0, 1.995, 0], [90, 0, 0], [0.5, 0.5, 1]) @ np.c_[QUAD, np.ones(4)].T).T[:, :3]
    assert np.allclose(np.unique(v.round(5), axis=0), np.unique(exp.round(5), axis=0), atol=1e-5)
    assert np.allclose(s.normals[s.indices[light].ravel()], [0, -1, 0], atol=1e-6)
    # column-major slab matrix: translation in the last four entries
    slab = np.nonzero(np.asarray(s.tri_material) == 5)[0]
    vs = s.positions[s.indices[slab].ravel()]
    assert np.allclose(vs.mean(axis=0), [-0.3, 0.55, 0.2], atol=1e-6)


def test_cameras():
    s0 = _load(camera=0)
    c = s0.camera
    assert np.allclose(c["position"], [0, 1, 4.2]) and np.allclose(c["near_far"], [0.01, 50])
    fx = math.radians(60.0)
    assert c["fov"][0] == pytest.approx(fx, rel=1e-6)
    assert c["fov"][1] == pytest.approx(2 * math.atan(math.tan(fx / 2) * 45.0 / 60.0), rel=1e-6)
    s1 = _load(camera=1)
    M = _trs([0.35, 0.2, 0.1], [0, 30, 0], [0.4, 0.4, 0.4])
    assert np.allclose(s1.camera["position"], M[:3, 3], atol=1e-6)
    assert np.allclose(s1.camera["gaze"], (M @ [0, 0, -1, 1])[:3], atol=1e-6)
    assert s0.meta["cameras"] == 2


@pytest.mark.parametrize("patch,needle", [
    (('"name": ".nodeTriangle",', '"name": "../Surfaces/mesh.obj",'), "file loader"),
    (('"type": "Lambert", "albedo": [0.5, 0.5, 0.5]',
      '"type": "Lambert", "albedo": {"texture": 0, "channel": "rgb"}'), "texture"),
    (('{ "id": 0, "type": "Null" }', '{ "id": 0, "type": "Point", "position": [0,1,0]}'),
     "boundary light"),
    (('"absorption": [0, 0, 0]', '"absorption": [0.1, 0, 0]'), "absorption"),
    (('"type": "Triangle",\n            "name": ".nodeTriangle",',
      '"type": "Sphere",\n            "name": ".nodeSphere",'), "primitive type"),
])
def test_unsupported_features_are_named(patch, needle):
    import meturay_b200 as m
    text = BOX.read_text()
    assert patch[0] in text
    with pytest.raises(m.MrbError) as e:
        _load(text.replace(patch[0], patch[1], 1))
    assert needle in str(e.value)


def test_malformed_json_reports_the_line():
    import meturay_b200 as m
    text = BOX.read_text().replace('"BaseMedium": 0,', '"BaseMedium": 0 "x",', 1)
    with pytest.raises(m.MrbError) as e:
        _load(text)
    assert "line" in str(e.value)
    with pytest.raises(m.MrbError):
        _load('{"Cameras": []}')


def test_tracer_config():
    import meturay_b200 as m
    cfg = """{
        // tracer configuration in MRay's format
        "TracerTypeName": "WFPGTracer",
        "TracerOptions": {
            "Samples": 1, "MaxDepth": 4, "NextEventEstimation": false,
            "OctreeLevel": 8, "BXDF-GuideMISRatio": 0.5, /* inline */ "DoProductPathGuiding": true,
        },
        "TracerParameters": {"seed": 3, "verbose": false}
    }"""
    t, o = m.load_tracer_config(cfg)
    assert t == "WFPGTracer"
    assert o == {"Samples": 1, "MaxDepth": 4, "NextEventEstimation": 0, "OctreeLevel": 8,
                 "BXDF-GuideMISRatio": 0.5, "DoProductPathGuiding": 1, "Seed": 3}
