"""Sparse voxel octree build on the GPU against the oracle.

The oracle voxelises every triangle with the restated conservative
rasteriser and then builds the tree in the reference's own order (mark
children from the root, scan child counts, set child and parent pointers).
The device build derives the same canonical layout from prefix ranks.  Voxel
counts, the sorted unique leaf codes, level offsets, every packed node
(child index | parent | child mask | leaf bit), leaf parents and leaf light
keys must be bit-exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases():
    from meturay_b200 import scenes
    return [("cornell64", lambda: scenes.cornell(seed=1), 64),
            ("cornell256", lambda: scenes.cornell(seed=2), 256),
            ("clusters128", lambda: scenes.clusters(seed=3, n_clusters=30, tris_per_cluster=300), 128),
            ("random1024", lambda: scenes.random_triangles(seed=4, n=2000), 1024)]


@pytest.mark.parametrize("name,make,res", _cases())
def test_svo_bit_exact(system, oracle, name, make, res):
    from meturay_b200 import GPUScene
    scene = make()
    g = GPUScene(system, scene)
    g.construct_accelerators()
    g.build_svo(res)
    gpu = g.export_svo()
    ref = oracle.svo_build(scene, oracle.scene_tables(scene)["tri_key"],
                           oracle.scene_extent(scene), res)
    assert ref["status"] == 0
    assert gpu["voxels"] == ref["voxels"]
    assert np.array_equal(gpu["level_offsets"], ref["level_offsets"])
    assert np.array_equal(gpu["leaf_codes"], ref["leaf_codes"])
    assert np.array_equal(gpu["nodes"], ref["nodes"])
    assert np.array_equal(gpu["leaf_parents"], ref["leaf_parents"])
    assert np.array_equal(gpu["leaf_lights"], ref["leaf_lights"])
    assert np.allclose(gpu["lo"], ref["params"][0:3]) and np.allclose(gpu["hi"], ref["params"][3:6])
    # structural invariants
    d = gpu["depth"]
    assert gpu["level_offsets"][1] == 1 and gpu["level_offsets"][-1] - gpu["level_offsets"][-2] == \
        gpu["leaves"]
    mask = (gpu["nodes"] >> np.uint64(55)) & np.uint64(0xFF)
    assert (mask != 0).all()


def test_svo_leaf_normals_are_unit_directions(system):
    from meturay_b200 import GPUScene, scenes
    scene = scenes.cornell(seed=1)
    g = GPUScene(system, scene)
    g.construct_accelerators()
    g.build_svo(128)
    s = g.export_svo()
    # VoxelPayload normal word: x, y 9-bit UNORM, length 7 bits, z sign bit 31
    w = s["leaf_normals"].astype(np.int64)
    nx = (w & 511) * (2.0 / 511.0) - 1.0
    ny = ((w >> 9) & 511) * (2.0 / 511.0) - 1.0
    nz = np.sqrt(np.maximum(0.0, 1.0 - nx * nx - ny * ny)) * np.where((w >> 31) & 1, -1.0, 1.0)
    n = np.stack([nx, ny, nz], 1)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    assert np.all(((w >> 18) & 127) >= 126)  # leaf normals are unit means (length ~1)
    # floor voxels (lowest y layer, away from walls) carry the floor's
    # geometric normal, cross(p1 - p0, p2 - p0) as the reference voxeliser
    # takes it (GPUPrimitiveTriangle.h:434-435); the floor's winding gives -y
    p = scene.positions[scene.indices[0]].astype(np.float64)
    gn = np.cross(p[1] - p[0], p[2] - p[0])
    gn /= np.linalg.norm(gn)
    assert abs(abs(gn[1]) - 1.0) < 1e-12
    codes = s["leaf_codes"]
    def decode(c, shift):
        v = np.zeros_like(c)
        for b in range(21):
            v |= ((c >> np.uint64(3 * b + shift)) & np.uint64(1)) << np.uint64(b)
        return v
    y = decode(codes, 1)
    x = decode(codes, 0)
    z = decode(codes, 2)
    floor = (y == y.min()) & (x > 20) & (x < 100) & (z > 20) & (z < 100)
    assert floor.sum() > 100
    assert np.median(n[floor][:, 1] * gn[1]) > 0.99
