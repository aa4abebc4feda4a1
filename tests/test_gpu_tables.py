"""The tables the loader builds on the device (HitKeys, material and light
tables, tangent-space rotations, scene extent) against the oracle's own
restatement of the reference's loader, which the parity tests use as their
input instead of reading anything back from the device."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _scenes():
    from meturay_b200 import scenes
    return [("cornell", lambda: scenes.cornell(seed=1)),
            ("cornell_mixed", lambda: scenes.cornell(seed=6, width=64, height=64, mixed=True)),
            ("clusters", lambda: scenes.clusters(seed=4, n_clusters=60, tris_per_cluster=400))]


@pytest.mark.parametrize("name,make", _scenes())
def test_device_tables_equal_the_oracle_tables(system, oracle, name, make):
    from meturay_b200 import GPUScene
    scene = make()
    g = GPUScene(system, scene)
    g.construct_accelerators()
    ex = g.export()
    ref = oracle.scene_tables(scene)
    ref["tbn"] = oracle.build_tbn(scene)
    for k in ("tri_key", "lambert", "metal", "refract", "refract_medium", "light_radiance",
              "light_prim", "lambertc", "unreal", "tbn"):
        a, b = np.asarray(ex[k]), np.asarray(ref[k])
        assert a.shape == b.shape, (k, a.shape, b.shape)
        assert np.array_equal(a.view(np.uint8), np.ascontiguousarray(b, a.dtype).view(np.uint8)), k
    assert np.array_equal(g.export_accel()["extent"][:6], oracle.scene_extent(scene))
