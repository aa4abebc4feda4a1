"""Choice of the 8-wide traversal kernel inside a tracer.

* The automatic choice times every kernel per depth on the tracer's own
  rays (the frame run before the graph capture), over the scene's layout
  and its alternate (the other collapse), and renders what a fixed kernel
  renders: relative mean error of the image below 1e-4 (the kernels and
  layouts differ only in which of two triangles at the same distance is
  reported).
* Every kernel renders the oracle's frame within the drop-in's 1e-4.
* A traversal setting changed after the capture is picked up by the next
  frame: the graph is captured again and the per-depth choice redone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-4
OPTS = {"Samples": 2, "MaxDepth": 5, "NextEventEstimation": 1, "RussianRouletteStart": 3,
        "DirectLightMIS": 0, "Seed": 3}
KERNELS = ("sorted", "octant", "sorted_refill", "octant_refill")
TUNED = KERNELS + tuple(k + "+alt" for k in KERNELS)   # "+alt": the alternate layout


def _rel(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-30))


@pytest.fixture(scope="module")
def cornell(system):
    from meturay_b200 import GPUScene, scenes
    scene = scenes.cornell(seed=1, width=96, height=64)
    g = GPUScene(system, scene)
    g.construct_accelerators()
    return scene, g


def _frames(system, g, frames=3):
    from meturay_b200 import PathTracer
    t = PathTracer(system, g)
    t.set_options(OPTS)
    for _ in range(frames):
        t.render_frame()
    img = t.image()
    orders = t.wide_orders()
    t.close()
    return img, orders


def test_auto_choice_renders_what_a_fixed_kernel_renders(system, cornell):
    scene, g = cornell
    g.set_traversal(1)
    g.set_wide_order("auto")
    auto, orders = _frames(system, g)
    assert len(orders) == OPTS["MaxDepth"] and all(o in TUNED for o in orders)
    assert all(v > 0 for v in g.wide_collapse()["probe_bytes"].values())  # both layouts built
    ms = g.wide_order()["ms"]
    assert all(v > 0 for v in ms.values())   # every kernel was timed
    for k in KERNELS:
        g.set_wide_order(k)
        img, orders = _frames(system, g)
        assert orders == [k] * OPTS["MaxDepth"]
        assert _rel(img[..., :3], auto[..., :3]) < REL_TOL, k
        assert np.array_equal(img[..., 3], auto[..., 3])
    g.set_wide_order("auto")


@pytest.mark.parametrize("kernel", KERNELS)
def test_every_kernel_matches_the_oracle(system, oracle, cornell, kernel):
    from meturay_b200 import PathTracer, camera_frame
    scene, g = cornell
    g.set_traversal(1)
    g.set_wide_order(kernel)
    t = PathTracer(system, g)
    t.set_options(OPTS)
    t.generate_work()
    while t.render():
        pass
    t.finalize()
    gpu = t.sample_radiance()[..., :3]
    t.close()
    g.set_wide_order("auto")
    os_ = oracle.OracleScene.from_scene(scene)
    cf = np.concatenate([camera_frame(scene.camera), np.float32(scene.camera["near_far"])])
    ref, _ = os_.render(cf, scene.width, scene.height, OPTS["Samples"], OPTS["MaxDepth"],
                        OPTS["RussianRouletteStart"], True, OPTS["Seed"])
    assert _rel(gpu, ref) < REL_TOL


def test_traversal_change_after_capture(system, cornell):
    from meturay_b200 import PathTracer
    scene, g = cornell
    g.set_traversal(1)
    g.set_wide_order("auto")
    t = PathTracer(system, g)
    t.set_options(OPTS)
    t.render_frame()
    assert all(o in TUNED for o in t.wide_orders())
    g.set_traversal(0)          # binary nodes from the next frame on
    t.render_frame()
    assert t.wide_orders() == [None] * OPTS["MaxDepth"]
    g.set_traversal(1)
    g.set_wide_order("octant")
    t.render_frame()
    assert t.wide_orders() == ["octant"] * OPTS["MaxDepth"]
    mixed = t.image()
    t.close()
    g.set_wide_order("auto")
    # the same three frames with one fixed kernel
    ref, _ = _frames(system, g)
    assert _rel(mixed[..., :3], ref[..., :3]) < REL_TOL
    assert np.array_equal(mixed[..., 3], ref[..., 3])
