"""End-to-end parity of the wavefront path tracer against the CPU oracle.

The oracle restates PathTracerKC.cuh (NEE, Russian roulette, Lambert /
Metal / Refract BxDFs, primitive lights) with the same counter-based RNG and
the same FP32 operation order.  Tolerance (the drop-in's bar): relative mean
error of the per-pixel radiance below 1e-4; in practice the images agree to
float atomic-addition order.  The FP64 oracle's error is reported, not bounded.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_MEAN_TOL = 1e-4


def _rel_mean_err(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-30))


def _setup(system, scene, opts):
    from meturay_b200 import GPUScene, PathTracer
    g = GPUScene(system, scene)
    g.construct_accelerators()
    t = PathTracer(system, g)
    t.set_options(opts)
    return g, t


def _oracle_render(oracle, g, scene, opts, frame=0, fp64=False):
    from meturay_b200 import camera_frame
    os_ = oracle.OracleScene.from_scene(scene)
    cf = np.concatenate([camera_frame(scene.camera), np.float32(scene.camera["near_far"])])
    img, rays = os_.render(cf, scene.width, scene.height, opts["Samples"], opts["MaxDepth"],
                           opts["RussianRouletteStart"], bool(opts["NextEventEstimation"]),
                           opts["Seed"], frame=frame, fp64=fp64)
    return img, rays


CORNELL_OPTS = {"Samples": 2, "MaxDepth": 5, "NextEventEstimation": 1,
                "RussianRouletteStart": 3, "DirectLightMIS": 0, "Seed": 1}


def test_cornell_stepwise_matches_oracle(system, oracle):
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=1)
    g, t = _setup(system, scene, CORNELL_OPTS)
    t.generate_work()
    steps = 0
    while t.render():
        steps += 1
    t.finalize()
    assert steps == CORNELL_OPTS["MaxDepth"] - 1
    gpu = t.sample_radiance()[..., :3]
    ref, ref_rays = _oracle_render(oracle, g, scene, CORNELL_OPTS)
    rays, frames = t.stats()
    assert rays == ref_rays
    err = _rel_mean_err(gpu, ref)
    assert err < REL_MEAN_TOL, err
    exact = np.mean(np.all(gpu == ref, axis=-1))
    assert exact > 0.99, exact
    assert gpu.sum() > 0


def test_cornell_graph_frames_match_stepwise(system, oracle):
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=3, width=64, height=48)
    g, t = _setup(system, scene, dict(CORNELL_OPTS, Seed=7))
    for _ in range(3):
        t.render_frame()
    img = t.image()
    assert img[..., 3].min() == 3.0
    # frames 0, 1, 2 through the oracle, pixel means averaged per frame
    s = CORNELL_OPTS["Samples"]
    acc = np.zeros((scene.height, scene.width, 3), np.float64)
    for f in range(3):
        ref, _ = _oracle_render(oracle, g, scene, dict(CORNELL_OPTS, Seed=7), frame=f)
        acc += ref.reshape(scene.height, s, scene.width, s, 3).mean(axis=(1, 3))
    err = _rel_mean_err(img[..., :3].astype(np.float64), acc)
    assert err < REL_MEAN_TOL, err


def test_clusters_all_materials_match_oracle(system, oracle):
    from meturay_b200 import scenes
    scene = scenes.clusters(seed=4, width=96, height=64, n_clusters=60, tris_per_cluster=400)
    opts = {"Samples": 1, "MaxDepth": 8, "NextEventEstimation": 1, "RussianRouletteStart": 3,
            "DirectLightMIS": 0, "Seed": 5}
    g, t = _setup(system, scene, opts)
    t.generate_work()
    while t.render():
        pass
    t.finalize()
    gpu = t.sample_radiance()[..., :3]
    ref, ref_rays = _oracle_render(oracle, g, scene, opts)
    rays, _ = t.stats()
    assert rays == ref_rays
    assert gpu.sum() > 0
    assert _rel_mean_err(gpu, ref) < REL_MEAN_TOL


def test_cornell_fp64_error_is_stated(system, oracle):
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=1, width=32, height=32)
    g, t = _setup(system, scene, CORNELL_OPTS)
    t.render_frame()
    gpu = t.image()[..., :3].astype(np.float64)
    ref64, _ = _oracle_render(oracle, g, scene, CORNELL_OPTS, fp64=True)
    s = CORNELL_OPTS["Samples"]
    ref64 = ref64.reshape(scene.height, s, scene.width, s, 3).mean(axis=(1, 3))
    err = _rel_mean_err(gpu, ref64)
    print(f"FP32 image vs FP64 oracle: relative mean error {err:.3e}")
    assert np.isfinite(err)


@pytest.mark.parametrize("mis", [0, 1])
def test_every_bxdf_with_and_without_mis(system, oracle, mis):
    """Lambert, LambertC, Metal, Unreal and Refract spheres; NEE with and
    without direct-light MIS (PathTracerKC.cuh:358-380,520-540)."""
    from meturay_b200 import camera_frame, scenes
    scene = scenes.cornell(seed=6, width=64, height=64, mixed=True)
    opts = dict(CORNELL_OPTS, DirectLightMIS=mis, Seed=3)
    g, t = _setup(system, scene, opts)
    t.generate_work()
    while t.render():
        pass
    t.finalize()
    gpu = t.sample_radiance()[..., :3]
    os_ = oracle.OracleScene.from_scene(scene)
    cf = np.concatenate([camera_frame(scene.camera), np.float32(scene.camera["near_far"])])
    ref, ref_rays = os_.render(cf, scene.width, scene.height, opts["Samples"], opts["MaxDepth"],
                               opts["RussianRouletteStart"], True, opts["Seed"], mis=bool(mis))
    rays, _ = t.stats()
    assert rays == ref_rays
    assert gpu.sum() > 0
    assert _rel_mean_err(gpu, ref) < REL_MEAN_TOL


def test_scene_file_renders_like_the_oracle(system, oracle):
    """An MRay scene file (tests/scenes/box_mixed.json) through the loader,
    the LBVH and the path tracer with MIS, against the oracle on the same
    description."""
    from pathlib import Path
    import meturay_b200 as m
    scene = m.load_scene(Path(__file__).resolve().parent / "scenes" / "box_mixed.json", 48, 36)
    opts = dict(CORNELL_OPTS, DirectLightMIS=1, Seed=5)
    g, t = _setup(system, scene, opts)
    t.generate_work()
    while t.render():
        pass
    t.finalize()
    gpu = t.sample_radiance()[..., :3]
    os_ = oracle.OracleScene.from_scene(scene)
    cf = np.concatenate([m.camera_frame(scene.camera), np.float32(scene.camera["near_far"])])
    ref, ref_rays = os_.render(cf, scene.width, scene.height, opts["Samples"], opts["MaxDepth"],
                               opts["RussianRouletteStart"], True, opts["Seed"], mis=True)
    rays, _ = t.stats()
    assert rays == ref_rays
    assert gpu.sum() > 0
    assert _rel_mean_err(gpu, ref) < REL_MEAN_TOL


def test_recapture_keeps_the_accumulated_image(system):
    """Changing an option re-captures the frame graph; the eager frame that
    precedes the capture is rewound, and the image and ray counters keep the
    frames rendered before it."""
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=1, width=32, height=32)
    opts = dict(CORNELL_OPTS, Seed=3)
    _, t = _setup(system, scene, opts)
    _, u = _setup(system, scene, opts)
    for _ in range(3):
        t.render_frame()
        u.render_frame()
    t.set_options({"Seed": 3})          # same value: only the graph is rebuilt
    t.render_frame()
    u.render_frame()
    a, b = t.image(), u.image()
    assert float(a[..., 3].mean()) == float(b[..., 3].mean()) == 4.0
    assert t.stats() == u.stats()
    assert _rel_mean_err(a[..., :3], b[..., :3]) < 1e-6


def test_async_image_readback_matches(system):
    """The pipelined read-back delivers the image as it stood when it was
    queued, while later frames keep rendering."""
    import torch
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=1, width=32, height=32)
    _, t = _setup(system, scene, dict(CORNELL_OPTS, Seed=5))
    host = [torch.empty(32 * 32 * 4, dtype=torch.float32).pin_memory() for _ in range(2)]
    t.render_frame()
    t.image_into_async(host[0].data_ptr())
    first_weight = None
    t.render_frame()
    t.wait_image()
    first_weight = float(host[0].view(32, 32, 4)[..., 3].mean())
    t.image_into_async(host[1].data_ptr())
    t.wait_image()
    assert first_weight == 1.0
    np.testing.assert_array_equal(host[1].numpy().reshape(32, 32, 4), t.image())
