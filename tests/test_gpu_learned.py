"""Learned guiding inside the WFPG tracer.

The network trains every frame from the path chains; each frame's batch is
scored before the step that learns from it, so the per-frame loss is a
held-out estimate of how well the mixture predicts where radiance arrives.
After the warm-up frames the network's sampler writes the guide words, and
the estimator stays unbiased (image mean against the plain tracer's).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPTS = {"Samples": 1, "MaxDepth": 5, "NextEventEstimation": 1, "RussianRouletteStart": 3,
        "DirectLightMIS": 0, "Seed": 5, "OctreeLevel": 6, "MinRayBinLevel": 3,
        "BinRayCount": 64, "LearnedGuiding": 1, "LearnedWarmupFrames": 4,
        "LearnedTrainSteps": 4, "LearnedSamples": 8192}


def _scene(system, w=64, h=48):
    from meturay_b200 import GPUScene, scenes
    g = GPUScene(system, scenes.cornell(seed=2, width=w, height=h))
    g.construct_accelerators()
    return g


def _mean(img):
    return img[..., :3].sum() / max(float(img[0, 0, 3]), 1.0) / (img.shape[0] * img.shape[1])


def test_learned_guiding_trains_and_guides(system):
    from meturay_b200 import PathTracer, WFPGTracer
    g = _scene(system)
    t = WFPGTracer(system, g)
    t.set_options(dict(OPTS, LearnedTrainSteps=4, LearnedWarmupFrames=40))
    t.set_options({"LearnedRate": 3e-3, "LearnedWeightMax": 5.0})
    t.render_frame()
    p0 = t.learned_params()
    losses = [t.learned_loss()]
    for _ in range(119):
        t.render_frame()
        losses.append(t.learned_loss())
    p1 = t.learned_params()
    assert np.all(np.isfinite(p1)) and not np.array_equal(p0, p1)
    assert all(np.isfinite(losses))
    # the held-out loss falls as the network learns the incident radiance
    assert np.mean(losses[-10:]) < np.mean(losses[:3]) - 0.3, (losses[:3], losses[-10:])
    # after the warm-up the network's sampler writes the guide words
    t.generate_work()
    assert t.render()
    gs = t.guide_state()
    valid = (gs["guide"][:, 1] >> 17) & 1
    assert valid.sum() > 0.5 * len(valid)
    while t.render():
        pass
    t.finalize()
    # unbiased: the image mean matches the plain tracer's within the noise
    guided = t.image()
    p = PathTracer(system, g)
    p.set_options({k: OPTS[k] for k in ("Samples", "MaxDepth", "NextEventEstimation",
                                         "RussianRouletteStart", "DirectLightMIS")})
    p.set_options({"Seed": 77})
    for _ in range(121):
        p.render_frame()
    a, b = _mean(guided), _mean(p.image())
    assert abs(a - b) < 0.05 * b, (a, b)


def test_learned_options_and_errors(system):
    import meturay_b200 as m
    from meturay_b200 import WFPGTracer
    g = _scene(system, 16, 16)
    t = WFPGTracer(system, g)
    with pytest.raises(m.MrbError):
        t.learned_params()                   # no network before the option and a frame
    for bad in ({"LearnedTrainSteps": 0}, {"LearnedSamples": 10}):
        with pytest.raises(m.MrbError):
            t.set_options(bad)
    with pytest.raises(m.MrbError):
        t.set_options({"LearnedRate": 2.0})
    t.set_options(dict(OPTS, LearnedWarmupFrames=1, LearnedSeed=9))
    for _ in range(3):
        t.render_frame()
    assert np.all(np.isfinite(t.learned_params()))


def _ratio_image(t):
    img = t.image().astype(np.float64)
    w = img[..., 3:]
    return np.where(w > 0, img[..., :3] / np.where(w > 0, w, 1.0), 0.0)


def test_learned_sampler_lowers_the_error_at_equal_samples(system):
    """What the trained network gains over the method without it, where
    guiding has something to gain: the Cornell scene with its light facing
    the ceiling above an opaque panel, so that the room is lit indirectly.
    The same tracer renders 400 frames of 4 spp twice per seed, once with the
    network guiding after 16 warm-up frames and once with the BxDF sampling
    every frame (the network never taking over).  Errors are taken against
    a plain render of two independent halves, less that render's own
    variance, over three seeds; the median of the per-seed ratios is the
    measure, because the online training adds its gradients with float
    atomics, so its trajectory, and now and then a firefly of one seed's
    learned run, differ from run to run.  (With next-event estimation on
    the scene with the ceiling-wide light, NEE's fireflies next to the light
    dominate every estimator's error; the next test guides that scene with
    NEE off.)"""
    from meturay_b200 import GPUScene, PathTracer, WFPGTracer, scenes
    g = GPUScene(system, scenes.cornell(seed=1, shielded=True))
    g.construct_accelerators()
    base = {"Samples": 2, "MaxDepth": 5, "NextEventEstimation": 1, "RussianRouletteStart": 3,
            "DirectLightMIS": 0}
    halves = []
    for seed in (4242, 5353):
        ref = PathTracer(system, g)
        ref.set_options(dict(base, Seed=seed))
        for _ in range(2048):
            ref.render_frame()
        halves.append(_ratio_image(ref))
        ref.close()
    reference = 0.5 * (halves[0] + halves[1])
    ref_var = float(np.mean((halves[0] - halves[1]) ** 2)) / 4.0
    mse = {"learned": [], "bxdf": []}
    for seed in (13, 14, 15):
        for name, warmup in (("learned", 16), ("bxdf", 1 << 30)):
            t = WFPGTracer(system, g)
            t.set_options(dict(base, Seed=seed, LearnedGuiding=1, LearnedWarmupFrames=warmup,
                               LearnedWarmupOctree=0, LearnedTrainSteps=4,
                               LearnedSamples=65536, OctreeLevel=10, MinRayBinLevel=5,
                               BinRayCount=512))
            t.set_options({"LearnedRate": 1e-2, "LearnedWeightMax": 5.0,
                           "BXDF-GuideMISRatio": 0.5})
            for _ in range(400):
                t.render_frame()
            mse[name].append(float(np.mean((_ratio_image(t) - reference) ** 2)) - ref_var)
            t.close()
    ratio = float(np.median(np.array(mse["learned"]) / np.array(mse["bxdf"])))
    print(mse, ratio)
    assert ratio < 0.85, mse


def test_learned_sampler_lowers_the_error_on_the_configured_scene(system):
    """The configured learned-guiding scene (config-1 Cornell box with its
    ceiling-wide light) with next-event estimation off, as the reference's
    own WFPG configurations run: the network, guiding after 16 warm-up
    frames, lowers the error of 400 frames of 4 spp against the same tracer
    sampling the BxDF every frame, averaged over two seeds.  The reference
    is the plain tracer with NEE and MIS (the same expectation at far lower
    variance), two independent halves, its variance subtracted."""
    from meturay_b200 import GPUScene, PathTracer, WFPGTracer, scenes
    g = GPUScene(system, scenes.cornell(seed=1))
    g.construct_accelerators()
    base = {"Samples": 2, "MaxDepth": 5, "NextEventEstimation": 0, "RussianRouletteStart": 3,
            "DirectLightMIS": 0}
    halves = []
    for seed in (4242, 5353):
        ref = PathTracer(system, g)
        ref.set_options(dict(base, Seed=seed, NextEventEstimation=1, DirectLightMIS=1))
        for _ in range(2048):
            ref.render_frame()
        halves.append(_ratio_image(ref))
        ref.close()
    reference = 0.5 * (halves[0] + halves[1])
    ref_var = float(np.mean((halves[0] - halves[1]) ** 2)) / 4.0
    mse = {"learned": [], "bxdf": []}
    for seed in (13, 14):
        for name, warmup in (("learned", 16), ("bxdf", 1 << 30)):
            t = WFPGTracer(system, g)
            t.set_options(dict(base, Seed=seed, LearnedGuiding=1, LearnedWarmupFrames=warmup,
                               LearnedWarmupOctree=0, LearnedTrainSteps=4,
                               LearnedSamples=65536, OctreeLevel=10, MinRayBinLevel=5,
                               BinRayCount=512, GuideBounceAmount=2))
            t.set_options({"LearnedRate": 1e-2, "LearnedWeightMax": 5.0,
                           "BXDF-GuideMISRatio": 0.5})
            for _ in range(400):
                t.render_frame()
            mse[name].append(float(np.mean((_ratio_image(t) - reference) ** 2)) - ref_var)
            t.close()
    learned, bxdf = float(np.mean(mse["learned"])), float(np.mean(mse["bxdf"]))
    print(mse)
    assert learned < 0.8 * bxdf, mse
