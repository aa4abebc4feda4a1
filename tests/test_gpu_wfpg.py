"""Wavefront path guiding (WFPGTracer) on the GPU against the CPU oracle.

The oracle restates the WFPG hot path depth by depth over every path:
octree payload (k-means voxel normals, light radiance, node normals,
averages and level filters), ray binning and bin collapse, the per-bin
radiance field (cone traces, Gaussian filter), the 8x8 product sampler with
BxDF MIS, guided shading, the path chain and the radiance deposit.  Bin
counts and radiance sums are integers and every random number is keyed by
path / bin, so the guide words, bin ids and the octree payload must agree
bit for bit; the per-sample radiance (float atomics on the device) must
agree to a relative mean error below 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_MEAN_TOL = 1e-4
PAYLOAD = ("leaf_normals", "node_normals", "leaf_irr", "leaf_cnt", "leaf_avg", "node_avg")
# what a frame changes: the radiance state, the shadow-ray counters
# (DepositNEEHitMiss) and the node guiding factors
FRAME_STATE = PAYLOAD[2:] + ("leaf_shadow", "node_factor")


def _rel_mean_err(a, b):
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-30))


def _oracle_svo(oracle, g, scene, res, omit=False):
    """The oracle's octree from its own tables and scene extent."""
    ex = oracle.scene_tables(scene)
    return oracle.OracleSvo(scene, ex["tri_key"], oracle.scene_extent(scene), res,
                            ex["light_radiance"], omit_direct=omit)


def _assert_payload(gpu, ref, keys=PAYLOAD):
    for k in keys:
        assert np.array_equal(gpu[k], ref[k]), (k, int(np.sum(gpu[k] != ref[k])))


@pytest.mark.parametrize("which,res", [("cornell", 64), ("clusters", 128)])
def test_svo_payload_matches_oracle(system, oracle, which, res):
    from meturay_b200 import GPUScene, scenes
    scene = (scenes.cornell(seed=2, mixed=True) if which == "cornell"
             else scenes.clusters(seed=3, n_clusters=30, tris_per_cluster=300))
    g = GPUScene(system, scene)
    g.construct_accelerators()
    g.build_svo(res)
    gpu = g.export_svo()
    ref = _oracle_svo(oracle, g, scene, res).export()
    assert ref["status"] == 0
    assert np.array_equal(gpu["nodes"], ref["nodes"])
    _assert_payload(gpu, ref)
    # light voxels start with radiance on both sides
    lit = gpu["leaf_lights"] != 0
    assert lit.any() and (gpu["leaf_cnt"][lit] == 10000).all()


WFPG_OPTS = {"Samples": 1, "MaxDepth": 5, "NextEventEstimation": 1, "RussianRouletteStart": 3,
             "DirectLightMIS": 0, "Seed": 3, "OctreeLevel": 6, "MinRayBinLevel": 3,
             "BinRayCount": 64}


def _wfpg(system, scene, opts):
    from meturay_b200 import GPUScene, WFPGTracer
    g = GPUScene(system, scene)
    g.construct_accelerators()
    t = WFPGTracer(system, g)
    t.set_options(opts)
    return g, t


def _oracle_kwargs(opts):
    return dict(min_bin_level=opts.get("MinRayBinLevel", 5),
                bin_ray_count=opts.get("BinRayCount", 512),
                pure_pg=bool(opts.get("PurePG", 0)), skip_pg=bool(opts.get("SkipPG", 0)),
                guide_bounce=opts.get("GuideBounceAmount", 512),
                mis_ratio=opts.get("BXDF-GuideMISRatio", 0.5),
                filter_alpha=opts.get("RFieldFilterAlpha", 1.0),
                mis=bool(opts.get("DirectLightMIS", 0)),
                product=bool(opts.get("DoProductPathGuiding", 1)))


def _cam(scene):
    from meturay_b200 import camera_frame
    return np.concatenate([camera_frame(scene.camera), np.float32(scene.camera["near_far"])])


@pytest.mark.parametrize("product", [1, 0])
def test_guide_words_and_bins_match_oracle(system, oracle, product):
    """Per-ray bins and guide words of the first wavefront, for the product
    sampler and for the 2D piecewise-constant sampler over the field
    (DoProductPathGuiding false)."""
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=6, width=32, height=32, mixed=True)
    opts = dict(WFPG_OPTS, DoProductPathGuiding=product)
    g, t = _wfpg(system, scene, opts)
    t.generate_work()
    t.render()
    st = t.guide_state()
    o = oracle.OracleScene.from_scene(scene)
    svo = _oracle_svo(oracle, g, scene, 1 << opts["OctreeLevel"])
    _, _, dg, db = o.render_wfpg(_cam(scene), scene.width, scene.height, 1, opts["MaxDepth"],
                                 opts["RussianRouletteStart"], True, opts["Seed"], svo,
                                 dump_iteration=0, **_oracle_kwargs(opts))
    n = len(st["samples"])
    assert n == scene.width * scene.height
    # per-ray bin from the sorted (bin, ray) pairs
    gbin = np.full(n, 0xFFFFFFFF, np.uint32)
    gbin[st["sorted_rid"]] = st["sorted_bin"]
    smp = st["samples"]
    assert np.array_equal(gbin, db[smp])
    valid = (st["guide"][:, 1] >> 17) & 1
    assert valid.sum() > 0
    assert np.array_equal(st["guide"][valid == 1], dg[smp][valid == 1])
    assert np.array_equal(valid, (dg[smp][:, 1] >> 17) & 1)


@pytest.mark.parametrize("variant", ["mis", "pure", "mis_nee_mis", "nonproduct",
                                     "nonproduct_pure", "nee_off"])
def test_wfpg_frames_match_oracle(system, oracle, variant):
    """Two stepwise frames: per-sample radiance and the octree payload after
    each frame's deposit."""
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=6, width=32, height=32, mixed=True)
    opts = dict(WFPG_OPTS)
    if variant in ("pure", "nonproduct_pure"):
        opts["PurePG"] = 1
    if variant.startswith("nonproduct"):
        opts["DoProductPathGuiding"] = 0
    if variant == "nee_off":
        # path rays reaching a light or leaving the box count as hits
        opts["NextEventEstimation"] = 0
    if variant == "mis_nee_mis":
        opts["DirectLightMIS"] = 1
        opts["BXDF-GuideMISRatio"] = 0.7
        opts["RFieldFilterAlpha"] = 0.6
    g, t = _wfpg(system, scene, opts)
    o = oracle.OracleScene.from_scene(scene)
    svo = _oracle_svo(oracle, g, scene, 1 << opts["OctreeLevel"])
    for frame in range(2):
        t.generate_work()
        while t.render():
            pass
        t.finalize()
        gpu = t.sample_radiance()[..., :3]
        ref, ref_rays, _, _ = o.render_wfpg(_cam(scene), scene.width, scene.height, 1,
                                            opts["MaxDepth"], opts["RussianRouletteStart"],
                                            bool(opts["NextEventEstimation"]), opts["Seed"], svo,
                                            frame=frame, **_oracle_kwargs(opts))
        rays, frames = t.stats()
        assert gpu.sum() > 0
        assert _rel_mean_err(gpu, ref) < REL_MEAN_TOL
        ex = t.export_svo()
        _assert_payload(ex, svo.export(), FRAME_STATE)
        # NEE rays reach their light from some vertices and are stopped
        # from others; nodes over leaves with shadow rays carry a factor
        sh = ex["leaf_shadow"]
        assert sh[:, 0].sum() > 0
        assert (sh[:, 1].sum() > 0) == (variant != "nee_off")
        assert np.count_nonzero(ex["node_factor"] != 0x7FFF) > 0


def test_wfpg_graph_frames_match_stepwise(system, oracle):
    """Frames replayed from the captured graph give the oracle's octree and
    image (the graph's warm-up frame does not leak into the cache)."""
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=7, width=32, height=32, mixed=True)
    opts = dict(WFPG_OPTS, Seed=11)
    g, t = _wfpg(system, scene, opts)
    o = oracle.OracleScene.from_scene(scene)
    svo = _oracle_svo(oracle, g, scene, 1 << opts["OctreeLevel"])
    acc = np.zeros((scene.height, scene.width, 3), np.float64)
    for frame in range(3):
        t.render_frame()
        ref, _, _, _ = o.render_wfpg(_cam(scene), scene.width, scene.height, 1, opts["MaxDepth"],
                                     opts["RussianRouletteStart"], True, opts["Seed"], svo,
                                     frame=frame, **_oracle_kwargs(opts))
        acc += ref
    img = t.image()
    assert img[..., 3].min() == 3.0
    assert _rel_mean_err(img[..., :3].astype(np.float64), acc) < REL_MEAN_TOL
    _assert_payload(t.export_svo(), svo.export(), FRAME_STATE)


def test_wfpg_skip_pg_is_unguided(system, oracle):
    """SkipPG keeps the chain and the deposit but samples every direction from
    the BxDF."""
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=6, width=32, height=32, mixed=True)
    opts = dict(WFPG_OPTS, SkipPG=1)
    g, t = _wfpg(system, scene, opts)
    o = oracle.OracleScene.from_scene(scene)
    svo = _oracle_svo(oracle, g, scene, 1 << opts["OctreeLevel"])
    t.generate_work()
    while t.render():
        pass
    t.finalize()
    ref, _, _, _ = o.render_wfpg(_cam(scene), scene.width, scene.height, 1, opts["MaxDepth"],
                                 opts["RussianRouletteStart"], True, opts["Seed"], svo,
                                 **_oracle_kwargs(opts))
    assert _rel_mean_err(t.sample_radiance()[..., :3], ref) < REL_MEAN_TOL
    _assert_payload(t.export_svo(), svo.export(), FRAME_STATE)


def test_wfpg_on_a_scene_file(system, oracle):
    """WFPG frames of an MRay scene file (transformed light, Unreal, Metal,
    Refract) match the oracle, image and octree."""
    from pathlib import Path
    import meturay_b200 as m
    scene = m.load_scene(Path(__file__).resolve().parent / "scenes" / "box_mixed.json", 32, 24)
    opts = dict(WFPG_OPTS, OctreeLevel=5, MinRayBinLevel=2, BinRayCount=32)
    g, t = _wfpg(system, scene, opts)
    o = oracle.OracleScene.from_scene(scene)
    svo = _oracle_svo(oracle, g, scene, 1 << opts["OctreeLevel"])
    for frame in range(2):
        t.generate_work()
        while t.render():
            pass
        t.finalize()
        ref, _, _, _ = o.render_wfpg(_cam(scene), scene.width, scene.height, 1, opts["MaxDepth"],
                                     opts["RussianRouletteStart"], True, opts["Seed"], svo,
                                     frame=frame, **_oracle_kwargs(opts))
        gpu = t.sample_radiance()[..., :3]
        assert gpu.sum() > 0
        assert _rel_mean_err(gpu, ref) < REL_MEAN_TOL
        _assert_payload(t.export_svo(), svo.export(), FRAME_STATE)
