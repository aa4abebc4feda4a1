"""Reconstruction filters on the GPU against the CPU oracle.

Integer-free but order-fixed: every pixel sums its samples in ascending
sample order on both sides, so the images must agree bit for bit.  The first
test is the reference's own filter test (Test_TracerCUDA/T_ReconFilter.cu)
at its full size.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FILTERS = [("Box", 0.0, {}), ("Box", 0.5, {}), ("Box", 1.25, {}), ("Tent", 1.0, {}),
           ("Tent", 1.5, {}), ("Gaussian", 1.5, {"alpha": 2.0}), ("Gaussian", 2.0, {"alpha": 0.5}),
           ("Mitchell", 2.0, {"b": 1 / 3, "c": 1 / 3})]


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


def _splat(cuda, ftype, radius, params, values, coords, res, segment=None, multiplier=1.0,
           repeat=1):
    import meturay_b200 as m
    ch = 1 if values.ndim == 1 else values.shape[1]
    img = m.ImageMemory(res[0], res[1], ch)
    if segment is not None:
        ox, oy, w, h = segment
        img.reportion((ox, oy), (ox + w, oy + h))
    f = m.ReconFilter(ftype, radius, params)
    dv = cuda.from_numpy(np.ascontiguousarray(values)).cuda()
    dc = cuda.from_numpy(np.ascontiguousarray(coords)).cuda()
    for _ in range(repeat):
        f.filter_to_img(img, dv, dc, coords.shape[0], multiplier)
    cuda.cuda.synchronize()
    return img.get_image()


def test_reference_filter_test(cuda, oracle):
    """T_ReconFilter.cu: 1M samples of 1.0 at mt19937(0) coordinates,
    1920x1080, Box radius 0.5, against the test's own CPU loop."""
    n, W, H = 1_000_000, 1920, 1080
    coords = oracle.mt19937_coords(n, W, H, 0)
    values = np.ones((n, 4), np.float32)
    px, cnt = _splat(cuda, "Box", 0.5, {}, values, coords, (W, H))
    ref_p, ref_c = oracle.filter_direct("Box", 0.5, values, coords, (W, H))
    assert _bits_equal(px, ref_p) and _bits_equal(cnt, ref_c)


@pytest.mark.parametrize("ftype,radius,params", FILTERS)
def test_filters_match_oracle(cuda, oracle, ftype, radius, params):
    rng = np.random.default_rng(5)
    n, W, H = 200_000, 320, 180
    # some samples off the image on every side
    coords = np.stack([rng.uniform(-3, W + 3, n), rng.uniform(-3, H + 3, n)],
                      1).astype(np.float32)
    values = rng.uniform(0, 8, (n, 4)).astype(np.float32)
    px, cnt = _splat(cuda, ftype, radius, params, values, coords, (W, H))
    ref_p, ref_c = oracle.filter_to_img(ftype, radius, values, coords, (W, H), **params)
    assert _bits_equal(px, ref_p) and _bits_equal(cnt, ref_c)


def test_single_channel_segment_multiplier_and_accumulation(cuda, oracle):
    rng = np.random.default_rng(9)
    n, W, H = 50_000, 200, 120
    coords = np.stack([rng.uniform(0, W, n), rng.uniform(0, H, n)], 1).astype(np.float32)
    values = rng.uniform(0, 2, n).astype(np.float32)
    seg = (33, 17, 101, 64)
    px, cnt = _splat(cuda, "Gaussian", 1.5, {"alpha": 1.0}, values, coords, (W, H), segment=seg,
                     multiplier=0.5, repeat=2)
    p1, c1 = oracle.filter_to_img("Gaussian", 1.5, values, coords, (W, H), segment=seg,
                                  multiplier=0.5, alpha=1.0)
    p2, c2 = oracle.filter_to_img("Gaussian", 1.5, values, coords, (W, H), segment=seg,
                                  multiplier=0.5, alpha=1.0, pixels=p1.copy(), counts=c1.copy())
    assert px.shape == (64, 101) and _bits_equal(px, p2) and _bits_equal(cnt, c2)


def test_empty_input_and_image_lifecycle(cuda):
    import meturay_b200 as m
    img = m.ImageMemory(64, 32, 4)
    assert img.info() == {"segment_offset": (0, 0), "segment_size": (64, 32),
                          "resolution": (64, 32), "channels": 4}
    f = m.ReconFilter("Tent", 1.0)
    empty = cuda.zeros((0, 4), dtype=cuda.float32, device="cuda")
    f.filter_to_img(img, empty, cuda.zeros((0, 2), dtype=cuda.float32, device="cuda"), 0)
    p, c = img.get_image()
    assert not p.any() and not c.any()
    # Reportion clamps the end to the resolution; Resize keeps the portion inside
    img.reportion((10, 4), (100, 20))
    assert img.info()["segment_size"] == (54, 16)
    with pytest.raises(m.MrbError):
        img.resize(40, 40)
    img.resize(80, 24)
    with pytest.raises(m.MrbError):
        f.filter_to_img(m.ImageMemory(8, 8, 1), cuda.zeros((4, 4), device="cuda"),
                        cuda.zeros((4, 2), device="cuda"), 4)


def test_nan_pixels_become_magenta_and_get_resets(cuda):
    import meturay_b200 as m
    img = m.ImageMemory(4, 2, 4)
    f = m.ReconFilter("Box", 0.0)
    v = cuda.tensor([[float("nan"), 0, 0, 1], [1, 2, 3, 4]], device="cuda")
    c = cuda.tensor([[0.5, 0.5], [2.5, 1.5]], device="cuda")
    f.filter_to_img(img, v, c, 2)
    p, cnt = img.get_image()
    assert _bits_equal(p[0, 0], np.array([1e30, 0.0, 1e30, 1.0], np.float32))
    assert p[1, 2].tolist() == [1.0, 2.0, 3.0, 4.0] and cnt[1, 2] == 1.0
    p2, c2 = img.get_image()
    assert not p2.any() and not c2.any()


# ---- the tracer's Finalize through a filter --------------------------------

OPTS = {"Samples": 2, "MaxDepth": 4, "NextEventEstimation": 1, "RussianRouletteStart": 3,
        "DirectLightMIS": 0, "Seed": 3}


def _tracer(system, scene, opts, tracer_type="PathTracer", flt=None):
    import meturay_b200 as m
    g = m.GPUScene(system, scene)
    g.construct_accelerators()
    t = system.generate_tracer(g, tracer_type, opts)
    if flt is not None:
        t.attach_recon_filter(m.ReconFilter(*flt))
    return g, t


@pytest.mark.parametrize("flt", [("Tent", 1.0, {}), ("Box", 0.5, {}),
                                 ("Gaussian", 2.0, {"alpha": 1.0}),
                                 ("Mitchell", 1.5, {"b": 1 / 3, "c": 1 / 3})])
def test_tracer_filter_matches_oracle_splat(system, cuda, oracle, flt):
    """One frame: the tracer's own samples, splatted by the oracle with the
    oracle's camera coordinates, equal the tracer's filtered image."""
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=2, width=48, height=40)
    g, t = _tracer(system, scene, OPTS, flt=flt)
    t.render_frame()
    img = t.image()
    samples = t.sample_radiance().reshape(-1, 4)
    coords = oracle.camera_img_coords(scene.width, scene.height, OPTS["Samples"], OPTS["Seed"], 0)
    ref_p, ref_c = oracle.filter_to_img(flt[0], flt[1], samples, coords,
                                        (scene.width, scene.height), **flt[2])
    assert _bits_equal(img[..., :3], ref_p[..., :3]) and _bits_equal(img[..., 3], ref_c)
    # and the general GPU path on the same samples gives the same bits
    px, cnt = _splat(cuda, flt[0], flt[1], flt[2], samples, coords, (scene.width, scene.height))
    assert _bits_equal(px[..., :3], img[..., :3]) and _bits_equal(cnt, img[..., 3])


@pytest.mark.parametrize("samples", [1, 3])
def test_tracer_filter_tile_and_fallback(system, oracle, samples):
    """The filter stages a 16x16 pixel tile's samples in shared memory where
    they fit (1 or 2 samples per pixel axis with these filters) and reads
    them from global memory otherwise (3 and more); either way the image is
    the oracle's splat bit for bit, on an image whose sides are not tile
    multiples."""
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=2, width=37, height=21)
    opts = dict(OPTS, Samples=samples)
    flt = ("Tent", 1.0, {})
    g, t = _tracer(system, scene, opts, flt=flt)
    t.render_frame()
    img = t.image()
    s = t.sample_radiance().reshape(-1, 4)
    coords = oracle.camera_img_coords(scene.width, scene.height, samples, opts["Seed"], 0)
    ref_p, ref_c = oracle.filter_to_img("Tent", 1.0, s, coords, (scene.width, scene.height))
    assert _bits_equal(img[..., :3], ref_p[..., :3]) and _bits_equal(img[..., 3], ref_c)


def test_tracer_filter_frames_accumulate_and_graph_matches_eager(system, oracle):
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=4, width=40, height=32)
    flt = ("Tent", 1.0, {})
    _, a = _tracer(system, scene, OPTS, flt=flt)
    _, b = _tracer(system, scene, OPTS, flt=flt)
    ref_p = ref_c = None
    for frame in range(3):
        a.render_frame()
        b.generate_work()
        while b.render():
            pass
        b.finalize()
        s = a.sample_radiance().reshape(-1, 4)
        coords = oracle.camera_img_coords(scene.width, scene.height, OPTS["Samples"],
                                          OPTS["Seed"], frame)
        ref_p, ref_c = oracle.filter_to_img("Tent", 1.0, s, coords, (scene.width, scene.height),
                                            pixels=ref_p, counts=ref_c)
    ia, ib = a.image(), b.image()
    assert _bits_equal(ia, ib)
    assert _bits_equal(ia[..., :3], ref_p[..., :3]) and _bits_equal(ia[..., 3], ref_c)
    # detaching returns to the per-pixel mean and restarts the image
    a.attach_recon_filter(None)
    a.render_frame()
    assert a.image()[..., 3].max() == 1.0


def test_wfpg_tracer_with_filter(system, oracle):
    from meturay_b200 import scenes
    scene = scenes.cornell(seed=5, width=32, height=32)
    opts = dict(OPTS, OctreeLevel=6, MinRayBinLevel=3, BinRayCount=64)
    flt = ("Gaussian", 1.5, {"alpha": 2.0})
    _, t = _tracer(system, scene, opts, "WFPGTracer", flt=flt)
    ref_p = ref_c = None
    for frame in range(2):
        t.render_frame()
        s = t.sample_radiance().reshape(-1, 4)
        coords = oracle.camera_img_coords(scene.width, scene.height, opts["Samples"],
                                          opts["Seed"], frame)
        ref_p, ref_c = oracle.filter_to_img(*flt[:2], s, coords, (scene.width, scene.height),
                                            pixels=ref_p, counts=ref_c, **flt[2])
    img = t.image()
    assert _bits_equal(img[..., :3], ref_p[..., :3]) and _bits_equal(img[..., 3], ref_c)
