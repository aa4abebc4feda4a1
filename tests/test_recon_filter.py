"""Reconstruction filters on the host: the oracle against the reference's own
filter test, the library's host functors against the oracle, option errors.

The reference's test (Test_TracerCUDA/T_ReconFilter.cu) splats 1,000,000
samples of value 1 at std::mt19937(0) uniform coordinates over 1920x1080
through a Box filter of radius 0.5 and checks the GPU image against a
direct CPU loop.  The oracle's restatement of the GPU algorithm (expand,
stable sort by pixel, per-pixel sums) must equal that loop exactly.
"""
import math

import numpy as np
import pytest

from oracle import oracle as o

FILTERS = [("Box", 0.5, {}), ("Box", 1.0, {}), ("Tent", 1.0, {}), ("Tent", 1.5, {}),
           ("Gaussian", 1.5, {"alpha": 2.0}), ("Gaussian", 2.0, {"alpha": 0.5}),
           ("Mitchell", 2.0, {"b": 1 / 3, "c": 1 / 3}), ("Mitchell", 1.25, {"b": 0.0, "c": 0.5})]


def test_pixel_window_table():
    # FilterRadiusToPixelWH: 0 -> 1, (0, 0.5] -> 2, (0.5, 1] -> 3, (1, 1.5] -> 4 ...
    import meturay_b200 as m
    table = {0.0: 1, 0.1: 2, 0.5: 2, 0.51: 3, 1.0: 3, 1.2: 4, 1.5: 4, 2.0: 5, 2.25: 6, 3.0: 7}
    for r, wh in table.items():
        assert o.filter_pixel_wh(r) == wh, r
        assert m.filter_pixel_wh(r) == wh, r


def _canonical_float(raw: np.ndarray) -> np.ndarray:
    # libstdc++ generate_canonical<float, 24> on a 32-bit engine: one draw,
    # float(r) / 2^32, clamped below 1
    c = raw.astype(np.float32) / np.float32(2.0 ** 32)
    return np.where(c >= 1.0, np.nextafter(np.float32(1), np.float32(0)), c).astype(np.float32)


def test_mt19937_inputs_match_the_standard_library_recipe():
    bg = np.random.MT19937(0)
    bg._legacy_seeding(0)  # init_genrand(0), as std::mt19937::seed(0)
    raw = bg.random_raw(2 * 1000).astype(np.uint32)
    c = _canonical_float(raw).reshape(-1, 2)
    exp = np.stack([c[:, 0] * np.float32(1920.0), c[:, 1] * np.float32(1080.0)], 1)
    got = o.mt19937_coords(1000, 1920, 1080, 0)
    assert np.array_equal(got, exp.astype(np.float32))


def test_oracle_equals_the_reference_tests_expectation():
    """The reference test itself, at its full size, on the CPU."""
    n, W, H = 1_000_000, 1920, 1080
    coords = o.mt19937_coords(n, W, H, 0)
    values = np.ones((n, 4), np.float32)
    p0, c0 = o.filter_direct("Box", 0.5, values, coords, (W, H))
    p1, c1 = o.filter_to_img("Box", 0.5, values, coords, (W, H))
    assert np.array_equal(p0, p1) and np.array_equal(c0, c1)
    # with value 1 in every channel, pixels = counts (box weights are 0/1)
    assert np.array_equal(p1[..., 0], c1) and c1.sum() > 0.7 * n


@pytest.mark.parametrize("ftype,radius,params", FILTERS)
def test_oracle_pipeline_equals_direct_loop(ftype, radius, params):
    rng = np.random.default_rng(7)
    n, W, H = 20000, 96, 64
    coords = np.stack([rng.uniform(-2, W + 2, n), rng.uniform(-2, H + 2, n)], 1).astype(np.float32)
    values = rng.uniform(0, 4, (n, 4)).astype(np.float32)
    p0, c0 = o.filter_direct(ftype, radius, values, coords, (W, H), **params)
    p1, c1 = o.filter_to_img(ftype, radius, values, coords, (W, H), **params)
    assert np.array_equal(p0, p1) and np.array_equal(c0, c1)


@pytest.mark.parametrize("ftype,radius,params", FILTERS + [("Box", 0.0, {})])
def test_library_host_functor_equals_oracle(ftype, radius, params):
    import meturay_b200 as m
    f = m.ReconFilter(ftype, radius, params)
    rng = np.random.default_rng(3)
    for _ in range(500):
        px, py = rng.integers(0, 50, 2) + 0.5
        sx, sy = px + rng.uniform(-radius - 0.5, radius + 0.5, 2)
        a = f.weight((px, py), (sx, sy))
        b = o.filter_weight(ftype, radius, px, py, sx, sy, **params)
        assert np.float32(a).tobytes() == np.float32(b).tobytes()


def test_filter_shapes():
    # Tent: linear in each axis; Gaussian: 0 at the radius, exp(-a d^2) - edge inside;
    # Mitchell (1/3, 1/3): the 1D kernel at 0 is (6 + 2b) / 6
    assert o.filter_weight("Tent", 1.0, 0.5, 0.5, 0.75, 0.5) == pytest.approx(0.75)
    assert o.filter_weight("Tent", 2.0, 0.5, 0.5, 1.5, 1.5) == pytest.approx(0.25)
    assert o.filter_weight("Gaussian", 1.5, 0.5, 0.5, 2.0, 0.5, alpha=2.0) == 0.0
    g = o.filter_weight("Gaussian", 1.5, 0.5, 0.5, 1.0, 0.5, alpha=2.0)
    edge = math.exp(-2.0 * 1.5 ** 2)
    assert g == pytest.approx((math.exp(-2.0 * 0.25) - edge) * (1 - edge), rel=1e-6)
    b = 1 / 3
    assert o.filter_weight("Mitchell", 2.0, 0.5, 0.5, 0.5, 0.5, b=b, c=b) == pytest.approx(
        ((6 + 2 * b) / 6) ** 2, rel=1e-6)
    assert o.filter_weight("Mitchell", 2.0, 0.5, 0.5, 2.5, 0.5, b=b, c=b) == 0.0
    # Box radius 0: every sample weighs 1 (the no-filter mode)
    assert o.filter_weight("Box", 0.0, 0.5, 0.5, 7.0, -3.0) == 1.0


def test_portable_exp_accuracy():
    x = np.linspace(-87.0, 88.0, 400001, dtype=np.float32)
    y = o.pexp(x).astype(np.float64)
    ref = np.exp(x.astype(np.float64))
    ulp = np.abs(y - ref) / np.spacing(ref.astype(np.float32)).astype(np.float64)
    assert ulp.max() < 2.0
    assert o.pexp(np.array([0.0, -200.0, 100.0], np.float32)).tolist() == [1.0, 0.0, math.inf]


def test_segment_and_multiplier():
    rng = np.random.default_rng(11)
    n, W, H = 5000, 40, 30
    coords = np.stack([rng.uniform(0, W, n), rng.uniform(0, H, n)], 1).astype(np.float32)
    values = rng.uniform(0, 1, n).astype(np.float32)
    full_p, full_c = o.filter_to_img("Tent", 1.0, values, coords, (W, H), multiplier=2.0)
    seg_p, seg_c = o.filter_to_img("Tent", 1.0, values, coords, (W, H), segment=(8, 5, 20, 12),
                                   multiplier=2.0)
    assert np.array_equal(seg_p, full_p[5:17, 8:28]) and np.array_equal(seg_c, full_c[5:17, 8:28])


@pytest.mark.parametrize("args,needle", [
    (("Gaussian", 1.0, {}), "alpha"),
    (("Mitchell", 1.0, {"b": 0.3}), '"c"'),
    (("Mitchell", 1.0, {"c": 0.3}), '"b"'),
    (("Lanczos", 1.0, {}), "unknown type"),
    (("Tent", 0.0, {}), "radius 0"),
    (("Box", -1.0, {}), "radius"),
    (("Box", 100.0, {}), "radius"),
])
def test_filter_option_errors(args, needle):
    import meturay_b200 as m
    with pytest.raises(m.MrbError) as e:
        m.ReconFilter(*args)
    assert needle in str(e.value)


def test_generate_recon_filter_from_options():
    import meturay_b200 as m
    f = m.ReconFilter.from_options({"type": "Tent", "radius": 1.0})
    assert f.type() == "Tent" and f.used_gpu_memory() == 0
    with pytest.raises(m.MrbError, match="radius"):
        m.ReconFilter.from_options({"type": "Tent"})
    with pytest.raises(m.MrbError, match="type"):
        m.ReconFilter.from_options({"radius": 1.0})
