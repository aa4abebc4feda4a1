"""Parity at the benchmark's own size: the seeded clusters scene of 1,000,008
triangles (1000 Gaussian clusters of 1000 triangles and four quad lights)
that the bench renders at 1920x1080, 1 sample per pixel, depth 8.

* Morton codes, the sort permutation and every LBVH array (left, right,
  parent, inner AABBs, root) bit-exact against the oracle;
* closest hits of the frame's camera rays (every 4th column of every 4th
  row: 129,600 rays): the binary layout bit-exact against the oracle's
  traversal of the same tree; the 8-wide layout, with every traversal
  kernel, with the same hit/miss and the same closest distance bit for bit,
  primitives differing only at ties (at most 0.1 % of rays);
* per-sample radiance of a band of 32 rows of the bench frame within the
  drop-in's 1e-4 relative mean error.

Everything the oracle uses is built by the oracle from the scene arrays.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_MEAN_TOL = 1e-4
OPTS = {"Samples": 1, "MaxDepth": 8, "NextEventEstimation": 1, "RussianRouletteStart": 3,
        "DirectLightMIS": 0, "Seed": 1}


@pytest.fixture(scope="module")
def big(system, oracle):
    from meturay_b200 import GPUScene, scenes
    scene = scenes.clusters(seed=1)
    assert scene.triangle_count == 1_000_008
    g = GPUScene(system, scene)
    g.construct_accelerators()
    return scene, g, oracle.OracleScene.from_scene(scene)


def test_lbvh_bit_exact_at_full_size(big, oracle):
    scene, g, _ = big
    acc = g.export_accel()
    aabbs, ext, delta, codes = oracle.morton_codes(scene.positions, scene.indices)
    n = scene.triangle_count
    sk, order = oracle.sort_pairs(codes, np.arange(n, dtype=np.uint32), 0, 63, False)
    assert np.array_equal(acc["codes"], sk)
    assert np.array_equal(acc["sorted_idx"], order)
    ref = oracle.lbvh(sk, order, aabbs)
    assert acc["root"][0] == ref["root"][0]
    for k in ("left", "right", "parent", "inner"):
        assert np.array_equal(acc[k], ref[k]), k


def _camera_rays(scene, step=4):
    """Pinhole rays (GPUCameraPinhole.cuh:209-243) through the centres of
    every step-th pixel of every step-th row, in float32 as the device
    computes them."""
    from meturay_b200 import camera_frame
    f = camera_frame(scene.camera)
    pos, bl, right, up, size = f[0:3], f[3:6], f[6:9], f[9:12], f[12:14]
    W, H = scene.width, scene.height
    xs = np.arange(0, W, step, dtype=np.float32)
    ys = np.arange(0, H, step, dtype=np.float32)
    px, py = np.meshgrid(xs, ys)
    dx, dy = np.float32(size[0] / np.float32(W)), np.float32(size[1] / np.float32(H))
    sx = (px * dx + np.float32(0.5) * dx).reshape(-1, 1).astype(np.float32)
    sy = (py * dy + np.float32(0.5) * dy).reshape(-1, 1).astype(np.float32)
    p = (bl + (sx * right + sy * up)).astype(np.float32)
    d = (p - pos).astype(np.float32)
    d = (d / np.sqrt((d * d).sum(1, keepdims=True))).astype(np.float32)
    rays = np.zeros((d.shape[0], 8), np.float32)
    rays[:, 0:3] = pos
    rays[:, 3] = scene.camera["near_far"][0]
    rays[:, 4:7] = d
    rays[:, 7] = scene.camera["near_far"][1]
    return rays


@pytest.mark.parametrize("mode", ["binary", "sorted", "octant", "sorted_refill",
                                  "octant_refill"])
def test_camera_closest_hits_at_full_size(big, cuda, mode):
    torch = cuda
    scene, g, os_ = big
    g.set_traversal(0 if mode == "binary" else 1)
    if mode != "binary":
        g.set_wide_order(mode)
    rays = _camera_rays(scene)
    n = rays.shape[0]
    assert n >= 100_000
    key, prim, t, bary = os_.trace(rays)
    ro = torch.from_numpy(np.ascontiguousarray(rays[:, 0:4])).cuda()
    rd = torch.from_numpy(np.ascontiguousarray(rays[:, 4:8])).cuda()
    dk = torch.zeros(n, dtype=torch.int32, device="cuda")
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    dt = torch.zeros(n, dtype=torch.float32, device="cuda")
    db = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    g.hit(ro.data_ptr(), rd.data_ptr(), n, dk.data_ptr(), dp.data_ptr(), dt.data_ptr(),
          db.data_ptr())
    torch.cuda.synchronize()
    g.set_traversal(1)
    g.set_wide_order("auto")
    gk = dk.cpu().numpy().view(np.uint32)
    gp = dp.cpu().numpy().view(np.uint32)
    gt = dt.cpu().numpy()
    gb = db.cpu().numpy()
    hit = prim != 0xFFFFFFFF
    assert hit.sum() > n // 50
    assert np.array_equal(gp != 0xFFFFFFFF, hit)
    assert np.array_equal(gt[hit].view(np.uint32), t[hit].view(np.uint32))
    same = gp == prim
    if mode == "binary":
        assert same.all()
    else:
        assert (~same).sum() <= n // 1000, f"{(~same).sum()} ties"
    assert np.array_equal(gk[same], key[same])
    assert np.array_equal(gb[same & hit].view(np.uint32), bary[same & hit].view(np.uint32))


def test_radiance_band_at_full_size(big, system):
    from meturay_b200 import PathTracer, camera_frame
    scene, g, os_ = big
    t = PathTracer(system, g)
    t.set_options(OPTS)
    t.generate_work()
    while t.render():
        pass
    t.finalize()
    gpu = t.sample_radiance()[..., :3]
    t.close()
    rows = (524, 556)
    cf = np.concatenate([camera_frame(scene.camera), np.float32(scene.camera["near_far"])])
    ref, rays = os_.render(cf, scene.width, scene.height, 1, OPTS["MaxDepth"],
                           OPTS["RussianRouletteStart"], True, OPTS["Seed"], rows=rows)
    a, b = gpu[rows[0]:rows[1]], ref[rows[0]:rows[1]]
    assert rays > 32 * scene.width
    assert b.sum() > 0
    err = float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-30))
    assert err < REL_MEAN_TOL, err
