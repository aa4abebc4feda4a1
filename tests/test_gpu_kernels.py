"""Kernel-level parity of the CUDA path against the CPU oracle.

Integer stages (Morton codes, sort permutations, LBVH node indices, partition
offsets) must be bit-exact; closest hits of the LBVH traversal must equal the
oracle's traversal of the same tree bit for bit (same arithmetic, same visit
order), and the brute-force reference accelerator except at recorded ties.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_portable_math_bit_identical(cuda, oracle):
    from meturay_b200._lib import check, lib
    torch = cuda
    rng = np.random.default_rng(3)
    x = np.concatenate([np.linspace(0, 2 * np.pi, 50001), rng.uniform(-8, 8, 50000),
                        [0.0, np.pi / 4, np.pi / 2, np.pi, 1e-30]]).astype(np.float32)
    y = np.concatenate([np.linspace(-1, 1, 50001), rng.uniform(-1, 1, 50005)]).astype(np.float32)
    n = x.shape[0]
    assert y.shape[0] == n
    dx, dy = _dev(torch, x), _dev(torch, y)
    sc = torch.zeros(2 * n, dtype=torch.float32, device="cuda")
    ac = torch.zeros(n, dtype=torch.float32, device="cuda")
    check(lib.mrb_debug_math(dx.data_ptr(), n, sc.data_ptr(), dy.data_ptr(), ac.data_ptr(), None))
    torch.cuda.synchronize()
    sc, ac = sc.cpu().numpy().reshape(n, 2), ac.cpu().numpy()
    s = C.c_float()
    c = C.c_float()
    ref_sc = np.zeros((n, 2), np.float32)
    for i in range(n):
        oracle.lib.oracle_sincosf(C.c_float(x[i]), C.byref(s), C.byref(c))
        ref_sc[i] = (s.value, c.value)
    ref_ac = np.array([oracle.lib.oracle_acosf(float(v)) for v in y], np.float32)
    assert np.array_equal(sc.view(np.uint32), ref_sc.view(np.uint32))
    assert np.array_equal(ac.view(np.uint32), ref_ac.view(np.uint32))
    # accuracy against libm (stated bound: 2 ulp-ish absolute on these ranges)
    assert np.abs(sc[:, 0] - np.sin(x.astype(np.float64))).max() < 5e-7
    assert np.abs(ac - np.arccos(y.astype(np.float64))).max() < 1e-6


@pytest.mark.parametrize("n", [1, 2, 3, 1000, 4096, 4097, 100000])
def test_morton_codes_bit_exact(cuda, oracle, n):
    from meturay_b200 import scenes
    from meturay_b200._lib import check, lib
    torch = cuda
    sc = scenes.random_triangles(seed=n, n=n)
    aabbs, ext, delta, codes = oracle.morton_codes(sc.positions, sc.indices)
    dp, di = _dev(torch, sc.positions), _dev(torch, sc.indices)
    da = torch.zeros((n, 6), dtype=torch.float32, device="cuda")
    de = torch.zeros(8, dtype=torch.float32, device="cuda")
    dc = torch.zeros(n, dtype=torch.int64, device="cuda")
    check(lib.mrb_morton_codes(dp.data_ptr(), di.data_ptr(), n, da.data_ptr(), de.data_ptr(),
                               dc.data_ptr(), None))
    torch.cuda.synchronize()
    assert np.array_equal(da.cpu().numpy(), aabbs)
    assert np.array_equal(de.cpu().numpy()[:6], ext)
    assert de.cpu().numpy()[6] == np.float32(delta)
    assert np.array_equal(dc.cpu().numpy().view(np.uint64), codes)


@pytest.mark.parametrize("n", [0, 1, 7, 4095, 4096, 4097, 65537, 1 << 20])
@pytest.mark.parametrize("bits,desc", [((0, 64), False), ((0, 63), False), ((8, 27), True),
                                       ((0, 5), True)])
def test_radix_sort_u64(cuda, oracle, n, bits, desc):
    from meturay_b200._lib import check, lib
    torch = cuda
    rng = np.random.default_rng(n + bits[0])
    keys = rng.integers(0, 2**63, size=n, dtype=np.uint64)
    if n > 10:
        keys[: n // 3] = keys[n // 3: 2 * (n // 3)]  # many equal keys: stability matters
    vals = rng.permutation(n).astype(np.uint32)
    ek, ev = oracle.sort_pairs(keys, vals, bits[0], bits[1], desc)
    if n == 0:
        return
    dk, dv = _dev(torch, keys.view(np.int64)), _dev(torch, vals.view(np.int32))
    tb = lib.mrb_radix_sort_temp_bytes(n, 8, bits[0], bits[1])
    tmp = torch.zeros(tb, dtype=torch.uint8, device="cuda")
    check(lib.mrb_radix_sort_pairs_u64(dk.data_ptr(), dv.data_ptr(), n, bits[0], bits[1],
                                       int(desc), tmp.data_ptr(), tb, None))
    torch.cuda.synchronize()
    assert np.array_equal(dk.cpu().numpy().view(np.uint64), ek)
    assert np.array_equal(dv.cpu().numpy().view(np.uint32), ev)


@pytest.mark.parametrize("n", [1, 33, 4097, 300000])
@pytest.mark.parametrize("bits,desc", [((0, 32), True), ((0, 12), True), ((3, 11), False)])
def test_radix_sort_u32(cuda, oracle, n, bits, desc):
    from meturay_b200._lib import check, lib
    torch = cuda
    rng = np.random.default_rng(7 * n + bits[1])
    keys = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    keys[::3] &= 0xF0F
    vals = np.arange(n, dtype=np.uint32)
    ek, ev = oracle.sort_pairs(keys, vals, bits[0], bits[1], desc)
    dk, dv = _dev(torch, keys.view(np.int32)), _dev(torch, vals.view(np.int32))
    tb = lib.mrb_radix_sort_temp_bytes(n, 4, bits[0], bits[1])
    tmp = torch.zeros(tb, dtype=torch.uint8, device="cuda")
    check(lib.mrb_radix_sort_pairs_u32(dk.data_ptr(), dv.data_ptr(), n, bits[0], bits[1],
                                       int(desc), tmp.data_ptr(), tb, None))
    torch.cuda.synchronize()
    assert np.array_equal(dk.cpu().numpy().view(np.uint32), ek)
    assert np.array_equal(dv.cpu().numpy().view(np.uint32), ev)


def _build(system, scene, tree=None, collapse=None):
    from meturay_b200 import GPUScene
    g = GPUScene(system, scene)
    if tree is not None:
        g.set_wide_tree(tree)
    if collapse is not None:
        g.set_wide_collapse(collapse)
    g.construct_accelerators()
    return g


def _scenes():
    from meturay_b200 import scenes
    return [("cornell", lambda: scenes.cornell(seed=1)),
            ("random2", lambda: scenes.random_triangles(seed=5, n=2)),
            ("random3", lambda: scenes.random_triangles(seed=6, n=3)),
            ("random50k", lambda: scenes.random_triangles(seed=9, n=50000)),
            ("clusters_small", lambda: scenes.clusters(seed=2, n_clusters=40,
                                                       tris_per_cluster=500))]


@pytest.mark.parametrize("name,make", _scenes())
def test_lbvh_bit_exact(system, oracle, name, make):
    scene = make()
    g = _build(system, scene)
    acc = g.export_accel()
    aabbs, ext, delta, codes = oracle.morton_codes(scene.positions, scene.indices)
    order = np.argsort(codes, kind="stable").astype(np.uint32)
    assert np.array_equal(acc["codes"], codes[order])
    assert np.array_equal(acc["sorted_idx"], order)
    ref = oracle.lbvh(codes[order], order, aabbs)
    n = scene.triangle_count
    assert acc["root"][0] == ref["root"][0]
    assert np.array_equal(acc["parent"], ref["parent"])
    if n > 1:
        assert np.array_equal(acc["left"], ref["left"])
        assert np.array_equal(acc["right"], ref["right"])
        assert np.array_equal(acc["inner"], ref["inner"])


def _rays_for(scene, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = scene.positions.min(0), scene.positions.max(0)
    span = hi - lo
    o = lo - 0.2 * span + rng.uniform(size=(n, 3)) * 1.4 * span
    tgt = scene.positions[rng.integers(0, scene.positions.shape[0], n)]
    d = tgt - o + rng.normal(size=(n, 3)) * 0.01 * span
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = 0.0
    rays[:, 4:7] = d
    rays[:, 7] = 3.0e38
    rays[::7, 7] = 0.5          # some short rays
    rays[1::11, 3] = 0.3        # some rays starting late
    rays[2::13, 4:7] = [0.0, 1.0, 0.0]  # axis-aligned directions (zero components)
    return rays


KERNELS = ("sorted", "octant", "sorted_refill", "octant_refill")
# the automatic collapse (default) with every kernel; each explicit one
# with two
WIDE = {f"{tree}-{k}": (t, k, None) for t, tree in enumerate(("lbvh", "ploc")) for k in KERNELS}
WIDE.update({f"{tree}-{c}-{k}": (t, k, ci) for t, tree in enumerate(("lbvh", "ploc"))
             for ci, c in enumerate(("greedy", "sah")) for k in ("sorted", "octant")})


@pytest.mark.parametrize("name,make", _scenes()[::2])
def test_wide_collapse_choice(system, name, make):
    """The automatic collapse keeps the layout of which the seeded probe
    rays read fewer bytes, and reports both measures; the explicit choices
    are kept as set."""
    scene = make()
    g = _build(system, scene)
    info = g.wide_collapse()
    b = info["probe_bytes"]
    assert b["largest_area"] > 0 and b["surface_area"] > 0
    assert info["used"] == ("largest_area" if b["largest_area"] < b["surface_area"]
                            else "surface_area")
    for c, name_ in ((0, "largest_area"), (1, "surface_area")):
        assert _build(system, scene, collapse=c).wide_collapse()["used"] == name_


@pytest.mark.parametrize("mode", ["binary"] + list(WIDE))
@pytest.mark.parametrize("name,make", _scenes())
def test_trace_closest_hit(system, cuda, oracle, name, make, mode):
    """binary: the LBVH nodes, bit-exact against the oracle's traversal of
    the same tree.  The 8-wide quantised nodes, collapsed from the LBVH or
    from the PLOC tree by either collapse, with every traversal kernel
    (sorted and octant child order, with and without refilled lanes): same
    hit/miss and the same closest distance bit for bit, same primitive except
    at ties."""
    torch = cuda
    scene = make()
    tree, order, collapse = WIDE.get(mode, (None, None, None))
    g = _build(system, scene, tree, collapse)
    g.set_traversal(0 if tree is None else 1)
    if order is not None:
        g.set_wide_order(order)
    info = g.accel_info()
    if scene.triangle_count > 1:
        assert 0 < info["wide_nodes"] <= scene.triangle_count - 1
        if tree is not None:
            assert info["wide_tree"] == ("ploc" if tree == 1 else "lbvh")
    os_ = oracle.OracleScene.from_scene(scene)
    n = 20000
    rays = _rays_for(scene, n, seed=11)
    key, prim, t, bary = os_.trace(rays)
    ro = _dev(torch, np.ascontiguousarray(rays[:, 0:4]))
    rd = _dev(torch, np.ascontiguousarray(rays[:, 4:8]))
    dk = torch.zeros(n, dtype=torch.int32, device="cuda")
    dp = torch.zeros(n, dtype=torch.int32, device="cuda")
    dt = torch.zeros(n, dtype=torch.float32, device="cuda")
    db = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    g.hit(ro.data_ptr(), rd.data_ptr(), n, dk.data_ptr(), dp.data_ptr(), dt.data_ptr(),
          db.data_ptr())
    torch.cuda.synchronize()
    gk = dk.cpu().numpy().view(np.uint32)
    gp = dp.cpu().numpy().view(np.uint32)
    gt = dt.cpu().numpy()
    gb = db.cpu().numpy()
    hit = prim != 0xFFFFFFFF
    assert hit.sum() > n // 20
    assert np.array_equal(gp != 0xFFFFFFFF, hit)
    assert np.array_equal(gt[hit].view(np.uint32), t[hit].view(np.uint32))
    same = gp == prim
    if mode == "binary":
        assert same.all()
    else:
        assert (~same).sum() <= max(2, n // 1000), f"{(~same).sum()} ties"
    assert np.array_equal(gk[same], key[same])
    assert np.array_equal(gb[same & hit].view(np.uint32), bary[same & hit].view(np.uint32))
    # against the brute-force accelerator: same closest distance everywhere,
    # same primitive except where two triangles report the same distance
    if scene.triangle_count <= 60000:
        m = 4000
        lk, lp, lt, lb = os_.trace(rays[:m], linear=True)
        assert np.array_equal(lp != 0xFFFFFFFF, gp[:m] != 0xFFFFFFFF)
        both = (lp != 0xFFFFFFFF)
        assert np.array_equal(lt[both], gt[:m][both])
        diff = both & (lp != gp[:m])
        assert diff.sum() <= max(2, m // 500), f"{diff.sum()} tie cases"


@pytest.mark.parametrize("n,id_bits", [(1, 1), (1000, 3), (70000, 10), (1 << 20, 10)])
def test_partition_offsets(cuda, oracle, n, id_bits):
    from meturay_b200._lib import check, lib
    torch = cuda
    rng = np.random.default_rng(n)
    batch = rng.integers(0, 5, n).astype(np.uint32)
    ids = rng.integers(0, 1 << id_bits, n).astype(np.uint32)
    keys = (batch << 24) | ids
    keys[batch == 0] = 0
    sk, si, portions = oracle.partition(keys, 3, id_bits)
    dk = _dev(torch, keys.view(np.int32))
    sid = torch.zeros(n, dtype=torch.int32, device="cuda")
    sd = torch.zeros(n, dtype=torch.int32, device="cuda")
    po = torch.zeros(8, dtype=torch.int32, device="cuda")
    pe = torch.zeros(8, dtype=torch.int32, device="cuda")
    nn = torch.zeros(1, dtype=torch.int32, device="cuda")
    tb = lib.mrb_partition_temp_bytes(n, id_bits)
    tmp = torch.zeros(tb, dtype=torch.uint8, device="cuda")
    check(lib.mrb_partition(dk.data_ptr(), n, id_bits, sid.data_ptr(), sd.data_ptr(),
                            po.data_ptr(), pe.data_ptr(), nn.data_ptr(), tmp.data_ptr(), tb, None))
    torch.cuda.synchronize()
    assert np.array_equal(sid.cpu().numpy().view(np.uint32), si)
    po, pe = po.cpu().numpy(), pe.cpu().numpy()
    for b, off, cnt in portions:
        assert po[b] == off and pe[b] - po[b] == cnt, (b, off, cnt, po[b], pe[b])
    present = {b for b, _, _ in portions}
    non_null = dict((b, o) for b, o, _ in portions).get(0, n)
    assert nn.cpu().numpy()[0] == non_null
    for b in range(5):
        if b not in present:
            assert pe[b] == po[b]
