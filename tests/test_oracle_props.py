"""CPU checks of the oracle itself and of the host logic (no GPU).

Philox known-answer vectors, portable math accuracy, sort/partition
semantics against numpy, LBVH invariants (including duplicate codes), the
oracle traversal against brute force, and determinism of the CPU render.
"""
import ctypes as C

import numpy as np
import pytest


def _p(a):
    return C.c_void_p(a.ctypes.data)


@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(oracle, ctr, key, expect):
    out = (C.c_uint32 * 4)()
    oracle.lib.oracle_philox4x32((C.c_uint32 * 4)(*ctr), (C.c_uint32 * 2)(*key), out)
    assert tuple(out) == expect


def test_portable_math_accuracy(oracle):
    s, c = C.c_float(), C.c_float()
    xs = np.linspace(0, 2 * np.pi, 20001, dtype=np.float32)
    err = 0.0
    for x in xs:
        oracle.lib.oracle_sincosf(C.c_float(x), C.byref(s), C.byref(c))
        err = max(err, abs(s.value - np.sin(np.float64(x))), abs(c.value - np.cos(np.float64(x))))
    assert err < 2.5e-7
    ys = np.linspace(-1, 1, 20001, dtype=np.float32)
    ea = max(abs(oracle.lib.oracle_acosf(float(y)) - np.arccos(np.float64(y))) for y in ys)
    assert ea < 5e-7


@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("bits", [(0, 64), (3, 40), (60, 64)])
def test_sort_semantics_against_numpy(oracle, desc, bits):
    rng = np.random.default_rng(1)
    keys = rng.integers(0, 2**63, 5000, dtype=np.uint64)
    keys[:2000] = keys[2000:4000]
    vals = np.arange(5000, dtype=np.uint32)
    k, v = oracle.sort_pairs(keys, vals, bits[0], bits[1], desc)
    mask = np.uint64((1 << (bits[1] - bits[0])) - 1) if bits[1] - bits[0] < 64 else \
        np.uint64(0xFFFFFFFFFFFFFFFF)
    sub = (keys >> np.uint64(bits[0])) & mask
    order = np.argsort(-sub.astype(np.float64) if desc else sub, kind="stable")
    if desc:
        # stable descending: sort by the complemented key
        order = np.argsort(mask - sub, kind="stable")
    assert np.array_equal(v, vals[order])
    assert np.array_equal(k, keys[order])


def test_partition_against_numpy(oracle):
    rng = np.random.default_rng(2)
    batch = rng.integers(0, 5, 10000).astype(np.uint32)
    ids = rng.integers(0, 300, 10000).astype(np.uint32)
    keys = (batch << 24) | ids
    keys[batch == 0] = 0
    sk, si, portions = oracle.partition(keys, 3, 9)
    dense = (batch.astype(np.int64) << 9) | np.where(batch == 0, 0, ids)
    order = np.argsort(-dense, kind="stable")
    assert np.array_equal(si, order)
    assert [b for b, _, _ in portions] == sorted({int(b) for b in batch})
    for b, off, cnt in portions:
        assert np.all(sk[off:off + cnt] >> 24 == b)
    assert sum(c for _, _, c in portions) == 10000


def _check_tree(r, n, aabbs, order):
    left, right, parent, inner, root = r["left"], r["right"], r["parent"], r["inner"], r["root"][0]
    assert parent[root] == 0xFFFFFFFF
    seen = np.zeros(2 * n - 1, np.int32)
    for j in range(n - 1):
        for c in (left[j], right[j]):
            seen[c] += 1
            assert parent[c] == n + j
            box = aabbs[order[c]] if c < n else inner[c - n]
            assert np.all(box[:3] >= inner[j][:3]) and np.all(box[3:] <= inner[j][3:])
    assert seen[root] == 0 and np.all(np.delete(seen, root) == 1)


def test_lbvh_invariants_with_duplicate_codes(oracle):
    from meturay_b200 import scenes
    sc = scenes.cornell(seed=2)   # quad walls: both triangles share one code
    aabbs, ext, delta, codes = oracle.morton_codes(sc.positions, sc.indices)
    order = np.argsort(codes, kind="stable").astype(np.uint32)
    assert len(np.unique(codes)) < len(codes)
    r = oracle.lbvh(codes[order], order, aabbs)
    assert r["status"] == 1   # duplicates reported, tree still built
    _check_tree(r, len(codes), aabbs, order)


def test_oracle_traversal_matches_brute_force(oracle):
    from meturay_b200 import scenes
    sc = scenes.random_triangles(seed=3, n=3000)
    ex = oracle.scene_tables(sc)
    ex["tbn"] = oracle.build_tbn(sc)
    os_ = oracle.OracleScene(sc, ex)
    rng = np.random.default_rng(4)
    n = 3000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-2, 12, (n, 3))
    rays[:, 4:7] = rng.uniform(0, 10, (n, 3)) - rays[:, 0:3]
    rays[:, 7] = 1e30
    k1, p1, t1, _ = os_.trace(rays)
    k2, p2, t2, _ = os_.trace(rays, linear=True)
    hit = p2 != 0xFFFFFFFF
    assert hit.sum() > 100
    assert np.array_equal(p1 != 0xFFFFFFFF, hit)
    assert np.array_equal(t1[hit], t2[hit])
    assert (p1 != p2).sum() <= 3


def test_cpu_render_is_deterministic_and_fp64_close(oracle):
    from meturay_b200 import scenes
    import bench
    sc = scenes.cornell(seed=1, width=16, height=16)
    ex = oracle.scene_tables(sc)
    ex["tbn"] = oracle.build_tbn(sc)
    os_ = oracle.OracleScene(sc, ex)
    cf = bench._camera16(sc)
    a, ra = os_.render(cf, 16, 16, 2, 5, 3, True, 9)
    b, rb = os_.render(cf, 16, 16, 2, 5, 3, True, 9, threads=1)
    assert ra == rb and np.array_equal(a, b)
    d, rd = os_.render(cf, 16, 16, 2, 5, 3, True, 9, fp64=True)
    assert a.sum() > 0 and np.isfinite(d).all()
    # same RNG stream; paths only part after precision-sensitive events
    assert abs(a.sum() - d.sum()) / d.sum() < 0.2


def _probe(oracle, name, vals, nout):
    import ctypes as C
    a = np.ascontiguousarray(vals, np.float32)
    o = np.zeros(nout, np.float32)
    assert oracle.lib.oracle_probe(name.encode(), a.ctypes.data_as(C.c_void_p),
                                   o.ctypes.data_as(C.c_void_p)) == 0
    return o


def test_half_conversion_is_ieee_round_to_nearest_even(oracle):
    """The guide words and radiance averages use a portable binary16
    conversion; it must equal IEEE round-to-nearest-even (numpy float16)."""
    rng = np.random.default_rng(5)
    xs = np.concatenate([
        rng.standard_normal(2000).astype(np.float32) * 10.0,
        (rng.random(2000) * 7e4).astype(np.float32),
        (rng.random(500) * 1e-4).astype(np.float32),            # subnormal halves
        np.array([0.0, -0.0, 65504.0, 65519.0, 65520.0, 1e9, 6e-8, 3e-8, 2.0 ** -25,
                  2.0 ** -24, 1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11], np.float32)])
    for x in xs:
        o = _probe(oracle, "half", [x], 2)
        with np.errstate(over="ignore"):
            ref = np.float32(np.float16(x))
        assert o[0] == ref or (np.isinf(ref) and np.isinf(o[0])), (x, o[0], ref)


def test_octahedral_map_round_trip(oracle):
    """Co-centric octahedral map (CoordinateConversion.h:112-183): direction
    -> (s, t) in [0,1]^2 -> the same direction."""
    rng = np.random.default_rng(6)
    d = rng.standard_normal((500, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    for v in d.astype(np.float32):
        o = _probe(oracle, "octa", v, 5)
        assert 0.0 <= o[0] <= 1.0 and 0.0 <= o[1] <= 1.0
        assert np.abs(o[2:5] - v).max() < 2e-6, (v, o)


def test_octahedral_int_wrap_mirrors_edges(oracle):
    """CocentricOctohedralWrapInt: stepping over an edge mirrors the other
    coordinate, a corner step goes to the opposite corner; in-range texels
    are unchanged."""
    X = 64
    for x, y, ex, ey in [(-1, 10, 0, 53), (64, 10, 63, 53), (10, -1, 53, 0), (10, 64, 53, 63),
                         (5, 7, 5, 7), (-3, -2, 61, 62)]:
        o = _probe(oracle, "octa_wrap_int", [x, y, X], 2)
        assert (int(o[0]), int(o[1])) == (ex, ey), (x, y, o)


def test_oracle_wfpg_is_deterministic_and_deposits(oracle):
    """Two oracle WFPG frames from identical caches agree bit for bit; the
    frame deposits one sample per path vertex into the cache."""
    from meturay_b200 import camera_frame, scenes
    sc = scenes.cornell(seed=6, width=16, height=16, mixed=True)
    ex = oracle.scene_tables(sc)
    ex["tbn"] = oracle.build_tbn(sc)
    os_ = oracle.OracleScene(sc, ex)
    ext = np.concatenate([sc.positions.min(0), sc.positions.max(0)]).astype(np.float32)
    cf = np.concatenate([camera_frame(sc.camera), np.float32(sc.camera["near_far"])])
    outs = []
    for _ in range(2):
        svo = oracle.OracleSvo(sc, ex["tri_key"], ext, 32, ex["light_radiance"])
        before = svo.export()
        img, rays, dg, db = os_.render_wfpg(cf, 16, 16, 1, 4, 3, True, 9, svo, min_bin_level=2,
                                            bin_ray_count=16, dump_iteration=0)
        after = svo.export()
        outs.append((img, rays, dg, db, after))
    a, b = outs
    assert np.array_equal(a[0], b[0]) and a[1] == b[1]
    assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
    for k in ("leaf_irr", "leaf_cnt", "leaf_avg", "node_avg"):
        assert np.array_equal(a[4][k], b[4][k])
    deposits = int(a[4]["leaf_cnt"].sum() - before["leaf_cnt"].sum())
    assert 0 < deposits <= 16 * 16 * 4
    guided = (a[2][:, 1] >> 17) & 1
    assert guided.sum() > 0 and np.all(a[3][guided == 1] != 0xFFFFFFFF)
