"""The accelerator-group and base-accelerator entry points, driven the way
MRay's RayCasterCUDA::HitRays drives GPUAcceleratorGroupI::Hit and
GPUBaseAcceleratorI::Hit (RayCasterCUDA.cu:35-166): RayGMem rays through a
RayId permutation, accelerator keys from the base accelerator, tMax updated
in place, 64-bit primitive ids.

* A one-surface identity group equals mrb_accel_hit (the scene's binary
  LBVH over the same triangles) bit for bit, whatever the ray-id order.
* Surfaces under rotations, scales and translations, traced through the
  base accelerator's resumable traversal until it hands out no more keys:
  the same closest distance as the oracle's two-level traversal bit for bit,
  the same key, transform, primitive and barycentrics except at ties.
* AcceleratorAABBs, TotalPrimitiveCount, TotalApproximateArea,
  SampleAreaWeightedPoints, EachPrimVoxelCount and VoxelizeSurfaces against
  the oracle.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _rigid(rng, scale=True):
    """A random rotation (times a scale) plus translation, row-major 3x4."""
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    s = np.diag(rng.uniform(0.5, 2.0, 3)) if scale else np.eye(3)
    m = np.zeros((3, 4))
    m[:, :3] = q @ s
    m[:, 3] = rng.uniform(-3, 3, 3)
    return m.astype(np.float32).reshape(12)


def _multi_surface_scene(seed):
    """Five surfaces: the Cornell walls (identity) and four spheres of the
    Cornell generator, each in its own local frame."""
    from meturay_b200 import scenes
    rng = np.random.default_rng(seed)
    sc = scenes.cornell(seed=seed)
    pos, idx = sc.positions.astype(np.float32), sc.indices.astype(np.uint32)
    T = idx.shape[0]
    cuts = [0, 12] + sorted(rng.choice(np.arange(13, T - 1), 3, replace=False).tolist()) + [T]
    surfaces = np.array([[cuts[i], cuts[i + 1], i] for i in range(5)], np.uint32)
    l2w = [np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32)]
    for i in range(1, 5):
        l2w.append(_rigid(rng, scale=(i % 2 == 0)))
    keys = (np.uint32(1) << np.uint32(24)) | (np.arange(T, dtype=np.uint32) % 7)
    return pos, idx, keys, surfaces, np.stack(l2w)


def _group(lib, check, system, pos, idx, keys, surfaces, l2w=None, tbn=None):
    g = C.c_void_p()
    surf = np.ascontiguousarray(surfaces, np.uint32)
    check(lib.mrb_accel_group_create(system._h, pos.ctypes.data, pos.shape[0],
                                     None if tbn is None else tbn.ctypes.data, idx.ctypes.data,
                                     keys.ctypes.data, None, None, idx.shape[0], surf.ctypes.data,
                                     surf.shape[0], C.byref(g)))
    if l2w is not None:
        m = np.ascontiguousarray(l2w, np.float32)
        check(lib.mrb_accel_group_attach_transforms(g, m.ctypes.data, m.shape[0], 0))
    check(lib.mrb_accel_group_construct(g, None))
    return g


def _rays(pos, n, seed):
    rng = np.random.default_rng(seed)
    lo, hi = pos.min(0), pos.max(0)
    span = hi - lo
    o = lo - 0.3 * span + rng.uniform(size=(n, 3)) * 1.6 * span
    tgt = lo + rng.uniform(size=(n, 3)) * span
    d = tgt - o
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 4:7] = d
    rays[:, 7] = 3.0e38
    rays[::9, 7] = 0.7
    rays[1::13, 3] = 0.2
    return rays


def _group_hit(torch, lib, check, g, rays, ids, keys):
    n = rays.shape[0]
    dr = _dev(torch, rays)
    mk = torch.zeros(n, dtype=torch.int32, device="cuda")
    tid = torch.zeros(n, dtype=torch.int32, device="cuda")
    pid = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    hs = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    di, dk = _dev(torch, ids.view(np.int32)), _dev(torch, keys.view(np.int32))
    check(lib.mrb_accel_group_hit(g, _ptr(mk), _ptr(tid), _ptr(pid), _ptr(hs), 8, _ptr(dr),
                                  _ptr(di), _ptr(dk), len(ids), None))
    torch.cuda.synchronize()
    return (dr.cpu().numpy(), mk.cpu().numpy().view(np.uint32), tid.cpu().numpy().view(np.uint32),
            pid.cpu().numpy().view(np.uint64), hs.cpu().numpy())


def test_single_surface_group_equals_accel_hit(system, cuda, oracle):
    from meturay_b200 import GPUScene, scenes
    from meturay_b200._lib import check, lib
    torch = cuda
    sc = scenes.clusters(seed=2, n_clusters=40, tris_per_cluster=500)
    g = GPUScene(system, sc)
    g.construct_accelerators()
    g.set_traversal(0)
    ex = oracle.scene_tables(sc)
    pos, idx = sc.positions.astype(np.float32), sc.indices.astype(np.uint32)
    T = idx.shape[0]
    grp = _group(lib, check, system, pos, idx, ex["tri_key"], [[0, T, 0]])
    n = 30000
    rays = _rays(pos, n, 3)
    # reference path: the scene's binary LBVH
    ro, rd = _dev(torch, rays[:, 0:4]), _dev(torch, rays[:, 4:8])
    k = torch.zeros(n, dtype=torch.int32, device="cuda")
    p = torch.zeros(n, dtype=torch.int32, device="cuda")
    t = torch.zeros(n, dtype=torch.float32, device="cuda")
    b = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    g.hit(ro.data_ptr(), rd.data_ptr(), n, k.data_ptr(), p.data_ptr(), t.data_ptr(), b.data_ptr())
    torch.cuda.synchronize()
    k, p = k.cpu().numpy().view(np.uint32), p.cpu().numpy().view(np.uint32)
    t, b = t.cpu().numpy(), b.cpu().numpy()
    # group path: a RayId permutation and the surface's accelerator key
    perm = np.random.default_rng(4).permutation(n).astype(np.uint32)
    keys = np.full(n, (2 << 24) | 0, np.uint32)
    out, mk, tid, pid, hs = _group_hit(torch, lib, check, grp, rays, perm, keys)
    hit = p != 0xFFFFFFFF
    assert hit.sum() > n // 10
    assert np.array_equal(out[:, 7].view(np.uint32)[hit], t.view(np.uint32)[hit])
    assert np.array_equal(out[~hit, 7], rays[~hit, 7])  # misses keep their tMax
    assert np.array_equal(pid[hit], p[hit].astype(np.uint64))
    assert np.all(pid[~hit] == np.uint64(0xFFFFFFFFFFFFFFFF))
    assert np.array_equal(mk[hit], k[hit])
    assert np.array_equal(hs[hit].view(np.uint32), b[hit].view(np.uint32))
    assert np.all(tid[hit] == 0)
    assert lib.mrb_accel_group_primitive_count(grp) == T
    assert lib.mrb_accel_group_accelerator_count(grp) == 1
    lib.mrb_accel_group_destroy(grp)
    g.set_traversal(1)


def test_transformed_surfaces_through_the_base_accelerator(system, cuda, oracle):
    from meturay_b200._lib import check, lib
    torch = cuda
    pos, idx, keys, surfaces, l2w = _multi_surface_scene(7)
    grp = _group(lib, check, system, pos, idx, keys, surfaces, l2w)
    S = surfaces.shape[0]
    aabbs = np.zeros((S, 6), np.float32)
    assert lib.mrb_accel_group_aabbs(grp, aabbs.ctypes.data, S) == S
    og = oracle.OracleGroup(pos, idx, keys, surfaces, l2w)
    assert og.status == 0
    assert np.array_equal(aabbs, og.aabbs())
    base = C.c_void_p()
    check(lib.mrb_base_accel_create(system._h, C.byref(base)))
    acc_keys = ((3 << 24) | np.arange(S)).astype(np.uint32)
    check(lib.mrb_base_accel_construct(base, aabbs.ctypes.data, acc_keys.ctypes.data, S))
    ext = np.zeros(6, np.float32)
    check(lib.mrb_base_accel_extents(base, ext.ctypes.data))
    assert np.array_equal(ext[:3], aabbs[:, :3].min(0)) and np.array_equal(ext[3:], aabbs[:, 3:].max(0))
    # world rays over the transformed scene
    wl, wh = aabbs[:, :3].min(0), aabbs[:, 3:].max(0)
    rng = np.random.default_rng(8)
    n = 40000
    o = wl - 0.3 * (wh - wl) + rng.uniform(size=(n, 3)) * 1.6 * (wh - wl)
    d = (wl + rng.uniform(size=(n, 3)) * (wh - wl)) - o
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 4:7], rays[:, 7] = o, d, 3.0e38
    ids = np.random.default_rng(9).permutation(n).astype(np.uint32)
    # the ray caster's loop: base hit, then the group hit on the rays that
    # got a key, until the base accelerator hands out none
    dr = _dev(torch, rays)
    mk = torch.zeros(n, dtype=torch.int32, device="cuda")
    tid = torch.zeros(n, dtype=torch.int32, device="cuda")
    pid = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    hs = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    check(lib.mrb_base_accel_get_ready(base, n, None))
    live = ids
    rounds = 0
    while live.size:
        dl = _dev(torch, live.view(np.int32))
        dk = torch.zeros(live.size, dtype=torch.int32, device="cuda")
        check(lib.mrb_base_accel_hit(base, _ptr(dk), _ptr(dr), _ptr(dl), live.size, None))
        torch.cuda.synchronize()
        k = dk.cpu().numpy().view(np.uint32)
        act = k != 0
        live, k = live[act], k[act]
        if live.size:
            # both device arrays stay referenced until the kernel has run (a
            # freed tensor's memory can be handed to the next allocation)
            d_ids = _dev(torch, live.view(np.int32))
            d_keys = _dev(torch, k.view(np.int32))
            check(lib.mrb_accel_group_hit(grp, _ptr(mk), _ptr(tid), _ptr(pid), _ptr(hs), 8,
                                          _ptr(dr), _ptr(d_ids), _ptr(d_keys), live.size, None))
            torch.cuda.synchronize()
            del d_ids, d_keys
        rounds += 1
        assert rounds <= S + 1
    torch.cuda.synchronize()
    out = dr.cpu().numpy()
    mk, tid = mk.cpu().numpy().view(np.uint32), tid.cpu().numpy().view(np.uint32)
    pid, hs = pid.cpu().numpy().view(np.uint64), hs.cpu().numpy()
    ref = og.trace(rays)
    hit = ref["prim"] != np.uint64(0xFFFFFFFFFFFFFFFF)
    assert hit.sum() > n // 10
    assert np.array_equal(pid != np.uint64(0xFFFFFFFFFFFFFFFF), hit)
    assert np.array_equal(out[:, 7].view(np.uint32), ref["t"].view(np.uint32))
    same = hit & (pid == ref["prim"])
    assert (hit & ~same).sum() <= max(2, n // 1000)
    assert np.array_equal(mk[same], ref["key"][same])
    assert np.array_equal(tid[same], ref["transform"][same])
    assert np.array_equal(hs[same].view(np.uint32), ref["bary"][same].view(np.uint32))
    assert len(np.unique(tid[hit])) == S          # every surface was hit somewhere
    lib.mrb_base_accel_destroy(base)
    lib.mrb_accel_group_destroy(grp)


def _world_positions(pos, idx, surfaces, l2w):
    """Vertices of every triangle in world space, per triangle (3 per
    triangle), summed in the order of the library's affine product."""
    f32 = np.float32
    out = np.zeros((idx.shape[0], 3, 3), f32)
    for b, e, t in surfaces:
        m = l2w[t].astype(f32)
        p = pos[idx[b:e]].astype(f32)
        for r in range(3):
            out[b:e, :, r] = ((m[4 * r] * p[..., 0] + m[4 * r + 1] * p[..., 1])
                              + m[4 * r + 2] * p[..., 2]) + m[4 * r + 3]
    return out


def test_group_area_sampling_and_voxelisation(system, cuda, oracle):
    from meturay_b200._lib import check, lib
    torch = cuda
    pos, idx, keys, surfaces, l2w = _multi_surface_scene(11)
    keys[:12] = (4 << 24) | np.arange(12, dtype=np.uint32)  # the walls are lights
    grp = _group(lib, check, system, pos, idx, keys, surfaces, l2w)
    T = idx.shape[0]
    wp = _world_positions(pos, idx, surfaces, l2w).astype(np.float64)
    area_ref = 0.5 * np.linalg.norm(np.cross(wp[:, 1] - wp[:, 0], wp[:, 2] - wp[:, 0]), axis=1)
    area = C.c_float()
    check(lib.mrb_accel_group_total_area(grp, C.byref(area), None))
    assert abs(area.value - area_ref.sum()) <= 1e-5 * area_ref.sum()
    # area-weighted points: on the world surfaces, spread over the surfaces
    # in proportion to their areas, unit normals
    m = 200000
    dp = torch.zeros((m, 3), dtype=torch.float32, device="cuda")
    dn = torch.zeros((m, 3), dtype=torch.float32, device="cuda")
    check(lib.mrb_accel_group_sample_points(grp, _ptr(dp), _ptr(dn), m, 1234, None))
    P, N = dp.cpu().numpy().astype(np.float64), dn.cpu().numpy().astype(np.float64)
    assert np.abs(np.linalg.norm(N, axis=1) - 1.0).max() < 1e-5
    aab = np.zeros((surfaces.shape[0], 6), np.float32)
    lib.mrb_accel_group_aabbs(grp, aab.ctypes.data, surfaces.shape[0])
    surf_area = np.array([area_ref[b:e].sum() for b, e, _ in surfaces])
    for s, (b, e, _) in enumerate(surfaces):
        inside = np.all((P >= aab[s, :3] - 1e-4) & (P <= aab[s, 3:] + 1e-4), axis=1)
        expect = m * surf_area[s] / surf_area.sum()
        assert inside.sum() >= expect - 5 * np.sqrt(expect)
    # EachPrimVoxelCount / VoxelizeSurfaces: the oracle's voxeliser over the
    # same world-space vertices
    res = 128
    # the octree box of Constrcut (AnisoSVO.cu:670-679) from the scene
    # extent, in float32 steps
    ext = np.concatenate([aab[:, :3].min(0), aab[:, 3:].max(0)]).astype(np.float32)
    world = (ext[3:] - ext[:3]).max()
    pad = np.float32(world / np.float32(res))
    box = np.concatenate([ext[:3] - pad, ext[:3] + (pad + world)]).astype(np.float32)
    dc = torch.zeros(T, dtype=torch.int64, device="cuda")
    check(lib.mrb_accel_group_voxel_counts(grp, _ptr(dc), res, box.ctypes.data, None))
    torch.cuda.synchronize()
    counts = dc.cpu().numpy().view(np.uint64)
    wpos = _world_positions(pos, idx, surfaces, l2w).reshape(-1, 3)
    widx = np.arange(3 * T, dtype=np.uint32).reshape(T, 3)
    oc, ocodes, onormals = oracle.voxelize(wpos, widx, ext, res)
    assert np.array_equal(counts, oc)
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint64)
    nv = int(offs[-1])
    dv = torch.zeros(nv, dtype=torch.int64, device="cuda")
    dnrm = torch.zeros(nv, dtype=torch.int32, device="cuda")
    dl = torch.zeros(nv, dtype=torch.int32, device="cuda")
    lights = np.sort(keys[:12]).astype(np.uint32)
    d_offs = _dev(torch, offs.view(np.int64))
    d_lights = _dev(torch, lights.view(np.int32))
    check(lib.mrb_accel_group_voxelize(grp, _ptr(dv), _ptr(dnrm), _ptr(dl), _ptr(d_offs),
                                       _ptr(d_lights), 12, res, box.ctypes.data, None))
    torch.cuda.synchronize()
    assert np.array_equal(dv.cpu().numpy().view(np.uint64), ocodes)
    assert np.array_equal(dnrm.cpu().numpy().view(np.uint32), onormals)
    lk = dl.cpu().numpy().view(np.uint32)
    tri_of = np.repeat(np.arange(T), counts.astype(np.int64))
    assert np.array_equal(lk, np.where(tri_of < 12, keys[tri_of], 0).astype(np.uint32))
    lib.mrb_accel_group_destroy(grp)
