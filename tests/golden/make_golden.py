"""Generate golden vectors from the MRay reference's own code.

Runs the reference routines compiled by ``make -C oracle ref`` into
``oracle/_ref/libmrayref.so`` (MRay headers #included from the reference
tree; LBVH kernels cut from LinearBVH.hpp and the octree kernels cut from
AnisoSVO.cu at build time) on seeded random inputs and stores inputs +
outputs in ``tests/golden/reference_vectors.npz`` and (octree: voxelizer,
level build, ray bins, cone traces) ``tests/golden/svo_reference_vectors.npz``.
The CPU oracle is then checked against these vectors by
``tests/test_oracle_golden.py``; the reference tree is not needed at test
time.

    python tests/golden/make_golden.py REF_ROOT     (or REF_ROOT=... in the environment)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = HERE / "reference_vectors.npz"


def _p(a):
    return C.c_void_p(a.ctypes.data)


def main(ref_root: str | None = None) -> None:
    ref_root = ref_root or os.environ.get("REF_ROOT")
    if not ref_root:
        sys.exit("make_golden: pass the MRay source tree as REF_ROOT (argument or environment)")
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "ref", f"REF_ROOT={ref_root}"],
                   check=True)
    R = C.CDLL(str(ROOT / "oracle" / "_ref" / "libmrayref.so"))
    for name in ("ref_dggx", "ref_gsmith_corr", "ref_gsmith_single", "ref_fresnel_dielectric",
                 "ref_vndf_pdf", "ref_power_heuristic"):
        getattr(R, name).restype = C.c_float
    R.ref_morton3d.restype = C.c_uint64
    rng = np.random.default_rng(20261203)
    f32 = np.float32
    g: dict[str, np.ndarray] = {}

    def unit(n):
        v = rng.normal(size=(n, 3))
        return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(f32)

    def quat(n):
        q = rng.normal(size=(n, 4))
        return (q / np.linalg.norm(q, axis=1, keepdims=True)).astype(f32)

    # --- MortonCode::Compose3D (MortonCode.h:150-158)
    xyz = rng.integers(0, 1 << 21, size=(1500, 3), dtype=np.uint32)
    xyz[:8] = [[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [(1 << 21) - 1] * 3,
               [1 << 21, 0, 0], [5, 9, 3], [123456, 654321, 2097151]]
    g["morton3d_in"] = xyz
    g["morton3d_out"] = np.array([R.ref_morton3d(*map(int, r)) for r in xyz], np.uint64)

    # --- KCGenMortonCodes body over AABB centroids
    n = 2000
    c = rng.uniform(-3, 7, (n, 3)).astype(f32)
    h = rng.uniform(0, 0.05, (n, 3)).astype(f32)
    aabb = np.concatenate([c - h, c + h], 1).astype(f32)
    ext = np.concatenate([aabb[:, :3].min(0), aabb[:, 3:].max(0)]).astype(f32)
    delta = f32(max(float(f32(ext[3 + i] - ext[i])) * (1.0 / (1 << 21)) for i in range(3)))
    codes = np.zeros(n, np.uint64)
    R.ref_morton_codes(_p(aabb), C.c_uint32(n), _p(ext), C.c_float(delta), _p(codes))
    g["morton_aabb"], g["morton_extent"], g["morton_delta"] = aabb, ext, np.array([delta], f32)
    g["morton_codes"] = codes

    # --- LBVH hierarchy + AABBs (LinearBVH.hpp:30-100,181-246,290-363)
    for tag, n in (("lbvh2", 2), ("lbvh3", 3), ("lbvh257", 257), ("lbvh2000", 2000)):
        cc = rng.uniform(0, 10, (n, 3)).astype(f32)
        la = np.concatenate([cc - 0.01, cc + 0.01], 1).astype(f32)
        e = np.concatenate([la[:, :3].min(0), la[:, 3:].max(0)]).astype(f32)
        dl = f32(max(float(f32(e[3 + i] - e[i])) * (1.0 / (1 << 21)) for i in range(3)))
        cd = np.zeros(n, np.uint64)
        R.ref_morton_codes(_p(la), C.c_uint32(n), _p(e), C.c_float(dl), _p(cd))
        assert len(np.unique(cd)) == n, "reference LBVH needs unique codes"
        order = np.argsort(cd, kind="stable").astype(np.uint32)
        sc = np.ascontiguousarray(cd[order])
        L = np.zeros(n - 1, np.uint32)
        Rr = np.zeros(n - 1, np.uint32)
        P = np.zeros(2 * n - 1, np.uint32)
        inner = np.zeros((n - 1, 6), f32)
        root = np.zeros(1, np.uint32)
        st = R.ref_lbvh(_p(sc), _p(order), _p(la), C.c_uint32(n), _p(L), _p(Rr), _p(P),
                        _p(inner), _p(root))
        assert st == 0
        g[f"{tag}_codes"], g[f"{tag}_order"], g[f"{tag}_leaf_aabb"] = sc, order, la
        g[f"{tag}_left"], g[f"{tag}_right"], g[f"{tag}_parent"] = L, Rr, P
        g[f"{tag}_inner"], g[f"{tag}_root"] = inner, root

    # --- Ray::IntersectsTriangle (Ray.hpp:143-184)
    n = 4000
    ro = rng.normal(size=(n, 3)).astype(f32)
    rd = rng.normal(size=(n, 3)).astype(f32)
    tri = (ro[:, None, :] + rd[:, None, :] * rng.uniform(0.5, 3, (n, 1, 1))
           + rng.normal(size=(n, 3, 3)) * 0.5).astype(f32)
    cull = (rng.uniform(size=n) < 0.3).astype(np.int32)
    hit = np.zeros(n, np.int32)
    tt = np.zeros(n, f32)
    bary = np.zeros((n, 3), f32)
    for i in range(n):
        t1 = np.zeros(1, f32)
        b1 = np.zeros(3, f32)
        v0, v1, v2 = (np.ascontiguousarray(tri[i, k]) for k in range(3))
        hit[i] = R.ref_intersect_tri(_p(ro[i]), _p(rd[i]), _p(v0), _p(v1), _p(v2), int(cull[i]),
                                     _p(t1), _p(b1))
        tt[i], bary[i] = t1[0], b1
    g.update(tri_ro=ro, tri_rd=rd, tri_p=tri, tri_cull=cull, tri_hit=hit, tri_t=tt, tri_bary=bary)

    # --- Ray::Nudge (Ray.hpp:503-556)
    n = 2000
    pos = (rng.normal(size=(n, 3)) * rng.choice([0.001, 0.02, 1.0, 100.0], (n, 1))).astype(f32)
    dirs = unit(n)
    outp = np.zeros((n, 3), f32)
    for i in range(n):
        o = np.zeros(3, f32)
        R.ref_nudge(_p(pos[i]), _p(dirs[i]), _p(o))
        outp[i] = o
    g.update(nudge_pos=pos, nudge_dir=dirs, nudge_out=outp)

    # --- Ray::Reflect / Ray::Refract (Ray.hpp:302-356)
    n = 1500
    d, nn = unit(n), unit(n)
    ior = rng.uniform(1.0, 2.0, (n, 2)).astype(f32)
    refl = np.zeros((n, 3), f32)
    refr = np.zeros((n, 3), f32)
    ok = np.zeros(n, np.int32)
    for i in range(n):
        o = np.zeros(3, f32)
        R.ref_reflect(_p(d[i]), _p(nn[i]), _p(o))
        refl[i] = o
        o = np.zeros(3, f32)
        ok[i] = R.ref_refract(_p(d[i]), _p(nn[i]), C.c_float(ior[i, 0]), C.c_float(ior[i, 1]), _p(o))
        refr[i] = o
    g.update(rr_d=d, rr_n=nn, rr_ior=ior, reflect_out=refl, refract_ok=ok, refract_out=refr)

    # --- HemiDistribution::HemiCosineCDF (HemiDistribution.h:10-30)
    n = 1500
    xi = rng.uniform(size=(n, 2)).astype(f32)
    hd = np.zeros((n, 3), f32)
    hp = np.zeros(n, f32)
    for i in range(n):
        o = np.zeros(3, f32)
        p = C.c_float()
        R.ref_hemi_cosine(_p(xi[i]), _p(o), C.byref(p))
        hd[i], hp[i] = o, p.value
    g.update(hemi_xi=xi, hemi_dir=hd, hemi_pdf=hp)

    # --- Quaternion ops (Quaternion.hpp:76-89,229-318,372-480)
    n = 1500
    q0 = quat(n)
    q1 = (q0 + rng.normal(size=(n, 4)) * 0.2).astype(f32)
    q2 = (q0 + rng.normal(size=(n, 4)) * 0.2).astype(f32)
    ab = rng.uniform(size=(n, 2)).astype(f32)
    flip = ab.sum(1) > 1
    ab[flip] = 1 - ab[flip]
    ab[:10] = [[0, 0], [1, 0], [0, 1], [0.5, 0.5], [1e-7, 1e-7], [0.3, 0], [0, 0.3],
               [0.999, 0.0005], [0.2, 0.2], [0.5, 0.25]]
    sl = np.zeros((n, 4), f32)
    rot = np.zeros((n, 3), f32)
    mul = np.zeros((n, 4), f32)
    vv = rng.normal(size=(n, 3)).astype(f32)
    for i in range(n):
        o = np.zeros(4, f32)
        a1, a2 = np.ascontiguousarray(q1[i]), np.ascontiguousarray(q2[i])
        R.ref_bary_slerp(_p(q0[i]), _p(a1), _p(a2), C.c_float(ab[i, 0]), C.c_float(ab[i, 1]),
                         _p(o))
        sl[i] = o
        o3 = np.zeros(3, f32)
        R.ref_quat_rotate(_p(q0[i]), _p(vv[i]), _p(o3))
        rot[i] = o3
        o = np.zeros(4, f32)
        R.ref_quat_mul(_p(q0[i]), _p(a1), _p(o))
        mul[i] = o
    g.update(q_q0=q0, q_q1=q1, q_q2=q2, q_ab=ab, q_slerp=sl, q_v=vv, q_rot=rot, q_mul=mul)

    # --- Tangent space of a mesh (GPUPrimitiveTriangle.cpp:160-320): the
    # loader loop composed from the reference's CalculateTangent,
    # OrthogonalVector and TransformGen::Space.
    sys.path.insert(0, str(ROOT))
    from meturay_b200.scenes import uv_sphere
    pos, nrm, uv, idx = uv_sphere((0.3, -0.2, 0.5), 0.7, 16, 8)
    qt = np.zeros((pos.shape[0], 4), f32)
    tan = np.zeros((pos.shape[0], 3), f32)
    for tri_ in idx:
        for k in range(3):
            a, b, c = tri_[k], tri_[(k + 1) % 3], tri_[(k + 2) % 3]
            o = np.zeros(3, f32)
            R.ref_calc_tangent(_p(pos[a]), _p(pos[b]), _p(pos[c]), _p(uv[a]), _p(uv[b]),
                               _p(uv[c]), _p(nrm[a]), _p(o))
            if np.isnan(o).any():
                R.ref_orthogonal(_p(nrm[a]), _p(o))
            tan[a] = (tan[a] + o).astype(f32)
    for vix in range(pos.shape[0]):
        n_, t_ = nrm[vix], tan[vix].copy()
        if f32(t_[0] * t_[0] + t_[1] * t_[1] + t_[2] * t_[2]) < f32(1e-5):
            R.ref_orthogonal(_p(n_), _p(t_))
        inv = f32(1) / np.sqrt(f32(t_[0] * t_[0] + t_[1] * t_[1] + t_[2] * t_[2]), dtype=f32)
        t_ = (t_ * inv).astype(f32)
        dt = f32(n_[0] * t_[0] + n_[1] * t_[1] + n_[2] * t_[2])
        x = (t_ - n_ * dt).astype(f32)
        inv = f32(1) / np.sqrt(f32(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]), dtype=f32)
        x = (x * inv).astype(f32)
        y = np.array([n_[1] * x[2] - n_[2] * x[1], n_[2] * x[0] - n_[0] * x[2],
                      n_[0] * x[1] - n_[1] * x[0]], f32)
        o = np.zeros(4, f32)
        zc = np.ascontiguousarray(n_)
        R.ref_space(_p(x), _p(y), _p(zc), _p(o))
        qt[vix] = o
    g.update(tbn_pos=pos, tbn_nrm=nrm, tbn_uv=uv, tbn_idx=idx, tbn_out=qt)

    # --- TracerFunctions.cuh: GGX / Fresnel / VNDF / MIS
    n = 1500
    ndh = rng.uniform(0, 1, n).astype(f32)
    alpha = rng.uniform(0.0025, 0.64, n).astype(f32)
    g["dggx_in"] = np.stack([ndh, alpha], 1)
    g["dggx_out"] = np.array([R.ref_dggx(C.c_float(a), C.c_float(b)) for a, b in zip(ndh, alpha)],
                             f32)
    wo, wi = unit(n), unit(n)
    wo[:, 2], wi[:, 2] = np.abs(wo[:, 2]) + 0.01, np.abs(wi[:, 2]) + 0.01
    g["gs_wo"], g["gs_wi"], g["gs_alpha"] = wo, wi, alpha
    g["gs_corr"] = np.array([R.ref_gsmith_corr(_p(wo[i]), _p(wi[i]), C.c_float(alpha[i]))
                             for i in range(n)], f32)
    g["gs_single"] = np.array([R.ref_gsmith_single(_p(wo[i]), C.c_float(alpha[i]))
                               for i in range(n)], f32)
    cosv = rng.uniform(0, 1, n).astype(f32)
    eta = rng.uniform(1.0, 50.0, (n, 3)).astype(f32)
    kk = np.where(rng.uniform(size=(n, 1)) < 0.5, 0, rng.uniform(0, 5, (n, 3))).astype(f32)
    fc = np.zeros((n, 3), f32)
    for i in range(n):
        o = np.zeros(3, f32)
        R.ref_fresnel_conductor(C.c_float(cosv[i]), _p(eta[i]), _p(kk[i]), _p(o))
        fc[i] = o
    g.update(fc_cos=cosv, fc_eta=eta, fc_k=kk, fc_out=fc)
    ior2 = rng.uniform(1.0, 2.0, (n, 2)).astype(f32)
    g["fd_in"] = np.stack([cosv, ior2[:, 0], ior2[:, 1]], 1).astype(f32)
    g["fd_out"] = np.array([R.ref_fresnel_dielectric(C.c_float(a), C.c_float(b), C.c_float(c))
                            for a, b, c in g["fd_in"]], f32)
    vx = rng.uniform(size=(n, 2)).astype(f32)
    vh = np.zeros((n, 3), f32)
    vp = np.zeros(n, f32)
    for i in range(n):
        o = np.zeros(3, f32)
        p = C.c_float()
        R.ref_vndf_sample(_p(wo[i]), C.c_float(alpha[i]), _p(vx[i]), _p(o), C.byref(p))
        vh[i], vp[i] = o, p.value
    g.update(vndf_v=wo, vndf_alpha=alpha, vndf_xi=vx, vndf_h=vh, vndf_pdf=vp)
    g["vndfpdf_out"] = np.array([R.ref_vndf_pdf(_p(wo[i]), _p(wi[i]), C.c_float(alpha[i]))
                                 for i in range(n)], f32)
    ph = rng.uniform(0, 5, (n, 4)).astype(f32)
    g["ph_in"] = ph
    g["ph_out"] = np.array([R.ref_power_heuristic(*[C.c_float(x) for x in r]) for r in ph], f32)

    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT} ({OUT.stat().st_size / 1024:.0f} KiB, {len(g)} arrays)")
    svo_golden(R)


def _scenes():
    """The seeded scene generator, loaded from its file alone."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("mrb_scenes_standalone",
                                                  ROOT / "meturay_b200" / "scenes.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def svo_golden(R) -> None:
    """Octree vectors from the reference's own code (oracle/ref_svo.cpp):
    TriFunctions::Voxelize, the Constrcut level kernels, ray binning with
    collapse, ConeTraceRay + ReadRadiance, KCAverageNormals,
    NormalizeAndFilterRadiance and DepositRadiance, on two seeded scenes.
    The cones and the normal averaging read the oracle's payload (leaf normal
    words from KCReduceVoxelPayload, half2 averages after the filters), stored
    beside them as input."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as o
    scenes = _scenes()
    R.ref_svo_voxelize.restype = C.c_int64
    R.ref_svo_build.restype = C.c_void_p
    g: dict[str, np.ndarray] = {}
    rng = np.random.default_rng(20261204)
    cases = (("cornell64", scenes.cornell(seed=1), 64),
             ("clusters128", scenes.clusters(seed=3, n_clusters=8, tris_per_cluster=300), 128))
    for tag, scene, res in cases:
        pos = np.ascontiguousarray(scene.positions, np.float32)
        idx = np.ascontiguousarray(scene.indices, np.uint32)
        ext = np.concatenate([pos.min(0), pos.max(0)]).astype(np.float32)
        tabs = o.scene_tables(scene)
        light_rad = tabs["light_radiance"]  # one per light triangle, as the keys index them
        T = idx.shape[0]
        counts = np.zeros(T, np.uint64)
        box = np.zeros(6, np.float32)
        n = R.ref_svo_voxelize(_p(pos), _p(idx), C.c_uint32(T), _p(ext), C.c_uint32(res),
                               _p(box), _p(counts), None, None, C.c_uint64(0))
        codes = np.zeros(n, np.uint64)
        normals = np.zeros(n, np.uint32)
        assert R.ref_svo_voxelize(_p(pos), _p(idx), C.c_uint32(T), _p(ext), C.c_uint32(res),
                                  _p(box), _p(counts), _p(codes), _p(normals),
                                  C.c_uint64(n)) == n
        st = C.c_int(0)
        h = C.c_void_p(R.ref_svo_build(_p(codes), C.c_uint64(n), _p(ext), C.c_uint32(res),
                                       C.byref(st)))
        assert st.value == 0
        sz = np.zeros(3, np.uint32)
        R.ref_svo_sizes(h, _p(sz))
        nodes = np.zeros(sz[0], np.uint64)
        parents = np.zeros(sz[1], np.uint32)
        leaf_codes = np.zeros(sz[1], np.uint64)
        offsets = np.zeros(sz[2], np.uint32)
        R.ref_svo_get(h, _p(nodes), _p(parents), _p(leaf_codes), _p(offsets))
        g.update({f"{tag}_pos": pos, f"{tag}_idx": idx, f"{tag}_ext": ext,
                  f"{tag}_res": np.array([res], np.uint32), f"{tag}_tri_key": tabs["tri_key"],
                  f"{tag}_light_rad": light_rad, f"{tag}_svo_box": box,
                  f"{tag}_tri_counts": counts, f"{tag}_codes": codes, f"{tag}_normals": normals,
                  f"{tag}_nodes": nodes, f"{tag}_leaf_parents": parents,
                  f"{tag}_leaf_codes": leaf_codes, f"{tag}_level_offsets": offsets})
        # rays hitting points inside random leaves, from random origins
        m = 4000
        lo, hi = box[:3].astype(np.float64), box[3:].astype(np.float64)
        vs = (hi - lo) / res
        c = leaf_codes[rng.integers(0, leaf_codes.shape[0], m)]
        cell = np.zeros((m, 3))
        for b in range(21):
            for k in range(3):
                cell[:, k] += ((c >> np.uint64(3 * b + k)) & np.uint64(1)).astype(np.float64) * (1 << b)
        hitp = lo + (cell + rng.uniform(0.05, 0.95, (m, 3))) * vs
        org = (hitp + rng.normal(size=(m, 3)) * 0.3 * (hi - lo)).astype(np.float32)
        d = hitp - org
        tt = np.linalg.norm(d, axis=1)
        d = (d / tt[:, None]).astype(np.float32)
        tt = tt.astype(np.float32)
        valid = (rng.uniform(size=m) > 0.1).astype(np.uint8)
        g.update({f"{tag}_bin_org": org, f"{tag}_bin_dir": d, f"{tag}_bin_t": tt,
                  f"{tag}_bin_valid": valid})
        for ml, brc in ((5, 512), (3, 64), (1, 4096)):
            out = np.zeros(m, np.uint32)
            R.ref_svo_bin_rays(h, _p(org), _p(d), _p(tt), _p(valid), C.c_uint32(m),
                               C.c_uint32(ml), C.c_uint32(brc), _p(out))
            g[f"{tag}_bins_{ml}_{brc}"] = out
        # cones over the oracle's payload
        svo = o.OracleSvo(scene, tabs["tri_key"], ext, res, light_rad)
        ex = svo.export()
        assert np.array_equal(ex["nodes"], nodes), "oracle octree differs from the reference"
        R.ref_svo_set_payload(h, _p(ex["leaf_normals"]), _p(ex["node_normals"]),
                              _p(ex["leaf_avg"]), _p(ex["node_avg"]))
        for k in ("leaf_normals", "node_normals", "leaf_avg", "node_avg"):
            g[f"{tag}_payload_{k}"] = ex[k]
        org = (lo + rng.uniform(0.02, 0.98, (m, 3)) * (hi - lo)).astype(np.float32)
        d = rng.normal(size=(m, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        tmin = (rng.uniform(0, 0.05, m) * (hi - lo).max()).astype(np.float32)
        tmin[: m // 4] = 0.0
        tmax = np.full(m, 3.0e38, np.float32)
        ap = (4.0 * np.pi / rng.choice([64.0 ** 2, 32.0 ** 2, 8.0 ** 2], m)).astype(np.float32)
        g.update({f"{tag}_cone_org": org, f"{tag}_cone_dir": d, f"{tag}_cone_tmin": tmin,
                  f"{tag}_cone_aperture": ap})
        for mq in (0, 2):
            t = np.zeros(m, np.float32)
            nid = np.zeros(m, np.uint32)
            leaf = np.zeros(m, np.uint8)
            rad = np.zeros(m, np.float32)
            R.ref_svo_cone_trace(h, _p(org), _p(d), _p(tmin), _p(tmax), _p(ap), C.c_uint32(mq),
                                 C.c_uint32(m), _p(t), _p(nid), _p(leaf), _p(rad))
            g.update({f"{tag}_cone{mq}_t": t, f"{tag}_cone{mq}_id": nid,
                      f"{tag}_cone{mq}_leaf": leaf, f"{tag}_cone{mq}_radiance": rad})
        # KCAverageNormals over the oracle's leaf normal words
        nn = np.zeros(nodes.shape[0], np.uint32)
        R.ref_svo_average_normals(h, _p(ex["leaf_normals"]), _p(nn))
        g[f"{tag}_node_normals"] = nn
        if tag == "clusters128":
            U = leaf_codes.shape[0]
            # NormalizeAndFilterRadiance over seeded sums (2^-24 fixed point;
            # the reference gets them as FP32) and counts, 60 % of them empty
            cnt = (rng.integers(1, 40, (U, 2)) * (rng.uniform(size=(U, 2)) < 0.4)).astype(np.uint32)
            fx = (rng.uniform(0, 2.0, (U, 2)) * cnt * (1 << 24)).astype(np.uint64)
            ffl = (fx.astype(np.float64) / (1 << 24)).astype(np.float32)
            la = np.zeros(U, np.uint32)
            na = np.zeros(nodes.shape[0], np.uint32)
            R.ref_svo_normalize_filter(h, _p(ffl), _p(cnt), _p(la), _p(na))
            g.update({f"{tag}_norm_irr": fx, f"{tag}_norm_cnt": cnt, f"{tag}_norm_leaf_avg": la,
                      f"{tag}_norm_node_avg": na})
            # DepositRadiance of vertices in and around random leaves
            m = 8000
            c = leaf_codes[rng.integers(0, U, m)]
            cell = np.zeros((m, 3))
            for b in range(21):
                for k in range(3):
                    cell[:, k] += ((c >> np.uint64(3 * b + k)) & np.uint64(1)).astype(np.float64) * (1 << b)
            pos = (lo + (cell + rng.uniform(-0.1, 1.1, (m, 3))) * vs).astype(np.float32)
            wo = rng.normal(size=(m, 3))
            wo = (wo / np.linalg.norm(wo, axis=1, keepdims=True)).astype(np.float32)
            lum = rng.uniform(0, 3, m).astype(np.float32)
            ri = np.zeros((U, 2), np.float32)
            rc = np.zeros((U, 2), np.uint32)
            R.ref_svo_deposit(h, _p(pos), _p(wo), _p(lum), C.c_uint32(m), _p(ri), _p(rc))
            g.update({f"{tag}_dep_pos": pos, f"{tag}_dep_wo": wo, f"{tag}_dep_lum": lum,
                      f"{tag}_dep_irr": ri, f"{tag}_dep_cnt": rc})
            # DepositNEEHitMiss at the same vertices (a stream of its own, so
            # the arrays above keep their values), then the guiding factors
            # of KCBottomUpFilterIrradiance over seeded counters, 70 % of
            # the leaves without a shadow ray
            rs = np.random.default_rng(20261205)
            is_hit = (rs.uniform(size=m) < 0.6).astype(np.uint8)
            nh = np.zeros(U, np.uint32)
            nm = np.zeros(U, np.uint32)
            R.ref_svo_deposit_nee(h, _p(pos), _p(is_hit), C.c_uint32(m), _p(nh), _p(nm))
            sh = (rs.integers(0, 50, (U, 2)) * (rs.uniform(size=(U, 1)) < 0.3)).astype(np.uint32)
            sh[rs.uniform(size=U) < 0.05, 0] = 0  # some leaves with misses only
            nf = np.zeros(nodes.shape[0], np.uint16)
            sh_hit, sh_miss = np.ascontiguousarray(sh[:, 0]), np.ascontiguousarray(sh[:, 1])
            R.ref_svo_guiding_factors(h, _p(sh_hit), _p(sh_miss), _p(nf))
            g.update({f"{tag}_nee_hit": is_hit, f"{tag}_nee_hits": nh, f"{tag}_nee_misses": nm,
                      f"{tag}_shadow": sh, f"{tag}_node_factor": nf})
        R.ref_svo_destroy(h)
    out = HERE / "svo_reference_vectors.npz"
    np.savez_compressed(out, **g)
    print(f"wrote {out} ({out.stat().st_size / 1024:.0f} KiB, {len(g)} arrays)")


if __name__ == "__main__":
    main(*(sys.argv[1:2]))
