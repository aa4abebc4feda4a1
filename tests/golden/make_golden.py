"""Generate golden vectors from the MRay reference's own code.

Runs the reference routines compiled by ``make -C oracle ref`` into
``oracle/_ref/libmrayref.so`` (MRay headers #included from the reference
tree; LBVH kernels cut from LinearBVH.hpp at build time) on seeded random
inputs and stores inputs + outputs in ``tests/golden/reference_vectors.npz``.
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


if __name__ == "__main__":
    main(*(sys.argv[1:2]))
