"""The CPU oracle against golden vectors produced by the MRay reference's own
code (tests/golden/make_golden.py, reference routines compiled from the MRay
sources).  This pins the oracle before it is used as the checker of the CUDA
path.

Bit-exact: Morton codes, LBVH topology and AABBs, ray/triangle intersection,
Nudge, Reflect/Refract, quaternion products, Fresnel, GGX D/G, VNDF pdf.
Within a stated tolerance: routines that go through sin/cos/acos, where the
oracle (like the CUDA path) uses its own portable polynomial instead of libm.
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

G = dict(np.load(Path(__file__).resolve().parent / "golden" / "reference_vectors.npz"))
# sin/cos/acos differences of up to ~2 ulp, amplified by at most ~10x in VNDF
TRANSCENDENTAL_ATOL = 2e-6
VNDF_ATOL = 2e-5


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _probe(oracle, name, rows, nout):
    out = np.zeros((rows.shape[0], nout), np.float32)
    for i, r in enumerate(rows):
        r = np.ascontiguousarray(r, np.float32)
        o = np.zeros(nout, np.float32)
        assert oracle.lib.oracle_probe(name.encode(), _p(r), _p(o)) == 0
        out[i] = o
    return out


def test_morton3d(oracle):
    got = np.array([oracle.lib.oracle_morton3d(*map(int, r)) for r in G["morton3d_in"]],
                   np.uint64)
    assert np.array_equal(got, G["morton3d_out"])


def test_morton_codes_of_centroids(oracle):
    aabb = G["morton_aabb"]
    n = aabb.shape[0]
    # triangles whose AABBs are exactly the stored boxes
    pos = np.zeros((3 * n, 3), np.float32)
    pos[0::3], pos[1::3], pos[2::3] = aabb[:, :3], aabb[:, 3:], aabb[:, :3]
    a, ext, delta, codes = oracle.morton_codes(pos, np.arange(3 * n, dtype=np.uint32).reshape(n, 3))
    assert np.array_equal(a, aabb)
    assert np.array_equal(ext, G["morton_extent"])
    assert np.float32(delta) == G["morton_delta"][0]
    assert np.array_equal(codes, G["morton_codes"])


@pytest.mark.parametrize("tag", ["lbvh2", "lbvh3", "lbvh257", "lbvh2000"])
def test_lbvh_topology_and_boxes(oracle, tag):
    r = oracle.lbvh(G[f"{tag}_codes"], G[f"{tag}_order"], G[f"{tag}_leaf_aabb"])
    assert r["status"] == 0
    assert r["root"][0] == G[f"{tag}_root"][0]
    assert np.array_equal(r["left"], G[f"{tag}_left"])
    assert np.array_equal(r["right"], G[f"{tag}_right"])
    assert np.array_equal(r["parent"], G[f"{tag}_parent"])
    assert np.array_equal(r["inner"], G[f"{tag}_inner"])


def test_ray_triangle(oracle):
    n = G["tri_hit"].shape[0]
    for i in range(n):
        t = np.zeros(1, np.float32)
        b = np.zeros(3, np.float32)
        p = [np.ascontiguousarray(G["tri_p"][i, k]) for k in range(3)]
        h = oracle.lib.oracle_intersect_tri(_p(np.ascontiguousarray(G["tri_ro"][i])),
                                            _p(np.ascontiguousarray(G["tri_rd"][i])), _p(p[0]),
                                            _p(p[1]), _p(p[2]), int(G["tri_cull"][i]), _p(t), _p(b))
        assert h == G["tri_hit"][i], i
        if h:
            assert t[0] == G["tri_t"][i] and np.array_equal(b, G["tri_bary"][i]), i
    assert G["tri_hit"].sum() > n // 10


def test_nudge(oracle):
    for i in range(G["nudge_pos"].shape[0]):
        o = np.zeros(3, np.float32)
        oracle.lib.oracle_nudge(_p(np.ascontiguousarray(G["nudge_pos"][i])),
                                _p(np.ascontiguousarray(G["nudge_dir"][i])), _p(o))
        assert np.array_equal(o.view(np.uint32), G["nudge_out"][i].view(np.uint32)), i


def test_reflect_refract(oracle):
    rows = np.concatenate([G["rr_d"], G["rr_n"], G["rr_ior"]], 1)
    refl = _probe(oracle, "reflect", rows, 3)
    assert np.array_equal(refl, G["reflect_out"])
    refr = _probe(oracle, "refract", rows, 4)
    ok = G["refract_ok"] == 1
    assert np.array_equal(refr[:, 0] == 1.0, ok)
    assert np.array_equal(refr[ok, 1:], G["refract_out"][ok])


def test_quaternion_product_and_rotation(oracle):
    mul = _probe(oracle, "quat_mul", np.concatenate([G["q_q0"], G["q_q1"]], 1), 4)
    assert np.array_equal(mul, G["q_mul"])
    rot = _probe(oracle, "quat_rotate", np.concatenate([G["q_q0"], G["q_v"]], 1), 3)
    assert np.array_equal(rot, G["q_rot"])


def test_bary_slerp_within_tolerance(oracle):
    n = G["q_ab"].shape[0]
    out = np.zeros((n, 4), np.float32)
    for i in range(n):
        o = np.zeros(4, np.float32)
        oracle.lib.oracle_bary_slerp(_p(np.ascontiguousarray(G["q_q0"][i])),
                                     _p(np.ascontiguousarray(G["q_q1"][i])),
                                     _p(np.ascontiguousarray(G["q_q2"][i])),
                                     C.c_float(G["q_ab"][i, 0]), C.c_float(G["q_ab"][i, 1]), _p(o))
        out[i] = o
    assert np.abs(out - G["q_slerp"]).max() < TRANSCENDENTAL_ATOL


def test_hemi_cosine_within_tolerance(oracle):
    out = _probe(oracle, "hemi_cosine", G["hemi_xi"], 4)
    # z = sqrt(1 - x^2 - y^2) amplifies the sin/cos ulps at grazing angles
    assert np.abs(out[:, :2] - G["hemi_dir"][:, :2]).max() < TRANSCENDENTAL_ATOL
    assert np.abs(out[:, 2] - G["hemi_dir"][:, 2]).max() < VNDF_ATOL
    assert np.abs(out[:, 3] - G["hemi_pdf"]).max() < TRANSCENDENTAL_ATOL


def test_tangent_space_of_mesh(oracle):
    out = np.zeros_like(G["tbn_out"])
    pos, nrm, uv, idx = (np.ascontiguousarray(G[k]) for k in ("tbn_pos", "tbn_nrm", "tbn_uv",
                                                              "tbn_idx"))
    oracle.lib.oracle_build_tbn(_p(pos), _p(nrm), _p(uv), _p(idx), C.c_uint32(pos.shape[0]),
                                C.c_uint32(idx.shape[0]), _p(out))
    assert np.array_equal(out, G["tbn_out"])


def test_ggx_fresnel_terms(oracle):
    d = _probe(oracle, "dggx", G["dggx_in"], 1)[:, 0]
    assert np.array_equal(d, G["dggx_out"])
    gc = _probe(oracle, "gsmith_corr",
                np.concatenate([G["gs_wo"], G["gs_wi"], G["gs_alpha"][:, None]], 1), 1)[:, 0]
    assert np.array_equal(gc, G["gs_corr"])
    gs = _probe(oracle, "gsmith_single",
                np.concatenate([G["gs_wo"], G["gs_alpha"][:, None]], 1), 1)[:, 0]
    assert np.array_equal(gs, G["gs_single"])
    fc = _probe(oracle, "fresnel_conductor",
                np.concatenate([G["fc_cos"][:, None], G["fc_eta"], G["fc_k"]], 1), 3)
    assert np.array_equal(fc, G["fc_out"])
    fd = _probe(oracle, "fresnel_dielectric", G["fd_in"], 1)[:, 0]
    assert np.array_equal(fd, G["fd_out"])
    vp = _probe(oracle, "vndf_pdf",
                np.concatenate([G["gs_wo"], G["gs_wi"], G["gs_alpha"][:, None]], 1), 1)[:, 0]
    assert np.array_equal(vp, G["vndfpdf_out"])
    ph = _probe(oracle, "power_heuristic", G["ph_in"], 1)[:, 0]
    assert np.array_equal(ph, G["ph_out"])


def test_vndf_sample_within_tolerance(oracle):
    rows = np.concatenate([G["vndf_v"], G["vndf_alpha"][:, None], G["vndf_xi"]], 1)
    out = _probe(oracle, "vndf_sample", rows, 4)
    assert np.abs(out[:, :3] - G["vndf_h"]).max() < VNDF_ATOL
    rel = np.abs(out[:, 3] - G["vndf_pdf"]) / np.maximum(np.abs(G["vndf_pdf"]), 1e-6)
    assert np.median(rel) < 1e-5 and rel.max() < 1e-2


# ---- octree (guided path): vectors from the reference's own voxelizer, level
# kernels, ray binning and cone tracer (tests/golden/make_golden.py svo_golden)
S = dict(np.load(Path(__file__).resolve().parent / "golden" / "svo_reference_vectors.npz"))
SVO_CASES = ("cornell64", "clusters128")


class _Mesh:
    def __init__(self, tag):
        self.positions = S[f"{tag}_pos"]
        self.indices = S[f"{tag}_idx"]


def _svo(oracle, tag):
    return oracle.OracleSvo(_Mesh(tag), S[f"{tag}_tri_key"], S[f"{tag}_ext"],
                            int(S[f"{tag}_res"][0]), S[f"{tag}_light_rad"])


@pytest.mark.parametrize("tag", SVO_CASES)
def test_svo_voxelize_matches_reference(oracle, tag):
    """TriFunctions::Voxelize: per-triangle voxel counts and Morton codes are
    bit-exact.  The packed spherical normal (two 16-bit UNORMs of atan2 and
    acos) may differ by one step where the oracle's portable atan2/acos and
    the C library round to neighbouring floats."""
    counts, codes, normals = oracle.voxelize(S[f"{tag}_pos"], S[f"{tag}_idx"], S[f"{tag}_ext"],
                                             int(S[f"{tag}_res"][0]))
    assert np.array_equal(counts, S[f"{tag}_tri_counts"])
    assert np.array_equal(codes, S[f"{tag}_codes"])
    ref = S[f"{tag}_normals"]
    du = np.abs((normals & 0xFFFF).astype(np.int64) - (ref & 0xFFFF).astype(np.int64))
    dv = np.abs((normals >> 16).astype(np.int64) - (ref >> 16).astype(np.int64))
    assert du.max() <= 1 and dv.max() <= 1
    assert np.count_nonzero(normals != ref) <= max(1, ref.shape[0] // 500)


@pytest.mark.parametrize("tag", SVO_CASES)
def test_svo_structure_matches_reference(oracle, tag):
    """AnisoSVOctreeCPU::Constrcut's level kernels: packed nodes (children,
    parent, child mask, leaf bit), leaf parents, leaf codes and level offsets
    bit-exact."""
    ex = _svo(oracle, tag).export()
    for k in ("nodes", "leaf_parents", "leaf_codes", "level_offsets"):
        assert np.array_equal(ex[k], S[f"{tag}_{k}"]), k


@pytest.mark.parametrize("tag", SVO_CASES)
@pytest.mark.parametrize("min_level,ray_count", [(5, 512), (3, 64), (1, 4096)])
def test_svo_bins_match_reference(oracle, tag, min_level, ray_count):
    """Ray binning: the leaf of each hit (NearestNodeIndex with the neighbour
    search), leaf ray counts, the bottom-up collapse to MinRayBinLevel until
    BinRayCount rays, and FindMarkedBin: every ray's bin id bit-exact."""
    svo = _svo(oracle, tag)
    got = svo.bin_rays(S[f"{tag}_bin_org"], S[f"{tag}_bin_dir"], S[f"{tag}_bin_t"],
                       S[f"{tag}_bin_valid"], min_level, ray_count)
    assert np.array_equal(got, S[f"{tag}_bins_{min_level}_{ray_count}"])


@pytest.mark.parametrize("tag", SVO_CASES)
@pytest.mark.parametrize("max_query_offset", [0, 2])
def test_svo_cone_trace_matches_reference(oracle, tag, max_query_offset):
    """ConeTraceRay + ReadRadiance: returned t, node or leaf index, leaf flag
    and radiance bit-exact for cones of three apertures, half of them from
    tMin 0 inside the octree.  The radiance is read from the oracle's payload,
    stored with the vectors as the reference's input."""
    svo = _svo(oracle, tag)
    ex = svo.export()
    for k in ("leaf_normals", "node_normals", "leaf_avg", "node_avg"):
        assert np.array_equal(ex[k], S[f"{tag}_payload_{k}"]), k
    got = svo.cone_trace(S[f"{tag}_cone_org"], S[f"{tag}_cone_dir"], S[f"{tag}_cone_tmin"],
                         S[f"{tag}_cone_aperture"], max_query_offset)
    p = f"{tag}_cone{max_query_offset}"
    assert np.array_equal(got["t"].view(np.uint32), S[f"{p}_t"].view(np.uint32))
    assert np.array_equal(got["id"], S[f"{p}_id"])
    assert np.array_equal(got["leaf"], S[f"{p}_leaf"])
    assert np.array_equal(got["radiance"].view(np.uint32), S[f"{p}_radiance"].view(np.uint32))
    assert np.count_nonzero(S[f"{p}_id"] != 0xFFFFFFFF) > 1000
    assert np.count_nonzero(S[f"{p}_radiance"]) > 50


@pytest.mark.parametrize("tag", SVO_CASES)
def test_svo_node_normals_match_reference(oracle, tag):
    """KCAverageNormals (k-means with K = 2 over the children's Toksvig-scaled
    normals, bottom-up): every node's normal/specular word bit-exact from the
    same leaf words."""
    ex = _svo(oracle, tag).export()
    assert np.array_equal(ex["leaf_normals"], S[f"{tag}_payload_leaf_normals"])
    assert np.array_equal(ex["node_normals"], S[f"{tag}_node_normals"])


def _half_steps(a, b):
    """Largest distance in binary16 steps between two arrays of half2 words."""
    ua = np.concatenate([a & 0xFFFF, a >> 16]).astype(np.int64)
    ub = np.concatenate([b & 0xFFFF, b >> 16]).astype(np.int64)
    return int(np.abs(ua - ub).max())


def test_svo_normalize_filter_matches_reference(oracle):
    """NormalizeAndFilterRadiance: leaf averages (sum / count, clamped, to
    half), bottom-up node averages over the children with the normal-side
    swap and the empty-marker rules, then the top-down fill.  The oracle
    divides the 2^-24 fixed-point sums in double and averages the children in
    FP32 with one rounding to half; the reference divides FP32 sums and adds
    the children in half precision.  Tolerances: leaf averages within one
    binary16 step, node averages within four, and the empty markers (which
    decide the top-down fill) identical."""
    tag = "clusters128"
    svo = _svo(oracle, tag)
    svo.set_radiance(S[f"{tag}_norm_irr"], S[f"{tag}_norm_cnt"])
    ex = svo.export()
    leaf_ref, node_ref = S[f"{tag}_norm_leaf_avg"], S[f"{tag}_norm_node_avg"]
    assert _half_steps(ex["leaf_avg"], leaf_ref) <= 1
    assert np.count_nonzero(ex["leaf_avg"] != leaf_ref) <= leaf_ref.shape[0] // 1000
    assert _half_steps(ex["node_avg"], node_ref) <= 4
    assert np.count_nonzero(ex["node_avg"] != node_ref) <= node_ref.shape[0] // 4
    for a, r in ((ex["leaf_avg"], leaf_ref), (ex["node_avg"], node_ref)):
        for sh in (0, 16):
            assert np.array_equal(((a >> sh) & 0xFFFF) == 0x7BFF, ((r >> sh) & 0xFFFF) == 0x7BFF)


def test_svo_deposit_matches_reference(oracle):
    """DepositRadiance: the leaf of each vertex (neighbour search), the side
    its normal puts wo on, and the per-leaf, per-side sample counts are
    bit-exact; the radiance sums agree within 1e-4 relative (the reference
    adds FP32 values, the oracle 2^-24 fixed-point ones)."""
    tag = "clusters128"
    svo = _svo(oracle, tag)
    svo.deposit(S[f"{tag}_dep_pos"], S[f"{tag}_dep_wo"], S[f"{tag}_dep_lum"])
    ex = svo.export()
    assert np.array_equal(ex["leaf_cnt"], S[f"{tag}_dep_cnt"])
    assert S[f"{tag}_dep_cnt"].sum() > 7000
    got = ex["leaf_irr"].astype(np.float64) / (1 << 24)
    ref = S[f"{tag}_dep_irr"].astype(np.float64)
    assert np.all(np.abs(got - ref) <= 1e-4 * np.maximum(ref, 1e-3))


def test_svo_nee_deposit_matches_reference(oracle):
    """DepositNEEHitMiss: the leaf of each vertex (the same neighbour search
    as DepositRadiance) takes one hit or one miss; per-leaf counters
    bit-exact."""
    tag = "clusters128"
    svo = _svo(oracle, tag)
    svo.deposit_nee(S[f"{tag}_dep_pos"], S[f"{tag}_nee_hit"])
    ex = svo.export()
    assert np.array_equal(ex["leaf_shadow"][:, 0], S[f"{tag}_nee_hits"])
    assert np.array_equal(ex["leaf_shadow"][:, 1], S[f"{tag}_nee_misses"])
    assert S[f"{tag}_nee_hits"].sum() > 4000 and S[f"{tag}_nee_misses"].sum() > 2500


def test_svo_guiding_factors_match_reference(oracle):
    """KCBottomUpFilterIrradiance's guiding factors: a leaf's miss ratio
    misses / (hits + misses), NaN without shadow rays; a node's the FP32 mean
    of its children's factors that are not NaN, rounded to binary16, and the
    NaN 0x7FFF when none has data.  Bit-exact over seeded counters (70 % of
    the leaves without any, some with misses only)."""
    tag = "clusters128"
    svo = _svo(oracle, tag)
    svo.set_shadow(S[f"{tag}_shadow"])
    ref = S[f"{tag}_node_factor"]
    got = svo.export()["node_factor"]
    assert np.array_equal(got, ref)
    nan = (ref & 0x7C00) == 0x7C00
    assert 0 < np.count_nonzero(nan) < ref.shape[0] // 2
    sh = S[f"{tag}_shadow"]
    assert np.count_nonzero((sh[:, 0] == 0) & (sh[:, 1] > 0)) > 100  # leaves with misses only


def test_product_sampler_matches_reference(oracle):
    """ProductSampler (ProductSampler.cuh:160-660): the reference's own
    sampler, run once on a B200 by the harness of oracle/psamp/ with table
    stand-ins for the material system and the random numbers
    (tests/golden/make_golden_product.py), against the oracle's restatement
    on the same tables: the cell means (a pairwise tree per 32 texels, as the
    reference's warp reduction adds them) and maxima, the BxDF-or-guide
    choice, the drawn map coordinates and the one-sample MIS pdf of 576 rays
    over 12 fields (smooth, with blobs, with spikes) are bit-exact."""
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    import make_golden_product as mk
    P = np.load(Path(__file__).resolve().parent / "golden" / "product_sampler_vectors.npz")
    fields, surfaces, streams = mk.inputs()
    assert mk.digest(fields, surfaces, streams) == P["input_digest"].tobytes()
    got = oracle.product_pin(fields, int(P["rays_per_bin"]), surfaces, streams,
                             float(P["mis_ratio"]), float(P["mult"]))
    for k in ("small", "norm", "uv", "pdf"):
        assert np.array_equal(got[k].view(np.uint32), P[k].view(np.uint32)), k
    assert np.array_equal(got["sel"], P["sel"])
    assert 0 < int(P["sel"].sum()) < P["sel"].shape[0]   # both branches covered
