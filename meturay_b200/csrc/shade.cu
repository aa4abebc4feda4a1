// Camera ray generation, ray partitioning helpers, shading and image resolve
// for the plain wavefront path tracer.
//
//   k_camera       KCGenCameraRaysFromArrayGPU + GPUCameraPinhole::GenerateRay
//                  (GenerationKernels.cuh:26-108, GPUCameraPinhole.cuh:209-243)
//   k_dense_keys   HitKey -> dense (batch, id) key for the partition sort
//                  (FillMatIdsForSortKC, RayMemory.cu:17-30)
//   k_portions     batch boundaries of the sorted keys -> device portion
//                  table (FindSplitsSparseKC/FindSplitBatchesKC,
//                  RayMemory.cu:64-104,230-312), found with warp ballots
//   k_shade        one launch over all non-null rays in partition order:
//                  PathTracerPathWork / PathTracerBoundaryWork
//                  (PathTracerKC.cuh:335-649) with Lambert, Metal (GGX) and
//                  Refract BxDFs; outputs are compacted with warp-aggregated
//                  atomics into the next wavefront
//   k_resolve      per-pixel mean of its s*s samples, accumulated per frame
#include "common.cuh"
#include "shade.cuh"

namespace mrb {

namespace {

struct Surface {
    V3 pos;
    Q4 w2t;
    V3 geo;
    bool back;
};

// TriangleSurfaceGenerator::GenBasicSurface (GPUPrimitiveTriangle.h:624-700)
__device__ __forceinline__ Surface gen_surface(const SceneDev& s, uint32_t prim, float a, float b,
                                               V3 rayDir) {
    const bool twoSided = s.triCull ? (s.triCull[prim] == 0) : true;
    const float c = 1.0f - a - b;
    const uint32_t i0 = s.idx[3 * prim], i1 = s.idx[3 * prim + 1], i2 = s.idx[3 * prim + 2];
    Q4 tbn = bary_slerp(q_from(__ldg(s.tbn + i0)), q_from(__ldg(s.tbn + i1)),
                        q_from(__ldg(s.tbn + i2)), a, b);
    tbn = qnormalize(tbn);
    const V3 p0 = ld3(s.pos + 3 * size_t(i0)), p1 = ld3(s.pos + 3 * size_t(i1)),
             p2 = ld3(s.pos + 3 * size_t(i2));
    Surface sf;
    sf.pos = (p0 * a + p1 * b) + p2 * c;
    V3 g = normalize(cross(p1 - p0, p2 - p0));
    g = normalize(g);
    sf.w2t = tbn;
    sf.back = twoSided && (dot(g, rayDir) > 0.0f);
    if (sf.back) {
        g = -g;
        sf.w2t = qmul(Q4{0.0f, 1.0f, 0.0f, 0.0f}, sf.w2t);
    }
    sf.geo = g;
    return sf;
}

struct BSample {
    V3 dir, pos, refl;
    float pdf;
    uint32_t medium;
};

// HemiDistribution::HemiCosineCDF (HemiDistribution.h:10-30)
__device__ __forceinline__ V3 hemi_cosine(float xi0, float xi1, float& pdf) {
    float coeff = 2.0f * kPiF * xi1;
    float sn, cs;
    pm_sincos(coeff, sn, cs);
    V3 d;
    d.x = sqrtf(xi0) * cs;
    d.y = sqrtf(xi0) * sn;
    d.z = sqrtf(fmaxf(0.0f, (1.0f - d.x * d.x - d.y * d.y)));
    pdf = d.z * kInvPiF;
    return d;
}

// TracerFunctions.cuh:8-30
__device__ __forceinline__ float fresnel_dielectric(float cosIn, float iorIn, float iorOut) {
    float sinIn = sqrtf(fmaxf(0.0f, 1.0f - cosIn * cosIn));
    float sinOut = iorIn / iorOut * sinIn;
    if (sinOut >= 1.0f) return 1.0f;
    float cosOut = sqrtf(fmaxf(0.0f, 1.0f - sinOut * sinOut));
    float par = ((iorOut * cosIn - iorIn * cosOut) / (iorOut * cosIn + iorIn * cosOut));
    par = par * par;
    float perp = ((iorIn * cosIn - iorOut * cosOut) / (iorIn * cosIn + iorOut * cosOut));
    perp = perp * perp;
    return (par + perp) * 0.5f;
}
// TracerFunctions.cuh:33-75
__device__ __forceinline__ V3 fresnel_conductor(float cosIn, V3 eta, V3 k) {
    float cosInSqr = cosIn * cosIn;
    float sinInSqr = fmaxf(0.0f, 1.0f - cosInSqr);
    float sinInSqr2 = sinInSqr * sinInSqr;
    float sinInSqr4 = sinInSqr2 * sinInSqr2;
    V3 etaSqr = eta * eta;
    V3 kSqr = k * k;
    V3 diff = etaSqr - kSqr - v3(sinInSqr, sinInSqr, sinInSqr);
    V3 a2b2 = diff * diff;
    a2b2 = a2b2 + 4.0f * etaSqr * kSqr;
    a2b2 = vsqrt(vmax0(a2b2));
    V3 a = 0.5f * (a2b2 + diff);
    a = vsqrt(vmax0(a));
    V3 perpT1 = a2b2 + v3(cosInSqr, cosInSqr, cosInSqr);
    V3 perpT2 = a * (2.0f * cosIn);
    V3 perp = vdiv(perpT1 - perpT2, perpT1 + perpT2);
    V3 parT1 = a2b2 * cosInSqr + v3(sinInSqr4, sinInSqr4, sinInSqr4);
    V3 parT2 = perpT2 * sinInSqr2;
    V3 par = vdiv(perp * (parT1 - parT2), parT1 + parT2);
    return (par + perp) * 0.5f;
}
__device__ __forceinline__ float dggx(float NdH, float alpha) {  // :77-86
    float a2 = alpha * alpha;
    float den = NdH * NdH * (a2 - 1.0f) + 1.0f;
    den = den * den;
    den *= kPiF;
    return a2 / den;
}
__device__ __forceinline__ float lambda_smith(V3 v, float alpha) {  // :88-97
    V3 s = v * v;
    float a2 = alpha * alpha;
    float inner = a2 * (s.x + s.y) / s.z;
    float l = sqrtf(1.0f + inner) - 1.0f;
    return l * 0.5f;
}
__device__ __forceinline__ float g_smith_single(V3 v, float alpha) {
    return 1.0f / (1.0f + lambda_smith(v, alpha));
}
__device__ __forceinline__ float g_smith_corr(V3 o, V3 i, float alpha) {
    return 1.0f / (lambda_smith(o, alpha) + lambda_smith(i, alpha) + 1.0f);
}
__device__ __forceinline__ float vndf_pdf(V3 V, V3 H, float alpha) {  // :181-190
    float VdH = fmaxf(0.0f, dot(H, V));
    float NdH = fmaxf(0.0f, H.z);
    float NdV = fmaxf(0.0f, V.z);
    float D = dggx(NdH, alpha);
    float G = g_smith_single(V, alpha);
    return (NdV == 0.0f) ? 0.0f : (VdH * D * G / NdV);
}
// VNDFGGXSmithSample (TracerFunctions.cuh:192-251), Heitz 2018
__device__ __forceinline__ V3 vndf_sample(float& pdf, V3 V, float alpha, float xi0, float xi1) {
    float a = alpha;
    V3 VH = normalize(v3(a * V.x, a * V.y, V.z));
    float lensq = VH.x * VH.x + VH.y * VH.y;
    V3 T1 = (lensq > 0.0f) ? v3(-VH.y, VH.x, 0.0f) / sqrtf(lensq) : v3(1.0f, 0.0f, 0.0f);
    V3 T2 = cross(VH, T1);
    float r = sqrtf(xi0);
    float phi = 2.0f * kPiF * xi1;
    float sn, cs;
    pm_sincos(phi, sn, cs);
    float t1 = r * cs;
    float t2 = r * sn;
    float s = 0.5f * (1.0f + VH.z);
    t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
    float val = 1.0f - t1 * t1 - t2 * t2;
    V3 NH = t1 * T1 + t2 * T2 + sqrtf(fmaxf(0.0f, val)) * VH;
    V3 NM = v3(a * NH.x, a * NH.y, fmaxf(0.0f, NH.z));
    float len2 = dot(NM, NM);
    if (len2 < 1.0e-5f) NM = v3(0.0f, 0.0f, 1.0f);
    else NM = NM * (1.0f / sqrtf(len2));
    pdf = vndf_pdf(V, NM, alpha);
    return NM;
}

struct MetalP {
    V3 eta, k, spec;
    float rough;
};
__device__ __forceinline__ MetalP metal_params(const float* p) {
    return {ld3(p), ld3(p + 3), ld3(p + 6), p[9]};
}

// MetalMatFuncs::Sample (MetalGlassMaterialsKC.cuh:26-146)
__device__ BSample metal_sample(const MetalP& m, V3 wi, const Surface& sf, float xi0, float xi1,
                                uint32_t medium) {
    float alpha = m.rough * m.rough;
    V3 V = to_tangent(wi, sf.w2t);
    BSample out;
    float pdf;
    V3 H = vndf_sample(pdf, V, alpha, xi0, xi1);
    float VdH = fmaxf(0.0f, dot(V, H));
    V3 L = 2.0f * VdH * H - V;
    pdf = (VdH == 0.0f) ? 0.0f : pdf / (4.0f * VdH);
    float LdH = fmaxf(0.0f, dot(L, H));
    float NdH = fmaxf(0.0f, H.z);
    float NdV = fmaxf(0.0f, V.z);
    V3 F = fresnel_conductor(VdH, m.eta, m.k);
    F = F * m.spec;
    float D = dggx(NdH, alpha);
    float G = g_smith_corr(V, L, alpha);
    G = (LdH == 0.0f) ? 0.0f : G;
    G = (VdH == 0.0f) ? 0.0f : G;
    V3 st = D * F * G * 0.25f / NdV;
    st = (NdV == 0.0f) ? v3(0.0f, 0.0f, 0.0f) : st;
    if (isinf(D) || isnan(D)) {
        if (m.rough == 0.0f) L = 2.0f * V.z * v3(0.0f, 0.0f, 1.0f) - V;
        st = G * F;
        float gs = g_smith_single(V, alpha);
        if (gs != 0.0f) st = st / gs;
        else st = v3(0.0f, 0.0f, 0.0f);
        pdf = 1.0f;
    }
    out.dir = to_space(L, sf.w2t);
    out.pos = nudge(sf.pos, sf.geo);
    out.refl = st;
    out.pdf = pdf;
    out.medium = medium;
    return out;
}
// MetalMatFuncs::Evaluate (MetalGlassMaterialsKC.cuh:174-214)
__device__ V3 metal_eval(const MetalP& m, V3 wo, V3 wi, const Surface& sf) {
    float alpha = m.rough * m.rough;
    V3 L = to_tangent(wo, sf.w2t);
    V3 V = to_tangent(wi, sf.w2t);
    V3 H = normalize(L + V);
    float LdH = fmaxf(0.0f, dot(L, H));
    float VdH = fmaxf(0.0f, dot(V, H));
    float NdH = fmaxf(0.0f, H.z);
    float NdV = fmaxf(0.0f, V.z);
    float D = dggx(NdH, alpha);
    D = (isnan(D) || isinf(D)) ? 0.0f : D;
    float G = g_smith_corr(V, L, alpha);
    G = (LdH == 0.0f) ? 0.0f : G;
    G = (VdH == 0.0f) ? 0.0f : G;
    V3 F = fresnel_conductor(VdH, m.eta, m.k);
    F = F * m.spec;
    V3 st = D * F * G * 0.25f / NdV;
    return (NdV == 0.0f) ? v3(0.0f, 0.0f, 0.0f) : st;
}
// LambertMatFuncs (LambertMaterialKC.cuh:14-103)
__device__ __forceinline__ BSample lambert_sample(V3 albedo, const Surface& sf, float xi0, float xi1,
                                                  uint32_t medium) {
    BSample out;
    float pdf;
    V3 d = hemi_cosine(xi0, xi1, pdf);
    d = normalize(d);
    float nDotL = fmaxf(d.z, 0.0f);
    out.dir = to_space(d, sf.w2t);
    out.pos = nudge(sf.pos, sf.geo);
    out.refl = nDotL * albedo * kInvPiF;
    out.pdf = pdf;
    out.medium = medium;
    return out;
}
__device__ __forceinline__ V3 lambert_eval(V3 albedo, V3 wo, const Surface& sf) {
    V3 n = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
    float nDotL = fmaxf(dot(n, wo), 0.0f);
    return nDotL * albedo * kInvPiF;
}
// RefractMatFuncs::Sample (SimpleMaterialsKC.cuh:172-286), Ray::Reflect /
// Ray::Refract (RayLib/Ray.hpp:302-356)
__device__ BSample refract_sample(V3 albedo, uint32_t matMedium, const SceneDev& s, V3 wi,
                                  const Surface& sf, uint32_t curMedium, float xi) {
    BSample out;
    float iIOR = s.mediumIor[matMedium];
    float dIOR = s.mediumIor[s.baseMedium];
    V3 n = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
    bool entering = !sf.back;
    float from = s.mediumIor[curMedium];
    float to = entering ? iIOR : dIOR;
    float f = fresnel_dielectric(fabsf(dot(wi, n)), from, to);
    if (xi < f) {
        out.dir = 2.0f * dot(wi, n) * n - wi;
        out.pos = nudge(sf.pos, sf.geo);
        out.pdf = f;
        out.medium = curMedium;
        out.refl = f * albedo;
        return out;
    }
    out.medium = entering ? matMedium : s.baseMedium;
    out.pdf = 1.0f - f;
    float ratio = from / to;
    float cosIn = dot(n, wi);
    float sinInSqr = fmaxf(0.0f, 1.0f - cosIn * cosIn);
    float sinOutSqr = ratio * ratio * sinInSqr;
    float cosOut = sqrtf(fmaxf(0.0f, 1.0f - sinOutSqr));
    if (sinOutSqr >= 1.0f) {
        out.pdf = 0.0f;
        out.refl = v3(0.0f, 0.0f, 0.0f);
        out.dir = wi;
        out.pos = sf.pos;
        return out;
    }
    out.dir = ratio * (-wi) + (ratio * cosIn - cosOut) * n;
    out.pos = nudge(sf.pos, -sf.geo);
    out.refl = albedo * 1.0f * (1.0f - f);
    return out;
}

// Quat::RotationBetweenZAxis (Quaternion.hpp:333-358)
__device__ __forceinline__ Q4 rotation_between_z(V3 b) {
    V3 zc = v3(-b.y, b.x, 0.0f);
    const float zd = b.z;
    const float sn = sqrtf((1.0f - zd) * 0.5f);
    const float cs = sqrtf((zd + 1.0f) * 0.5f);
    zc = normalize(zc);
    if (fabsf(zd + 1.0f) < 1.0e-4f) return Q4{0.0f, 0.0f, 1.0f, 0.0f};
    if (fabsf(zd - 1.0f) < 1.0e-4f) return Q4{1.0f, 0.0f, 0.0f, 0.0f};
    return Q4{cs, zc.x * sn, zc.y * sn, zc.z * sn};
}

// LambertConstFuncs, "LambertC" (SimpleMaterialsKC.cuh:16-103): uniform
// hemisphere sampling around the shading normal
__device__ __forceinline__ BSample lambertc_sample(V3 albedo, const Surface& sf, float xi0, float xi1,
                                                   uint32_t medium) {
    BSample out;
    const V3 n = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
    // HemiDistribution::HemiUniformCDF (HemiDistribution.h:34-51)
    const float c0 = sqrtf(fmaxf(0.0f, 1.0f - xi0 * xi0));
    const float c1 = 2.0f * kPiF * xi1;
    float sn, cs;
    pm_sincos(c1, sn, cs);
    V3 d = v3(c0 * cs, c0 * sn, xi0);
    out.pdf = kInvPiF * 0.5f;
    d = normalize(d);
    d = qrotate(rotation_between_z(n), d);
    const float nDotL = fabsf(dot(n, d));
    out.dir = d;
    out.pos = nudge(sf.pos, sf.geo);
    out.refl = nDotL * albedo * kInvPiF;
    out.medium = medium;
    return out;
}
__device__ __forceinline__ V3 lambertc_eval(V3 albedo, V3 wo, const Surface& sf) {
    const V3 n = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
    return fmaxf(dot(n, wo), 0.0f) * albedo * kInvPiF;
}
__device__ __forceinline__ float lambert_pdf(V3 wo, const Surface& sf) {
    const V3 n = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
    return fmaxf(dot(wo, n), 0.0f) * kInvPiF;
}
// MetalMatFuncs::Pdf (MetalGlassMaterialsKC.cuh:148-172)
__device__ float metal_pdf(const MetalP& m, V3 wo, V3 wi, const Surface& sf) {
    const float alpha = m.rough * m.rough;
    const V3 L = to_tangent(wo, sf.w2t), V = to_tangent(wi, sf.w2t);
    const V3 H = normalize(L + V);
    const float NdH = fmaxf(0.0f, H.z), VdH = fmaxf(0.0f, dot(V, H));
    float p = vndf_pdf(V, H, alpha);
    const float D = dggx(NdH, alpha);
    p = (isnan(D) || isinf(D)) ? 0.0f : p;
    return (VdH == 0.0f) ? 0.0f : p / (4.0f * VdH);
}

// UnrealDeviceFuncs (UnrealMaterialKC.cuh:19-359): Lambert + GGX with
// Schlick Fresnel, lobes chosen by a luminance-based ratio
struct UnrealP {
    V3 albedo;
    float rough, metallic, specular;
};
__device__ __forceinline__ UnrealP unreal_params(const float* p) {
    return {ld3(p), p[3], p[4], p[5]};
}
__device__ __forceinline__ float luminance(V3 c) {  // ColorConversion.h:15-21
    return 0.2120f * c.x + 0.7150f * c.y + 0.0722f * c.z;
}
__device__ __forceinline__ float unreal_mis_ratio(float metallic, float specular, float lum) {
    float diffuse = 2.0f * kPiF * lum;
    diffuse *= (1.0f - metallic);
    const float specRatio = (1.0f - metallic) * specular + metallic * lum;
    const float total = specRatio + diffuse;
    return diffuse / total;
}
__device__ __forceinline__ V3 unreal_f0(V3 albedo, float metallic, float specular) {
    specular *= 0.08f;
    // Vector3::Lerp(a, b, t) = a * (1 - t) + b * t
    const V3 a = v3(specular, specular, specular);
    return a * (1.0f - metallic) + albedo * metallic;
}
__device__ __forceinline__ V3 f_schlick(float VdH, V3 f0) {  // TracerFunctions.cuh:160-179
    const float pt = 1.0f - VdH;
    float p5 = pt * pt;
    p5 *= p5;
    p5 *= pt;
    V3 r = (v3(1.0f, 1.0f, 1.0f) - f0) * p5;
    return r + f0;
}
__device__ BSample unreal_sample(const UnrealP& m, V3 wi, const Surface& sf, float xiSel,
                                 float xi0, float xi1, uint32_t medium) {
    BSample out;
    const float alpha = m.rough * m.rough;
    const V3 V = to_tangent(wi, sf.w2t);
    float misRatio = unreal_mis_ratio(m.metallic, m.specular, luminance(m.albedo));
    const bool diffuse = xiSel < misRatio;
    float VdH, pdfSel, pdfOther;
    V3 H, L;
    if (diffuse) {
        L = hemi_cosine(xi0, xi1, pdfSel);
        H = normalize(V + L);
        VdH = fmaxf(0.0f, dot(V, H));
        pdfOther = vndf_pdf(V, H, alpha);
        pdfOther = (VdH == 0.0f) ? 0.0f : pdfOther / (4.0f * VdH);
    } else {
        H = vndf_sample(pdfSel, V, alpha, xi0, xi1);
        VdH = fmaxf(0.0f, dot(V, H));
        L = 2.0f * VdH * H - V;
        pdfOther = fmaxf(0.0f, L.z) * kInvPiF;
        pdfSel = (VdH == 0.0f) ? 0.0f : pdfSel / (4.0f * VdH);
        misRatio = 1.0f - misRatio;
    }
    float& pdfSpec = diffuse ? pdfOther : pdfSel;
    pdfSpec = (VdH == 0.0f) ? 0.0f : pdfSpec;
    const float LdH = fmaxf(0.0f, dot(L, H)), NdH = fmaxf(0.0f, H.z), NdV = fmaxf(0.0f, V.z);
    const float D = dggx(NdH, alpha);
    float G = g_smith_corr(V, L, alpha);
    G = (LdH == 0.0f) ? 0.0f : G;
    G = (VdH == 0.0f) ? 0.0f : G;
    const V3 F = f_schlick(VdH, unreal_f0(m.albedo, m.metallic, m.specular));
    V3 spec = D * F * G * 0.25f / NdV;
    spec = (NdV == 0.0f) ? v3(0.0f, 0.0f, 0.0f) : spec;
    if (isinf(D) || isnan(D)) {
        spec = G * F / g_smith_single(V, alpha);
        pdfSpec = diffuse ? 0.0f : 1.0f;
    }
    const float NdL = fmaxf(0.0f, L.z);
    const V3 diffAlbedo = (1.0f - m.metallic) * m.albedo;
    const V3 diffTerm = NdL * diffAlbedo * kInvPiF;
    // TracerFunctions::BalanceHeuristic
    const float w0 = misRatio * pdfSel, w1 = (1.0f - misRatio) * pdfOther;
    const float misWeight = w0 / (w0 + w1);
    out.pdf = (pdfSel == 0.0f) ? 0.0f : (misRatio * pdfSel / misWeight);
    out.dir = to_space(L, sf.w2t);
    out.pos = nudge(sf.pos, sf.geo);
    out.refl = diffTerm + spec;
    out.medium = medium;
    return out;
}
__device__ V3 unreal_eval(const UnrealP& m, V3 wo, V3 wi, const Surface& sf) {
    const float alpha = m.rough * m.rough;
    const V3 L = to_tangent(wo, sf.w2t), V = to_tangent(wi, sf.w2t);
    const V3 H = normalize(L + V);
    const float LdH = fmaxf(0.0f, dot(L, H)), VdH = fmaxf(0.0f, dot(V, H));
    const float NdH = fmaxf(0.0f, H.z), NdV = fmaxf(0.0f, V.z);
    float D = dggx(NdH, alpha);
    D = (isnan(D) || isinf(D)) ? 0.0f : D;
    float G = g_smith_corr(V, L, alpha);
    G = (LdH == 0.0f) ? 0.0f : G;
    G = (VdH == 0.0f) ? 0.0f : G;
    const V3 F = f_schlick(VdH, unreal_f0(m.albedo, m.metallic, m.specular));
    V3 spec = D * F * G * 0.25f / NdV;
    spec = (NdV == 0.0f) ? v3(0.0f, 0.0f, 0.0f) : spec;
    const float NdL = fmaxf(0.0f, L.z);
    const V3 diffTerm = NdL * ((1.0f - m.metallic) * m.albedo) * kInvPiF;
    return diffTerm + spec;
}
__device__ float unreal_pdf(const UnrealP& m, V3 wo, V3 wi, const Surface& sf) {
    const float alpha = m.rough * m.rough;
    const V3 L = to_tangent(wo, sf.w2t), V = to_tangent(wi, sf.w2t);
    const V3 H = normalize(L + V);
    const float NdH = fmaxf(0.0f, H.z), VdH = fmaxf(0.0f, dot(V, H));
    float ps = vndf_pdf(V, H, alpha);
    const float D = dggx(NdH, alpha);
    ps = (isnan(D) || isinf(D)) ? 0.0f : ps;
    ps = (VdH == 0.0f) ? 0.0f : ps / (4.0f * VdH);
    const float pd = fmaxf(0.0f, L.z) * kInvPiF;
    const float r = unreal_mis_ratio(m.metallic, m.specular, luminance(m.albedo));
    return r * pd + (1.0f - r) * ps;
}
__device__ __forceinline__ float power_heuristic(float p0, float p1) {  // n0 = n1 = 1
    const float w0 = 1.0f * p0, w1 = 1.0f * p1;
    return (w0 * w0) / (w0 * w0 + w1 * w1);
}

__global__ void __launch_bounds__(256) k_camera(const CameraDev* __restrict__ camPtr,
                                                PathOptions opt, uint32_t baseMedium,
                                                float4* __restrict__ rayO,
                                                float4* __restrict__ rayD,
                                                RayAux* __restrict__ aux,
                                                float4* __restrict__ samples,
                                                uint32_t* __restrict__ count, uint32_t total) {
    const uint32_t SW = opt.width * opt.samples, SH = opt.height * opt.samples;
    const uint32_t frame = *opt.frame;
    const CameraDev cam = *camPtr;
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = total;
    for (uint32_t sid = blockIdx.x * blockDim.x + threadIdx.x; sid < total;
         sid += gridDim.x * blockDim.x) {
        const uint32_t sx = sid % SW, sy = sid / SW;
        Rand4 rc = philox_uniform4(sid, frame, kTagCamera, 0u, opt.seedLo, opt.seedHi);
        float dx = cam.planeSize[0] / static_cast<float>(SW);
        float dy = cam.planeSize[1] / static_cast<float>(SH);
        float sdx = static_cast<float>(sx) * dx;
        float sdy = static_cast<float>(sy) * dy;
        sdx += rc.u[0] * dx;
        sdy += rc.u[1] * dy;
        V3 sp = {cam.bottomLeft[0] + ((sdx * cam.right[0]) + (sdy * cam.up[0])),
                 cam.bottomLeft[1] + ((sdx * cam.right[1]) + (sdy * cam.up[1])),
                 cam.bottomLeft[2] + ((sdx * cam.right[2]) + (sdy * cam.up[2]))};
        V3 dir = normalize(sp - ld3(cam.position));
        rayO[sid] = make_float4(cam.position[0], cam.position[1], cam.position[2], cam.nearFar[0]);
        rayD[sid] = make_float4(dir.x, dir.y, dir.z, cam.nearFar[1]);
        RayAux a;
        a.rf[0] = a.rf[1] = a.rf[2] = 1.0f;
        a.sample = sid;
        a.endpoint = kInvalid;
        a.medium = static_cast<uint16_t>(baseMedium);
        a.depth = 0;
        a.type = kCameraRay;
        a.prevPDF = __int_as_float(0x7fc00000);
        a.pad = 0;
        aux[sid] = a;
        samples[sid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

__global__ void __launch_bounds__(256) k_dense_keys(const uint32_t* __restrict__ hitKey,
                                                    const uint32_t* __restrict__ dCount,
                                                    uint32_t idBits, uint32_t* __restrict__ dense,
                                                    PortionTable table) {
    const uint32_t n = *dCount;
    if (blockIdx.x == 0 && threadIdx.x < 8) {
        table.offset[threadIdx.x] = 0;
        table.end[threadIdx.x] = 0;
        if (threadIdx.x == 0) *table.nonNull = n;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t k = hitKey[i];
        dense[i] = ((k >> kIdBits) << idBits) | (k & ((1u << idBits) - 1u));
    }
}

// Batch boundaries of the sorted dense keys.  Each warp compares every key
// with its predecessor (shuffle, one global read at the warp edge), and the
// lanes where the batch changes write the portion bounds.
__global__ void __launch_bounds__(256) k_portions(const uint32_t* __restrict__ sortedDense,
                                                  const uint32_t* __restrict__ dCount,
                                                  uint32_t idBits, PortionTable table) {
    const uint32_t n = *dCount;
    const uint32_t lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const bool ok = i < n;
        const uint32_t b = ok ? (sortedDense[i] >> idBits) : 0xFFFFFFFFu;
        uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, b, 1);
        uint32_t next = __shfl_down_sync(0xFFFFFFFFu, b, 1);
        if (lane == 0) prev = (i > 0 && ok) ? (sortedDense[i - 1] >> idBits) : 0xFFFFFFFEu;
        if (lane == 31) next = (i + 1 < n) ? (sortedDense[i + 1] >> idBits) : 0xFFFFFFFEu;
        if (!ok) continue;
        if (i + 1 == n) next = 0xFFFFFFFEu;
        if (b != prev) {
            table.offset[b] = i;
            if (b == kBatchNull) *table.nonNull = i;
        }
        if (b != next) table.end[b] = i + 1;
    }
}

struct ShadeArgs {
    SceneDev sc;
    const float4* rayO;
    const float4* rayD;
    const RayAux* aux;
    HitIn hit;
    const uint32_t* sortedIds;
    const uint32_t* nonNull;
    float4* samples;
    PathOptions opt;
    int gen;
    float4* outO;
    float4* outD;
    RayAux* outAux;
    uint32_t* outCount;
};

__device__ __forceinline__ void accumulate(float4* samples, uint32_t s, V3 v) {
    float* p = reinterpret_cast<float*>(samples + s);
    atomicAdd(p + 0, v.x);
    atomicAdd(p + 1, v.y);
    atomicAdd(p + 2, v.z);
}

__global__ void __launch_bounds__(128) k_shade(ShadeArgs A) {
    const uint32_t n = *A.nonNull;
    const uint32_t frame = *A.opt.frame;
    const SceneDev& s = A.sc;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t ltMask = (1u << lane) - 1u;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const uint32_t j = base + threadIdx.x;
        bool emitNee = false, emitPath = false;
        float4 neeO, neeD, pathO, pathD;
        RayAux neeAux, pathAux;
        if (j < n) {
            const uint32_t rid = A.sortedIds[j];
            const uint32_t key = A.hit.key[rid];
            const uint32_t batch = key >> kIdBits, id = key & kIdMask;
            const float4 rd = A.rayD[rid];
            const RayAux aux = A.aux[rid];
            if (batch == kBatchLight) {
                // PathTracerBoundaryWork (PathTracerKC.cuh:335-426)
                const bool pathAsMis = A.opt.mis && aux.type == kPathRay;
                const bool camera = aux.type == kCameraRay;
                const bool specPath = aux.type == kSpecPathRay;
                const bool neeOn = A.opt.nee && aux.type == kNeeRay;
                const bool pathNeeOff =
                    (!A.opt.nee) && (aux.type == kPathRay || aux.type == kSpecPathRay);
                const bool correct = neeOn && (aux.endpoint == id);
                float misWeight = 1.0f;
                if (pathAsMis) {
                    // light pdf of this hit: GPULightSamplerUniform::Pdf and
                    // GPULight::Pdf(distance, position, direction, tbn)
                    const uint32_t prim = A.hit.prim[rid];
                    const float2 hb = A.hit.bary[rid];
                    const V3 d = {rd.x, rd.y, rd.z};
                    const Surface sf = gen_surface(s, prim, hb.x, hb.y, d);
                    const V3 dir = normalize(d);
                    float pdfM = 0.0f, pdfC = 0.0f;
                    if (id < s.lightCount) {
                        pdfM = 1.0f / static_cast<float>(s.lightCount);
                        const uint32_t i0 = s.idx[3 * prim], i1 = s.idx[3 * prim + 1],
                                       i2 = s.idx[3 * prim + 2];
                        const V3 p0 = ld3(s.pos + 3 * size_t(i0)), p1 = ld3(s.pos + 3 * size_t(i1)),
                                 p2 = ld3(s.pos + 3 * size_t(i2));
                        const V3 cr = cross(p1 - p0, p2 - p0);
                        const float area = sqrtf(dot(cr, cr)) * 0.5f;
                        const V3 ln = to_space(v3(0.0f, 0.0f, 1.0f), sf.w2t);
                        const float nDotL = fabsf(dot(ln, -dir));
                        const float dist = A.hit.t[rid];
                        pdfC = (1.0f / area) * dist * dist / nDotL;
                    }
                    misWeight = power_heuristic(aux.prevPDF, pdfC * pdfM);
                }
                if (pathNeeOff || pathAsMis || correct || camera || specPath) {
                    V3 total = ld3(s.lightRadiance + 3 * id) * v3(aux.rf[0], aux.rf[1], aux.rf[2]);
                    total = total * misWeight;
                    accumulate(A.samples, aux.sample, total);
                }
            } else if (aux.type != kNeeRay && A.gen) {
                // PathTracerPathWork (PathTracerKC.cuh:428-649)
                const uint32_t prim = A.hit.prim[rid];
                const float2 hb = A.hit.bary[rid];
                const V3 d = {rd.x, rd.y, rd.z};
                const Surface sf = gen_surface(s, prim, hb.x, hb.y, d);
                const V3 wi = -normalize(d);
                const V3 rf = {aux.rf[0], aux.rf[1], aux.rf[2]};
                bool specular;
                if (batch == kBatchLambert || batch == kBatchLambertC) specular = false;
                else if (batch == kBatchMetal) specular = (1.0f - s.metalParams[10 * id + 9]) >= 0.99f;
                else if (batch == kBatchUnreal) specular = (1.0f - s.unrealParams[6 * id + 3]) >= 0.99f;
                else specular = true;
                const Rand4 ra = philox_uniform4(aux.sample, frame, aux.depth, 0u,
                                                 A.opt.seedLo, A.opt.seedHi);
                const Rand4 rb = philox_uniform4(aux.sample, frame, aux.depth, 1u,
                                                 A.opt.seedLo, A.opt.seedHi);
                // ---- NEE: GPULightSamplerUniform::SampleLight + primitive light
                if (A.opt.nee && !specular && s.lightCount > 0) {
                    const uint32_t lc = s.lightCount;
                    float r1 = ra.u[0] * static_cast<float>(lc);
                    uint32_t li = static_cast<uint32_t>(r1);
                    if (li == lc) li--;
                    const uint32_t lp = s.lightPrim[li];
                    // TriangleSurfaceGenerator SamplePosition (GPUPrimitiveTriangle.h:65-115)
                    const float sx = sqrtf(ra.u[1]);
                    const float r2 = ra.u[2];
                    const float la = 1.0f - sx;
                    const float lb = (1.0f - r2) * sx;
                    const float lcw = sx * r2;
                    const uint32_t i0 = s.idx[3 * lp], i1 = s.idx[3 * lp + 1], i2 = s.idx[3 * lp + 2];
                    const V3 p0 = ld3(s.pos + 3 * size_t(i0)), p1 = ld3(s.pos + 3 * size_t(i1)),
                             p2 = ld3(s.pos + 3 * size_t(i2));
                    const V3 cr = cross(p1 - p0, p2 - p0);
                    const float area = sqrtf(dot(cr, cr)) * 0.5f;
                    float lpdf = 1.0f / area;
                    Q4 q = bary_slerp(qnormalize(q_from(__ldg(s.tbn + i0))),
                                      qnormalize(q_from(__ldg(s.tbn + i1))),
                                      qnormalize(q_from(__ldg(s.tbn + i2))), la, lb);
                    V3 ln = to_space(v3(0.0f, 0.0f, 1.0f), q);
                    const V3 lpos = (p0 * la + p1 * lb) + p2 * lcw;
                    ln = normalize(ln);
                    V3 ldir = lpos - sf.pos;
                    const float d2 = dot(ldir, ldir);
                    const float dist = sqrtf(d2);
                    ldir = ldir * (1.0f / dist);
                    const float nDotL = fabsf(dot(ln, -ldir));
                    lpdf *= d2 / nDotL;
                    lpdf *= (1.0f / static_cast<float>(lc));
                    V3 refl;
                    float pdfBxdf;
                    if (batch == kBatchLambert) {
                        refl = lambert_eval(ld3(s.lambertAlbedo + 3 * id), ldir, sf);
                        pdfBxdf = A.opt.mis ? lambert_pdf(ldir, sf) : 0.0f;
                    } else if (batch == kBatchLambertC) {
                        refl = lambertc_eval(ld3(s.lambertCAlbedo + 3 * id), ldir, sf);
                        pdfBxdf = A.opt.mis ? lambert_pdf(ldir, sf) : 0.0f;
                    } else if (batch == kBatchUnreal) {
                        const UnrealP up = unreal_params(s.unrealParams + 6 * id);
                        refl = unreal_eval(up, ldir, wi, sf);
                        pdfBxdf = A.opt.mis ? unreal_pdf(up, ldir, wi, sf) : 0.0f;
                    } else {
                        const MetalP mp = metal_params(s.metalParams + 10 * id);
                        refl = metal_eval(mp, ldir, wi, sf);
                        pdfBxdf = A.opt.mis ? metal_pdf(mp, ldir, wi, sf) : 0.0f;
                    }
                    float pdfNee = lpdf;
                    if (A.opt.mis) {
                        pdfNee /= power_heuristic(lpdf, pdfBxdf);
                        if (isnan(pdfNee)) pdfNee = 0.0f;
                    }
                    V3 nrf = rf * refl;
                    nrf = (pdfNee == 0.0f) ? v3(0.0f, 0.0f, 0.0f) : (nrf / pdfNee);
                    if (nonzero(nrf)) {
                        const V3 o = nudge(sf.pos, sf.geo);
                        emitNee = true;
                        neeO = make_float4(o.x, o.y, o.z, 0.0f);
                        neeD = make_float4(ldir.x, ldir.y, ldir.z, kFltMax);
                        neeAux = aux;
                        neeAux.rf[0] = nrf.x;
                        neeAux.rf[1] = nrf.y;
                        neeAux.rf[2] = nrf.z;
                        neeAux.endpoint = li;
                        neeAux.type = kNeeRay;
                        neeAux.prevPDF = __int_as_float(0x7fc00000);
                    }
                }
                // ---- BxDF sample
                BSample bs;
                if (batch == kBatchLambert) {
                    bs = lambert_sample(ld3(s.lambertAlbedo + 3 * id), sf, rb.u[0], rb.u[1],
                                        aux.medium);
                } else if (batch == kBatchLambertC) {
                    bs = lambertc_sample(ld3(s.lambertCAlbedo + 3 * id), sf, rb.u[0], rb.u[1],
                                         aux.medium);
                } else if (batch == kBatchUnreal) {
                    bs = unreal_sample(unreal_params(s.unrealParams + 6 * id), wi, sf, rb.u[2],
                                       rb.u[0], rb.u[1], aux.medium);
                } else if (batch == kBatchMetal) {
                    bs = metal_sample(metal_params(s.metalParams + 10 * id), wi, sf, rb.u[0],
                                      rb.u[1], aux.medium);
                } else {
                    bs = refract_sample(ld3(s.refractAlbedo + 3 * id), s.refractMedium[id], s, wi,
                                        sf, aux.medium, rb.u[0]);
                }
                V3 prf = rf * bs.refl;
                prf = (bs.pdf == 0.0f) ? v3(0.0f, 0.0f, 0.0f) : (prf / bs.pdf);
                const float avg = dot(prf, v3(0.333f, 0.333f, 0.333f));
                bool term = false;
                if (!specular && aux.depth > A.opt.rrStart) {
                    // TracerFunctions::RussianRoulette (TracerFunctions.cuh:320-331)
                    const float prob = fminf(fmaxf(avg, 0.005f), 1.0f);
                    if (ra.u[3] >= prob) term = true;
                    else prf = prf * (1.0f / prob);
                }
                if ((!term || specular) && nonzero(prf)) {
                    emitPath = true;
                    pathO = make_float4(bs.pos.x, bs.pos.y, bs.pos.z, 0.0f);
                    pathD = make_float4(bs.dir.x, bs.dir.y, bs.dir.z, kFltMax);
                    pathAux = aux;
                    pathAux.medium = static_cast<uint16_t>(bs.medium);
                    pathAux.rf[0] = prf.x;
                    pathAux.rf[1] = prf.y;
                    pathAux.rf[2] = prf.z;
                    pathAux.type = specular ? kSpecPathRay : kPathRay;
                    pathAux.prevPDF = bs.pdf;
                    pathAux.depth = static_cast<uint8_t>(aux.depth + 1);
                }
            }
        }
        // warp-aggregated compaction of the outputs into the next wavefront
        const uint32_t bN = __ballot_sync(0xFFFFFFFFu, emitNee);
        const uint32_t bP = __ballot_sync(0xFFFFFFFFu, emitPath);
        const uint32_t tot = __popc(bN) + __popc(bP);
        if (tot == 0) continue;
        uint32_t wbase = 0;
        if (lane == 0) wbase = atomicAdd(A.outCount, tot);
        wbase = __shfl_sync(0xFFFFFFFFu, wbase, 0);
        if (emitNee) {
            const uint32_t o = wbase + __popc(bN & ltMask);
            A.outO[o] = neeO;
            A.outD[o] = neeD;
            A.outAux[o] = neeAux;
        }
        if (emitPath) {
            const uint32_t o = wbase + __popc(bN) + __popc(bP & ltMask);
            A.outO[o] = pathO;
            A.outD[o] = pathD;
            A.outAux[o] = pathAux;
        }
    }
}

__global__ void __launch_bounds__(256) k_resolve(const float4* __restrict__ samples,
                                                 uint32_t width, uint32_t height, uint32_t sp,
                                                 float4* __restrict__ image) {
    const uint32_t SW = width * sp;
    const float inv = 1.0f / static_cast<float>(sp * sp);
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < width * height;
         p += gridDim.x * blockDim.x) {
        const uint32_t px = p % width, py = p / width;
        float r = 0.0f, g = 0.0f, b = 0.0f;
        for (uint32_t j = 0; j < sp; j++)
            for (uint32_t i = 0; i < sp; i++) {
                float4 v = samples[(py * sp + j) * SW + (px * sp + i)];
                r += v.x;
                g += v.y;
                b += v.z;
            }
        float4 acc = image[p];
        image[p] = make_float4(acc.x + r * inv, acc.y + g * inv, acc.z + b * inv, acc.w + 1.0f);
    }
}

__global__ void k_add_u64(unsigned long long* acc, const uint32_t* v) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *acc += *v;
}
__global__ void k_frame_advance(uint32_t* frame) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *frame += 1u;
}

inline uint32_t grid_for(uint32_t n, uint32_t block, uint32_t cap) {
    uint32_t g = (n + block - 1) / block;
    return g < cap ? (g ? g : 1) : cap;
}

}  // namespace

int camera_generate(const CameraDev* cam, const PathOptions& opt, uint32_t baseMedium,
                    float4* rayO, float4* rayD, RayAux* aux, float4* samples, uint32_t* count,
                    cudaStream_t stream) {
    const uint32_t total = opt.width * opt.samples * opt.height * opt.samples;
    k_camera<<<grid_for(total, 256, 148 * 16), 256, 0, stream>>>(cam, opt, baseMedium, rayO, rayD,
                                                                aux, samples, count, total);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int dense_keys(const uint32_t* hitKey, const uint32_t* dCount, uint32_t maxCount, uint32_t idBits,
               uint32_t* dense, const PortionTable& table, cudaStream_t stream) {
    k_dense_keys<<<grid_for(maxCount, 256, 148 * 8), 256, 0, stream>>>(hitKey, dCount, idBits, dense,
                                                                      table);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int find_portions(const uint32_t* sortedDense, const uint32_t* dCount, uint32_t maxCount,
                  uint32_t idBits, const PortionTable& table, cudaStream_t stream) {
    k_portions<<<grid_for(maxCount, 256, 148 * 8), 256, 0, stream>>>(sortedDense, dCount, idBits,
                                                                    table);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int shade(const SceneDev& sc, const float4* rayO, const float4* rayD, const RayAux* aux,
          const HitIn& hit, const uint32_t* sortedIds, const uint32_t* nonNull, uint32_t maxCount,
          float4* samples, const PathOptions& opt, bool gen, float4* outO, float4* outD,
          RayAux* outAux, uint32_t* outCount, cudaStream_t stream) {
    ShadeArgs a{sc,   rayO,    rayD, aux,  hit,  sortedIds, nonNull, samples,
                opt,  gen ? 1 : 0, outO, outD, outAux, outCount};
    k_shade<<<grid_for(maxCount, 128, 148 * 16), 128, 0, stream>>>(a);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int resolve(const float4* samples, uint32_t width, uint32_t height, uint32_t sp, float4* image,
            cudaStream_t stream) {
    k_resolve<<<grid_for(width * height, 256, 148 * 8), 256, 0, stream>>>(samples, width, height,
                                                                         sp, image);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int add_count(unsigned long long* acc, const uint32_t* v, cudaStream_t stream) {
    k_add_u64<<<1, 32, 0, stream>>>(acc, v);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int frame_advance(uint32_t* frame, cudaStream_t stream) {
    k_frame_advance<<<1, 32, 0, stream>>>(frame);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb
