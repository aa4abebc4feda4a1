// Surface generation and the BxDFs of the wavefront core, shared by the
// shading kernel and the path-guiding kernels:
//   gen_surface   TriangleSurfaceGenerator::GenBasicSurface
//                 (GPUPrimitiveTriangle.h:624-700)
//   Lambert       LambertMatFuncs (LambertMaterialKC.cuh:14-103)
//   LambertC      LambertConstFuncs (SimpleMaterialsKC.cuh:16-103)
//   Metal         MetalMatFuncs (MetalGlassMaterialsKC.cuh:11-222)
//   Unreal        UnrealDeviceFuncs (UnrealMaterialKC.cuh:19-359)
//   Refract       RefractMatFuncs (SimpleMaterialsKC.cuh:172-302)
// and the material dispatch by HitKey batch used where one kernel sees
// every material.
#pragma once
#include "common.cuh"

namespace mrb {

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
__device__ inline BSample metal_sample(const MetalP& m, V3 wi, const Surface& sf, float xi0, float xi1,
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
__device__ inline V3 metal_eval(const MetalP& m, V3 wo, V3 wi, const Surface& sf) {
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
__device__ inline BSample refract_sample(V3 albedo, uint32_t matMedium, const SceneDev& s, V3 wi,
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
__device__ inline float metal_pdf(const MetalP& m, V3 wo, V3 wi, const Surface& sf) {
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
__device__ inline BSample unreal_sample(const UnrealP& m, V3 wi, const Surface& sf, float xiSel,
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
__device__ inline V3 unreal_eval(const UnrealP& m, V3 wo, V3 wi, const Surface& sf) {
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
__device__ inline float unreal_pdf(const UnrealP& m, V3 wo, V3 wi, const Surface& sf) {
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


// ---------------------------------------------------------------------------
// dispatch by batch (the MGroup static functions of each material)
// ---------------------------------------------------------------------------
// Specularity >= SPECULAR_THRESHOLD (TracerConstants.h:6): Metal and Unreal
// give 1 - roughness, Lambert(C) 0, Refract 1.
__device__ __forceinline__ bool mat_specular(const SceneDev& s, uint32_t batch, uint32_t id) {
    if (batch == kBatchLambert || batch == kBatchLambertC) return false;
    if (batch == kBatchMetal) return (1.0f - s.metalParams[10 * id + 9]) >= 0.99f;
    if (batch == kBatchUnreal) return (1.0f - s.unrealParams[6 * id + 3]) >= 0.99f;
    return true;
}
__device__ inline V3 mat_eval(const SceneDev& s, uint32_t batch, uint32_t id, V3 wo, V3 wi,
                              const Surface& sf) {
    if (batch == kBatchLambert) return lambert_eval(ld3(s.lambertAlbedo + 3 * id), wo, sf);
    if (batch == kBatchLambertC) return lambertc_eval(ld3(s.lambertCAlbedo + 3 * id), wo, sf);
    if (batch == kBatchUnreal) return unreal_eval(unreal_params(s.unrealParams + 6 * id), wo, wi, sf);
    if (batch == kBatchMetal) return metal_eval(metal_params(s.metalParams + 10 * id), wo, wi, sf);
    return v3(0.0f, 0.0f, 0.0f);
}
__device__ inline float mat_pdf(const SceneDev& s, uint32_t batch, uint32_t id, V3 wo, V3 wi,
                                const Surface& sf) {
    if (batch == kBatchLambert || batch == kBatchLambertC) return lambert_pdf(wo, sf);
    if (batch == kBatchUnreal) return unreal_pdf(unreal_params(s.unrealParams + 6 * id), wo, wi, sf);
    if (batch == kBatchMetal) return metal_pdf(metal_params(s.metalParams + 10 * id), wo, wi, sf);
    return 0.0f;
}
// BxDF sample from three uniforms (u0, u1: direction; u2: Unreal lobe /
// Refract reflect-or-refract choice)
__device__ inline BSample mat_sample(const SceneDev& s, uint32_t batch, uint32_t id, V3 wi,
                                     const Surface& sf, uint32_t medium, float u0, float u1,
                                     float u2) {
    if (batch == kBatchLambert) return lambert_sample(ld3(s.lambertAlbedo + 3 * id), sf, u0, u1, medium);
    if (batch == kBatchLambertC)
        return lambertc_sample(ld3(s.lambertCAlbedo + 3 * id), sf, u0, u1, medium);
    if (batch == kBatchUnreal)
        return unreal_sample(unreal_params(s.unrealParams + 6 * id), wi, sf, u2, u0, u1, medium);
    if (batch == kBatchMetal) return metal_sample(metal_params(s.metalParams + 10 * id), wi, sf, u0, u1, medium);
    return refract_sample(ld3(s.refractAlbedo + 3 * id), s.refractMedium[id], s, wi, sf, medium, u0);
}

}  // namespace mrb
