// Per-ray closest-hit traversal of one binary LBVH (AccelDev), shared by
// the wavefront traversal kernel and the accelerator-group Hit kernel.
// Reference: KCIntersectBVH (GPUAcceleratorBVHKC.cuh:229-346) with AcceptHit
// (GPUAcceleratorCommonKC.cuh:35-78) and Moller-Trumbore (RayLib/Ray.hpp:
// 143-184).
#pragma once
#include "common.cuh"

namespace mrb {

constexpr int kTraceStack = 96;

__device__ __forceinline__ float safe_dir(float d) {
    return (fabsf(d) > 1e-20f) ? d : copysignf(1e-20f, d);
}

__device__ __forceinline__ bool box_hit(float lx, float hx, float ly, float hy, float lz, float hz,
                                        V3 inv, V3 ooi, float tmin, float tmax, float& tn) {
    float ax = __fmaf_rn(lx, inv.x, -ooi.x), bx = __fmaf_rn(hx, inv.x, -ooi.x);
    float ay = __fmaf_rn(ly, inv.y, -ooi.y), by = __fmaf_rn(hy, inv.y, -ooi.y);
    float az = __fmaf_rn(lz, inv.z, -ooi.z), bz = __fmaf_rn(hz, inv.z, -ooi.z);
    float tlx = fminf(ax, bx), thx = fmaxf(ax, bx);
    float tly = fminf(ay, by), thy = fmaxf(ay, by);
    float tlz = fminf(az, bz), thz = fmaxf(az, bz);
    tn = fmaxf(fmaxf(tlx, tly), fmaxf(tlz, tmin));
    float tf = fminf(fminf(thx, thy), fminf(thz, tmax));
    return tn <= tf;
}

// Ray::IntersectsTriangle with the reference's epsilons; writes the hit if
// t lies in [tmin, closest).
__device__ __forceinline__ void tri_test(const AccelDev& acc, int s, V3 o, V3 d, float tmin,
                                         float& closest, int& hitTri, float& hb0, float& hb1) {
    float4 a = __ldg(acc.tv0 + s), b = __ldg(acc.te0 + s), c = __ldg(acc.te1 + s);
    V3 v0 = {a.x, a.y, a.z}, e0 = {b.x, b.y, b.z}, e1 = {c.x, c.y, c.z};
    bool cull = __float_as_uint(c.w) != 0u;
    V3 p = cross(d, e1);
    float det = dot(e0, p);
    if ((cull && (det < 1.0e-7f)) || (fabsf(det) < 1.0e-7f)) return;
    float invDet = 1.0f / det;
    V3 tv = o - v0;
    float u = dot(tv, p) * invDet;
    if (u < 0.0f || u > 1.0f) return;
    V3 q = cross(tv, e0);
    float v = dot(d, q) * invDet;
    if ((v < 0.0f) || (v + u) > 1.0f) return;
    float t = dot(e1, q) * invDet;
    if (t <= 1.0e-7f) return;
    if (t >= tmin && t < closest) {
        closest = t;
        hitTri = s;
        hb0 = 1.0f - u - v;
        hb1 = u;
    }
}

// Closest hit of one ray in [tmin, closest): at each inner node both child
// boxes are tested against the current closest distance, the nearer child
// is entered and the farther pushed (ties enter the left child).  hitTri is
// the sorted triangle slot (-1: no hit closer than `closest`).
template <bool kCount>
__device__ __forceinline__ void trace_ray(const AccelDev& acc, V3 o, V3 d, float tmin,
                                          float& closest, int& hitTri, float& hb0, float& hb1,
                                          uint32_t* errorFlag, uint32_t& nodeVisits,
                                          uint32_t& triTests) {
    if (acc.triCount == 1) {
        if (kCount) triTests++;
        tri_test(acc, 0, o, d, tmin, closest, hitTri, hb0, hb1);
    } else if (acc.triCount > 1) {
        const V3 inv = {1.0f / safe_dir(d.x), 1.0f / safe_dir(d.y), 1.0f / safe_dir(d.z)};
        const V3 ooi = {o.x * inv.x, o.y * inv.y, o.z * inv.z};
        int stack[kTraceStack];
        int sp = 0;
        int node = acc.root;
        for (;;) {
            if (node >= 0) {
                if (kCount) nodeVisits++;
                const float4* np = reinterpret_cast<const float4*>(acc.nodes + node);
                const float4 na = __ldg(np), nb = __ldg(np + 1), nc = __ldg(np + 2);
                const int4 nd = __ldg(reinterpret_cast<const int4*>(np + 3));
                float tn0, tn1;
                const bool h0 = box_hit(na.x, na.y, na.z, na.w, nc.x, nc.y, inv, ooi, tmin,
                                        closest, tn0);
                const bool h1 = box_hit(nb.x, nb.y, nb.z, nb.w, nc.z, nc.w, inv, ooi, tmin,
                                        closest, tn1);
                if (h0 && h1) {
                    const bool swap = tn1 < tn0;
                    if (sp < kTraceStack) stack[sp++] = swap ? nd.x : nd.y;
                    else atomicExch(errorFlag, 2u);
                    node = swap ? nd.y : nd.x;
                    continue;
                } else if (h0) {
                    node = nd.x;
                    continue;
                } else if (h1) {
                    node = nd.y;
                    continue;
                }
            } else {
                if (kCount) triTests++;
                tri_test(acc, ~node, o, d, tmin, closest, hitTri, hb0, hb1);
            }
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
}

}  // namespace mrb
