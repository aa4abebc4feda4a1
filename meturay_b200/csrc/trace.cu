// Closest-hit traversal of the LBVH (GPUAccBVHGroup::Hit replacement;
// reference kernel KCIntersectBVH, GPUAcceleratorBVHKC.cuh:229-346, with
// AcceptHit, GPUAcceleratorCommonKC.cuh:35-78, and Moller-Trumbore,
// RayLib/Ray.hpp:143-184).
//
// Layout: inner nodes hold both child boxes (one 64-byte node = four 16-byte
// vector loads); triangles are stored in Morton order as v0 / e0 / e1
// float4 triples with the original index, HitKey and cull flag in .w.  At
// each inner node both child boxes are tested against the current closest
// distance, the nearer child is entered and the farther pushed (ties enter
// the left child).  The per-thread stack lives in local memory (L1).
#include "common.cuh"
#include "trace.cuh"

namespace mrb {

namespace {

constexpr int kStack = 96;

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

// kCount: also count inner nodes visited and triangles tested (for the
// algorithmic-bytes figure of the roofline); results are unchanged.
template <bool kCount>
__global__ void __launch_bounds__(128) k_trace(AccelDev acc, const float4* __restrict__ rayO,
                                               const float4* __restrict__ rayD,
                                               const uint32_t* __restrict__ dCount,
                                               uint32_t hCount, HitOut out, uint32_t* errorFlag,
                                               unsigned long long* counters) {
    const uint32_t n = dCount ? *dCount : hCount;
    uint32_t nodeVisits = 0, triTests = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 ro = rayO[i], rd = rayD[i];
        const V3 o = {ro.x, ro.y, ro.z}, d = {rd.x, rd.y, rd.z};
        const float tmin = ro.w;
        float closest = rd.w;
        int hitTri = -1;
        float hb0 = 0.0f, hb1 = 0.0f;
        if (acc.triCount == 1) {
            if (kCount) triTests++;
            tri_test(acc, 0, o, d, tmin, closest, hitTri, hb0, hb1);
        } else if (acc.triCount > 1) {
            const V3 inv = {1.0f / safe_dir(d.x), 1.0f / safe_dir(d.y), 1.0f / safe_dir(d.z)};
            const V3 ooi = {o.x * inv.x, o.y * inv.y, o.z * inv.z};
            int stack[kStack];
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
                        if (sp < kStack) stack[sp++] = swap ? nd.x : nd.y;
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
        if (hitTri >= 0) {
            out.key[i] = __float_as_uint(__ldg(&acc.te0[hitTri].w));
            out.prim[i] = __float_as_uint(__ldg(&acc.tv0[hitTri].w));
            out.t[i] = closest;
            out.bary[i] = make_float2(hb0, hb1);
        } else {
            out.key[i] = kBatchNull;
            out.prim[i] = kInvalid;
            out.t[i] = closest;
            out.bary[i] = make_float2(0.0f, 0.0f);
        }
    }
    if (kCount) {
        unsigned long long a = nodeVisits, b = triTests;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
            b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(counters + 0, a);
            atomicAdd(counters + 1, b);
        }
    }
}

}  // namespace

int trace_closest(const AccelDev& acc, const float4* rayO, const float4* rayD,
                  const uint32_t* dCount, uint32_t maxCount, const HitOut& out,
                  uint32_t* errorFlag, cudaStream_t stream, unsigned long long* counters) {
    if (maxCount == 0) return 0;
    uint32_t blocks = (maxCount + 127) / 128;
    blocks = blocks < 148u * 16u ? blocks : 148u * 16u;
    if (counters)
        k_trace<true><<<blocks, 128, 0, stream>>>(acc, rayO, rayD, dCount, maxCount, out,
                                                  errorFlag, counters);
    else
        k_trace<false><<<blocks, 128, 0, stream>>>(acc, rayO, rayD, dCount, maxCount, out,
                                                   errorFlag, nullptr);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb
