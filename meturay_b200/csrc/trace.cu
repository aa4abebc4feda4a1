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
#include "trace_dev.cuh"

namespace mrb {

namespace {

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
        trace_ray<kCount>(acc, o, d, tmin, closest, hitTri, hb0, hb1, errorFlag, nodeVisits,
                          triTests);
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
