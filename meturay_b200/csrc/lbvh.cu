// LBVH construction for the "LBVH" triangle accelerator group.
//
// Kernels (all device-resident, no host round trip between them):
//   k_tri_bounds    per-triangle AABB + scene extent (min/max reduce)
//   k_morton        Morton code of each AABB centroid (LinearBVH.hpp:118-166,
//                   delta from FindMortonDelta, LinearBVH.hpp:398-414)
//   (onesweep sort of (code, index), sort.cu)
//   k_lbvh_build    single-pass bottom-up hierarchy + AABBs: each leaf walks
//                   up, choosing its parent exactly as ChooseParentAndUpdate
//                   (LinearBVH.hpp:30-100) does; the second child to reach a
//                   parent continues with the parent's range and box
//                   (Apetrei 2014).  Replaces the reference's CDP polling
//                   loops (LinearBVH.hpp:249-288,365-396) with one launch.
//   k_gather_tris   triangles in Morton order with precomputed edges.
// The node arrays in reference numbering (leaves 0..n-1, inner n..2n-2) are
// kept for parity checks; the traversal reads the 64-byte BvhNode layout.
#include "common.cuh"
#include "lbvh.cuh"
#include "sort.cuh"

namespace mrb {

namespace {

__device__ __forceinline__ void atomic_min_f(float* a, float v) {
    if (v >= 0.0f) atomicMin(reinterpret_cast<int*>(a), __float_as_int(v));
    else atomicMax(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f(float* a, float v) {
    if (v >= 0.0f) atomicMax(reinterpret_cast<int*>(a), __float_as_int(v));
    else atomicMin(reinterpret_cast<unsigned*>(a), __float_as_uint(v));
}

__global__ void k_extent_init(float* extent) {
    if (threadIdx.x < 3) extent[threadIdx.x] = __int_as_float(0x7f800000);
    else if (threadIdx.x < 6) extent[threadIdx.x] = __int_as_float(0xff800000);
}

// Triangle::BoundingBox per triangle, then the extent reduce
// (ReduceArrayGPU<AABB3f>, LinearBVH.hpp:452-457).
__global__ void __launch_bounds__(256) k_tri_bounds(const float* __restrict__ pos,
                                                    const uint32_t* __restrict__ idx, uint32_t n,
                                                    float* __restrict__ aabb, float* extent) {
    __shared__ float red[6][8];
    float lo[3] = {__int_as_float(0x7f800000), __int_as_float(0x7f800000),
                   __int_as_float(0x7f800000)};
    float hi[3] = {-lo[0], -lo[1], -lo[2]};
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        uint32_t i0 = idx[3 * t], i1 = idx[3 * t + 1], i2 = idx[3 * t + 2];
        float* a = aabb + 6 * size_t(t);
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float v0 = pos[3 * size_t(i0) + c], v1 = pos[3 * size_t(i1) + c],
                  v2 = pos[3 * size_t(i2) + c];
            float mn = fminf(fminf(v0, v1), v2), mx = fmaxf(fmaxf(v0, v1), v2);
            a[c] = mn;
            a[3 + c] = mx;
            lo[c] = fminf(lo[c], mn);
            hi[c] = fmaxf(hi[c], mx);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[c] = fminf(lo[c], __shfl_xor_sync(0xFFFFFFFFu, lo[c], o));
            hi[c] = fmaxf(hi[c], __shfl_xor_sync(0xFFFFFFFFu, hi[c], o));
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        for (int c = 0; c < 3; c++) {
            red[c][warp] = lo[c];
            red[3 + c][warp] = hi[c];
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int c = threadIdx.x;
        float v = red[c][0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++)
            v = (c < 3) ? fminf(v, red[c][w]) : fmaxf(v, red[c][w]);
        if (c < 3) atomic_min_f(extent + c, v);
        else atomic_max_f(extent + c, v);
    }
}

__device__ __forceinline__ uint64_t expand3d(uint32_t val) {  // MortonCode.h:45-56
    uint64_t x = val;
    x &= 0x1fffff;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

__global__ void __launch_bounds__(256) k_morton(const float* __restrict__ aabb, uint32_t n,
                                                const float* __restrict__ extent,
                                                uint64_t* __restrict__ codes,
                                                uint32_t* __restrict__ iota, float* deltaOut) {
    __shared__ float sExt[6];
    __shared__ float sDelta;
    if (threadIdx.x < 6) sExt[threadIdx.x] = extent[threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        // FindMortonDelta: largest span / 2^21, in double, then to float
        const double res = 1.0 / 2097152.0;
        double dx = static_cast<double>(sExt[3] - sExt[0]) * res;
        double dy = static_cast<double>(sExt[4] - sExt[1]) * res;
        double dz = static_cast<double>(sExt[5] - sExt[2]) * res;
        sDelta = static_cast<float>(fmax(fmax(dx, dy), dz));
        if (blockIdx.x == 0 && deltaOut) *deltaOut = sDelta;
    }
    __syncthreads();
    const float d = sDelta;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const float* a = aabb + 6 * size_t(t);
        uint32_t g[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float span = a[3 + c] - a[c];
            float center = a[c] + span * 0.5f;
            float rel = center - sExt[c];
            g[c] = static_cast<uint32_t>(floorf(rel / d));
        }
        codes[t] = expand3d(g[0]) | (expand3d(g[1]) << 1) | (expand3d(g[2]) << 2);
        if (iota) iota[t] = t;
    }
}

// Delta of LinearBVH.hpp:30-39 with the index-augmented tie break for equal
// codes (Karras 2012, section 4); identical to the reference for unique codes.
__device__ __forceinline__ uint32_t lbvh_delta(const uint64_t* __restrict__ c, uint32_t i) {
    uint64_t d = c[i] ^ c[i + 1];
    if (d != 0) return static_cast<uint32_t>(__clzll(static_cast<long long>(d)));
    return 64u + static_cast<uint32_t>(__clz(static_cast<int>(i ^ (i + 1))));
}

__device__ __forceinline__ void write_child(BvhNode* nodes, uint32_t p, int slot, int enc,
                                            const float lo[3], const float hi[3]) {
    BvhNode* nd = nodes + p;
    if (slot == 0) {
        nd->a = make_float4(lo[0], hi[0], lo[1], hi[1]);
        reinterpret_cast<float2*>(&nd->c)[0] = make_float2(lo[2], hi[2]);
        nd->d.x = enc;
    } else {
        nd->b = make_float4(lo[0], hi[0], lo[1], hi[1]);
        reinterpret_cast<float2*>(&nd->c)[1] = make_float2(lo[2], hi[2]);
        nd->d.y = enc;
    }
}

__global__ void __launch_bounds__(256) k_lbvh_build(
    const uint64_t* __restrict__ codes, const uint32_t* __restrict__ sortedIdx,
    const float* __restrict__ triAabb, uint32_t n, uint32_t* left, uint32_t* right,
    uint32_t* parent, float* inner, uint32_t* rangeLo, uint32_t* rangeHi, uint32_t* flags,
    uint32_t* root, BvhNode* nodes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t lo = i, hi = i, cur = i;
    float blo[3], bhi[3];
    {
        const float* a = triAabb + 6 * size_t(sortedIdx[i]);
        for (int c = 0; c < 3; c++) {
            blo[c] = a[c];
            bhi[c] = a[3 + c];
        }
    }
    int enc = ~static_cast<int>(i);
    for (;;) {
        if (lo == 0 && hi == n - 1) {
            *root = cur;
            parent[cur] = kInvalid;
            break;
        }
        const uint32_t ld = (lo == 0) ? 0u : lbvh_delta(codes, lo - 1);
        const uint32_t rd = (hi == n - 1) ? 0u : lbvh_delta(codes, hi);
        uint32_t p;
        int slot;
        if (rd > ld) {  // parent is the right range end: we are its left child
            p = hi;
            slot = 0;
            left[p] = cur;
            rangeLo[p] = lo;
        } else {        // parent is lo - 1: we are its right child
            p = lo - 1;
            slot = 1;
            right[p] = cur;
            rangeHi[p] = hi;
        }
        parent[cur] = n + p;
        write_child(nodes, p, slot, enc, blo, bhi);
        __threadfence();
        if (atomicAdd(flags + p, 1u) == 0u) break;  // sibling not done yet
        __threadfence();
        // second arrival: finish the parent
        if (slot == 0) hi = __ldcg(rangeHi + p);
        else lo = __ldcg(rangeLo + p);
        const BvhNode* nd = nodes + p;
        float4 ob = (slot == 0) ? __ldcg(&nd->b) : __ldcg(&nd->a);
        float2 oz = __ldcg(reinterpret_cast<const float2*>(&nd->c) + (slot == 0 ? 1 : 0));
        blo[0] = fminf(blo[0], ob.x);
        bhi[0] = fmaxf(bhi[0], ob.y);
        blo[1] = fminf(blo[1], ob.z);
        bhi[1] = fmaxf(bhi[1], ob.w);
        blo[2] = fminf(blo[2], oz.x);
        bhi[2] = fmaxf(bhi[2], oz.y);
        // BottomUpAABBInter (LinearBVH.hpp:308-363): union(left, right)
        float* o = inner + 6 * size_t(p);
        for (int c = 0; c < 3; c++) {
            o[c] = blo[c];
            o[3 + c] = bhi[c];
        }
        cur = n + p;
        enc = static_cast<int>(p);
    }
}

__global__ void __launch_bounds__(256) k_gather_tris(const float* __restrict__ pos,
                                                     const uint32_t* __restrict__ idx,
                                                     const uint32_t* __restrict__ key,
                                                     const uint8_t* __restrict__ cull,
                                                     const uint32_t* __restrict__ sortedIdx,
                                                     uint32_t n, float4* tv0, float4* te0,
                                                     float4* te1) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        uint32_t t = sortedIdx[s];
        uint32_t i0 = idx[3 * size_t(t)], i1 = idx[3 * size_t(t) + 1], i2 = idx[3 * size_t(t) + 2];
        V3 p0 = ld3(pos + 3 * size_t(i0)), p1 = ld3(pos + 3 * size_t(i1)),
           p2 = ld3(pos + 3 * size_t(i2));
        V3 e0 = p1 - p0, e1 = p2 - p0;
        tv0[s] = make_float4(p0.x, p0.y, p0.z, __uint_as_float(t));
        te0[s] = make_float4(e0.x, e0.y, e0.z, __uint_as_float(key[t]));
        te1[s] = make_float4(e1.x, e1.y, e1.z, __uint_as_float(cull ? uint32_t(cull[t]) : 0u));
    }
}

}  // namespace

int lbvh_morton(const float* pos, const uint32_t* idx, uint32_t n, float* triAabb, float* extent,
                uint64_t* codes, uint32_t* iota, float* deltaOut, cudaStream_t stream) {
    if (n == 0) return 0;
    const int grid = static_cast<int>(std::min<uint32_t>((n + 255) / 256, 148u * 8u));
    k_extent_init<<<1, 32, 0, stream>>>(extent);
    k_tri_bounds<<<grid, 256, 0, stream>>>(pos, idx, n, triAabb, extent);
    k_morton<<<grid, 256, 0, stream>>>(triAabb, n, extent, codes, iota, deltaOut);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int lbvh_hierarchy(const uint64_t* sortedCodes, const uint32_t* sortedIdx, const float* triAabb,
                   uint32_t n, const LbvhArrays& a, cudaStream_t stream) {
    if (n < 2) {
        if (n == 1) {
            MRB_CUDA(cudaMemsetAsync(a.root, 0, 4, stream));
            MRB_CUDA(cudaMemsetAsync(a.parent, 0xFF, 4, stream));
        }
        return 0;
    }
    MRB_CUDA(cudaMemsetAsync(a.flags, 0, size_t(n - 1) * 4, stream));
    k_lbvh_build<<<(n + 255) / 256, 256, 0, stream>>>(sortedCodes, sortedIdx, triAabb, n, a.left,
                                                      a.right, a.parent, a.inner, a.rangeLo,
                                                      a.rangeHi, a.flags, a.root, a.nodes);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int lbvh_gather(const float* pos, const uint32_t* idx, const uint32_t* key, const uint8_t* cull,
                const uint32_t* sortedIdx, uint32_t n, float4* tv0, float4* te0, float4* te1,
                cudaStream_t stream) {
    if (n == 0) return 0;
    const int grid = static_cast<int>(std::min<uint32_t>((n + 255) / 256, 148u * 8u));
    k_gather_tris<<<grid, 256, 0, stream>>>(pos, idx, key, cull, sortedIdx, n, tv0, te0, te1);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb
