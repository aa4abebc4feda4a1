// Accelerator group of triangle surfaces and the base (top-level)
// accelerator: the interface MRay's ray caster drives
// (GPUAcceleratorGroupI / GPUBaseAcceleratorI, GPUAcceleratorI.h:46-173;
// RayCasterCUDA::HitRays, RayCasterCUDA.cu:35-166).
//
// Group: every surface (a range of the group's triangles with one
// local-to-world transform) gets its own binary LBVH in local space, built
// by the same Morton / onesweep / hierarchy kernels as the scene's LBVH.
// Hit (KCIntersectBVH, GPUAcceleratorBVHKC.cuh:229-346) takes RayGMem rays
// (position, tMin, direction, tMax: 32 B) through a RayId indirection and an
// accelerator key per ray, moves the ray into the surface's local space with
// the inverse transform (direction not renormalised, so t is shared), runs
// the per-ray binary traversal and, for a hit closer than the ray's tMax,
// writes tMax back in place together with the material key, the transform
// id, the 64-bit primitive id and the barycentrics (TriangleHit).
//
// Base: a binary BVH over the surfaces' world AABBs, built on the host
// (there are few surfaces), with a resumable traversal: each Hit call moves
// every ray from where it stopped to the next surface whose box it crosses
// in [tMin, tMax] (left-first order, pruned by the tMax that the group's Hit
// has shrunk meanwhile) and writes that surface's accelerator key, or 0
// (the null batch) once the traversal is over.  The reference keeps a
// 27-level bit stack per ray (KCIntersectBaseBVH, GPUAcceleratorBVHKC.cuh:
// 513-652); parent links make one node index per ray enough here.
//
// The tracers' own frames do not go through this interface: they trace
// their wavefronts with one traversal launch per depth over the scene's
// world-space tree (trace.cu, wide.cu).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/mrb200.h"
#include "common.cuh"
#include "lbvh.cuh"
#include "objects.cuh"
#include "sort.cuh"
#include "svo.cuh"
#include "trace_dev.cuh"

namespace mrb {
namespace {

constexpr uint32_t kDone = 0xFFFFFFFFu;

struct SurfaceDev {
    AccelDev acc;       // local-space LBVH of the surface
    uint32_t triBegin;  // group index of the surface's first triangle
    uint32_t transform; // global transform index
};

struct BaseNode {
    float lo[3], hi[3];
    uint32_t left, right, parent;  // node indices; left = kDone for a leaf
    uint32_t key;                  // accelerator key of a leaf
};

__global__ void __launch_bounds__(128) k_group_hit(
    const SurfaceDev* __restrict__ surf, uint32_t surfCount, const float* __restrict__ w2l,
    const unsigned long long* __restrict__ primTable, uint32_t* matKeys, uint32_t* transformIds,
    unsigned long long* primIds, char* hits, uint32_t hitStride, float4* rays,
    const uint32_t* __restrict__ rayIds, const uint32_t* __restrict__ accKeys, uint32_t n,
    uint32_t* errorFlag) {
    uint32_t nv = 0, tt = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t id = rayIds[i];
        const uint32_t acc = accKeys[i] & ((1u << kIdBits) - 1u);
        if (acc >= surfCount) continue;
        const SurfaceDev s = surf[acc];
        const float4 ro = rays[2 * size_t(id)], rd = rays[2 * size_t(id) + 1];
        const float* m = w2l + 12 * size_t(s.transform);
        const V3 o = xform_point(m, v3(ro.x, ro.y, ro.z));
        const V3 d = xform_dir(m, v3(rd.x, rd.y, rd.z));
        float closest = rd.w;
        int hitTri = -1;
        float hb0 = 0.0f, hb1 = 0.0f;
        trace_ray<false>(s.acc, o, d, ro.w, closest, hitTri, hb0, hb1, errorFlag, nv, tt);
        if (hitTri >= 0) {
            reinterpret_cast<float*>(rays + 2 * size_t(id) + 1)[3] = closest;
            float* h = reinterpret_cast<float*>(hits + size_t(id) * hitStride);
            h[0] = hb0;
            h[1] = hb1;
            transformIds[id] = s.transform;
            matKeys[id] = __float_as_uint(__ldg(&s.acc.te0[hitTri].w));
            const uint32_t t = s.triBegin + __float_as_uint(__ldg(&s.acc.tv0[hitTri].w));
            primIds[id] = primTable ? primTable[t] : static_cast<unsigned long long>(t);
        }
    }
}

__device__ __forceinline__ uint32_t base_next(const BaseNode* __restrict__ nodes, uint32_t node) {
    while (node != 0u) {
        const uint32_t p = nodes[node].parent;
        if (nodes[p].left == node) return nodes[p].right;
        node = p;
    }
    return kDone;
}

__global__ void __launch_bounds__(128) k_base_hit(const BaseNode* __restrict__ nodes,
                                                  uint32_t nodeCount, uint32_t* states,
                                                  uint32_t* keys, const float4* __restrict__ rays,
                                                  const uint32_t* __restrict__ rayIds, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t id = rayIds[i];
        uint32_t node = states[id];
        uint32_t key = kBatchNull;
        if (node != kDone) {
            const float4 ro = rays[2 * size_t(id)], rd = rays[2 * size_t(id) + 1];
            const V3 inv = {1.0f / safe_dir(rd.x), 1.0f / safe_dir(rd.y), 1.0f / safe_dir(rd.z)};
            const V3 ooi = {ro.x * inv.x, ro.y * inv.y, ro.z * inv.z};
            // every node is entered at most once per call
            for (uint32_t step = 0; step <= nodeCount && node != kDone; step++) {
                const BaseNode b = nodes[node];
                float tn;
                if (box_hit(b.lo[0], b.hi[0], b.lo[1], b.hi[1], b.lo[2], b.hi[2], inv, ooi, ro.w,
                            rd.w, tn)) {
                    if (b.left == kDone) {
                        key = b.key;
                        node = base_next(nodes, node);
                        break;
                    }
                    node = b.left;
                } else {
                    node = base_next(nodes, node);
                }
            }
            if (key == kBatchNull) node = kDone;
            states[id] = node;
        }
        keys[i] = key;
    }
}

// TriFunctions::Area (GPUPrimitiveTriangle.h:321-343) in world space
__device__ __forceinline__ float tri_world_area(const float* pos, const uint32_t* idx,
                                                const float* m, uint32_t t, V3& p0, V3& p1,
                                                V3& p2) {
    p0 = xform_point(m, ld3(pos + 3 * size_t(idx[3 * size_t(t)])));
    p1 = xform_point(m, ld3(pos + 3 * size_t(idx[3 * size_t(t) + 1])));
    p2 = xform_point(m, ld3(pos + 3 * size_t(idx[3 * size_t(t) + 2])));
    const V3 c = cross(p1 - p0, p2 - p0);
    return sqrtf(dot(c, c)) * 0.5f;
}

__global__ void k_tri_areas(const float* __restrict__ pos, const uint32_t* __restrict__ idx,
                            const uint32_t* __restrict__ triTransform,
                            const float* __restrict__ l2w, uint32_t T, float* areas) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
        V3 a, b, c;
        areas[t] = tri_world_area(pos, idx, l2w + 12 * size_t(triTransform[t]), t, a, b, c);
    }
}

// SampleAreaWeightedPoints (GPUAcceleratorBVH.hpp:887-1004 with
// KCSampleSurfacePatch, GPUAcceleratorCommonKC.cuh:389-440, and
// TriFunctions::SamplePosition, GPUPrimitiveTriangle.h:65-116): a triangle
// by the area CDF (the first t with cdf[t + 1] > xi0 * total), Osada
// barycentrics, the tangent-frame normal (geometric when no frames were
// given), both to world space.  Philox counter (sample, 0, 0x50000, 0).
__global__ void k_sample_points(const float* __restrict__ pos, const uint32_t* __restrict__ idx,
                                const float4* __restrict__ tbn,
                                const uint32_t* __restrict__ triTransform,
                                const float* __restrict__ l2w, const double* __restrict__ cdf,
                                uint32_t T, uint32_t count, uint32_t seedLo, uint32_t seedHi,
                                float* outPos, float* outNrm) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += gridDim.x * blockDim.x) {
        const Rand4 r = philox_uniform4(i, 0u, 0x50000u, 0u, seedLo, seedHi);
        const double target = static_cast<double>(r.u[0]) * cdf[T];
        uint32_t lo = 0, hi = T;
        while (lo + 1 < hi) {  // cdf[lo] <= target < cdf[hi]
            const uint32_t mid = (lo + hi) >> 1;
            if (cdf[mid] <= target) lo = mid;
            else hi = mid;
        }
        const uint32_t t = lo;
        const float* m = l2w + 12 * size_t(triTransform[t]);
        const float r1 = sqrtf(r.u[1]), r2 = r.u[2];
        const float a = 1.0f - r1, b = (1.0f - r2) * r1, c = r1 * r2;
        const uint32_t i0 = idx[3 * size_t(t)], i1 = idx[3 * size_t(t) + 1],
                       i2 = idx[3 * size_t(t) + 2];
        const V3 q0 = ld3(pos + 3 * size_t(i0)), q1 = ld3(pos + 3 * size_t(i1)),
                 q2 = ld3(pos + 3 * size_t(i2));
        V3 nl;
        if (tbn) {
            const Q4 t0 = qnormalize(q_from(tbn[i0])), t1 = qnormalize(q_from(tbn[i1])),
                     t2 = qnormalize(q_from(tbn[i2]));
            nl = to_space(v3(0.0f, 0.0f, 1.0f), bary_slerp(t0, t1, t2, a, b));
        } else {
            nl = cross(q1 - q0, q2 - q0);
        }
        const V3 p = xform_point(m, (q0 * a + q1 * b) + q2 * c);
        const V3 nw = normalize(xform_dir(m, nl));
        outPos[3 * size_t(i)] = p.x;
        outPos[3 * size_t(i) + 1] = p.y;
        outPos[3 * size_t(i) + 2] = p.z;
        outNrm[3 * size_t(i)] = nw.x;
        outNrm[3 * size_t(i) + 1] = nw.y;
        outNrm[3 * size_t(i) + 2] = nw.z;
    }
}

inline uint32_t blocks_for(uint32_t n, uint32_t block, uint32_t cap) {
    const uint32_t b = (n + block - 1) / block;
    return b < 1 ? 1 : (b > cap ? cap : b);
}

// Row-major 3x4 inverse of an affine local-to-world matrix, in double,
// each entry rounded once to float.
bool affine_inverse(const float* m, float* out) {
    double a[3][3], t[3];
    for (int r = 0; r < 3; r++) {
        for (int c = 0; c < 3; c++) a[r][c] = m[4 * r + c];
        t[r] = m[4 * r + 3];
    }
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return false;
    double inv[3][3];
    inv[0][0] = c00 / det;
    inv[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
    inv[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
    inv[1][0] = c01 / det;
    inv[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
    inv[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
    inv[2][0] = c02 / det;
    inv[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
    inv[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
    for (int r = 0; r < 3; r++) {
        double tr = 0.0;
        for (int c = 0; c < 3; c++) {
            out[4 * r + c] = static_cast<float>(inv[r][c]);
            tr -= inv[r][c] * t[c];
        }
        out[4 * r + 3] = static_cast<float>(tr);
    }
    return true;
}

// Host build of the base BVH: median split of the box centroids along the
// largest centroid extent, node 0 the root.
uint32_t base_build(std::vector<BaseNode>& nodes, std::vector<uint32_t>& items, uint32_t b,
                    uint32_t e, uint32_t parent, const float* boxes, const uint32_t* keys) {
    const uint32_t me = static_cast<uint32_t>(nodes.size());
    nodes.push_back(BaseNode{});
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t k = b; k < e; k++) {
        const float* bx = boxes + 6 * size_t(items[k]);
        for (int c = 0; c < 3; c++) {
            lo[c] = std::min(lo[c], bx[c]);
            hi[c] = std::max(hi[c], bx[3 + c]);
            const float ce = 0.5f * (bx[c] + bx[3 + c]);
            clo[c] = std::min(clo[c], ce);
            chi[c] = std::max(chi[c], ce);
        }
    }
    BaseNode nd{};
    for (int c = 0; c < 3; c++) {
        nd.lo[c] = lo[c];
        nd.hi[c] = hi[c];
    }
    nd.parent = parent;
    if (e - b == 1) {
        nd.left = nd.right = kDone;
        nd.key = keys[items[b]];
        nodes[me] = nd;
        return me;
    }
    int ax = 0;
    for (int c = 1; c < 3; c++)
        if (chi[c] - clo[c] > chi[ax] - clo[ax]) ax = c;
    const uint32_t mid = b + (e - b) / 2;
    std::nth_element(items.begin() + b, items.begin() + mid, items.begin() + e,
                     [&](uint32_t x, uint32_t y) {
                         const float cx = boxes[6 * size_t(x) + ax] + boxes[6 * size_t(x) + 3 + ax];
                         const float cy = boxes[6 * size_t(y) + ax] + boxes[6 * size_t(y) + 3 + ax];
                         return cx < cy || (cx == cy && x < y);
                     });
    nd.left = base_build(nodes, items, b, mid, me, boxes, keys);
    nd.right = base_build(nodes, items, mid, e, me, boxes, keys);
    nd.key = 0;
    nodes[me] = nd;
    return me;
}

}  // namespace
}  // namespace mrb

struct mrb_accel_group {
    mrb_system* sys = nullptr;
    uint32_t V = 0, T = 0;
    std::vector<mrb_surface> surfaces;
    std::vector<float> l2w, w2l;  // 12 per transform
    uint32_t identity = 0;
    bool built = false;
    // device: triangle data, per-triangle transform, transforms
    DBuf dPos, dIdx, dKey, dCull, dTbn, dTriXf, dL2W, dW2L, dPrimId;
    // device: per-surface LBVHs (nodes, triangles), surface table
    DBuf triAabb, extent, codes, sorted, left, right, parent, inner, scratch, root, nodes, tv0,
        te0, te1, sortTemp, surfDev, err;
    std::vector<float> surfAabbs;  // world AABB per surface (6 each)
};

struct mrb_base_accel {
    mrb_system* sys = nullptr;
    std::vector<BaseNode> nodes;
    float extent[6] = {0, 0, 0, 0, 0, 0};
    DBuf dNodes, states;
    uint32_t stateCount = 0;
};

namespace {

int group_set_device(mrb_system* s) {
    MRB_CUDA(cudaSetDevice(s->device));
    return 0;
}

int upload_transforms(mrb_accel_group* g) {
    int r;
    if ((r = upload(g->dL2W, g->l2w)) || (r = upload(g->dW2L, g->w2l))) return r;
    std::vector<uint32_t> triXf(g->T, 0u);
    for (const mrb_surface& s : g->surfaces)
        for (uint32_t t = s.tri_begin; t < s.tri_end; t++) triXf[t] = s.transform_id;
    return upload(g->dTriXf, triXf);
}

}  // namespace

extern "C" {

int mrb_accel_group_create(mrb_system* sys, const float* positions, uint32_t vertexCount,
                           const float* tbn, const uint32_t* indices, const uint32_t* triKeys,
                           const uint8_t* triCull, const uint64_t* primitiveIds,
                           uint32_t triCount, const mrb_surface* surfaces,
                           uint32_t surfaceCount, mrb_accel_group** out) {
    if (!sys || !positions || !indices || !triKeys || !surfaces || !out || surfaceCount == 0 ||
        triCount == 0 || surfaceCount > (1u << kIdBits)) {
        set_error("accel group: invalid arguments");
        return MRB_E_ARG;
    }
    for (uint32_t i = 0; i < 3 * triCount; i++)
        if (indices[i] >= vertexCount) {
            set_error("accel group: index %u out of %u vertices", indices[i], vertexCount);
            return MRB_E_ARG;
        }
    // surfaces: non-empty, disjoint triangle ranges in ascending order
    for (uint32_t s = 0; s < surfaceCount; s++) {
        const mrb_surface& f = surfaces[s];
        if (f.tri_begin >= f.tri_end || f.tri_end > triCount ||
            (s > 0 && f.tri_begin < surfaces[s - 1].tri_end)) {
            set_error("accel group: surface %u range [%u, %u) invalid", s, f.tri_begin, f.tri_end);
            return MRB_E_ARG;
        }
    }
    if (group_set_device(sys)) return MRB_E_CUDA;
    auto g = new mrb_accel_group();
    g->sys = sys;
    g->V = vertexCount;
    g->T = triCount;
    g->surfaces.assign(surfaces, surfaces + surfaceCount);
    // identity transform 0 until transforms are attached
    g->l2w = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    g->w2l = g->l2w;
    int r = 0;
    std::vector<float> pos(positions, positions + 3 * size_t(vertexCount));
    std::vector<uint32_t> idx(indices, indices + 3 * size_t(triCount));
    std::vector<uint32_t> key(triKeys, triKeys + triCount);
    std::vector<uint8_t> cull(triCount, 0);
    if (triCull) cull.assign(triCull, triCull + triCount);
    if ((r = upload(g->dPos, pos)) || (r = upload(g->dIdx, idx)) || (r = upload(g->dKey, key)) ||
        (r = upload(g->dCull, cull))) {
        delete g;
        return r;
    }
    if (tbn) {
        std::vector<float> q(tbn, tbn + 4 * size_t(vertexCount));
        if ((r = upload(g->dTbn, q))) {
            delete g;
            return r;
        }
    }
    if (primitiveIds) {
        std::vector<uint64_t> ids(primitiveIds, primitiveIds + triCount);
        if ((r = upload(g->dPrimId, ids))) {
            delete g;
            return r;
        }
    }
    *out = g;
    return 0;
}

void mrb_accel_group_destroy(mrb_accel_group* g) { delete g; }

int mrb_accel_group_attach_transforms(mrb_accel_group* g, const float* localToWorld,
                                      uint32_t count, uint32_t identityIndex) {
    if (!g || !localToWorld || count == 0 || identityIndex >= count) return MRB_E_ARG;
    for (const mrb_surface& s : g->surfaces)
        if (s.transform_id >= count) {
            set_error("accel group: surface transform %u out of %u", s.transform_id, count);
            return MRB_E_ARG;
        }
    g->l2w.assign(localToWorld, localToWorld + 12 * size_t(count));
    g->w2l.assign(12 * size_t(count), 0.0f);
    for (uint32_t i = 0; i < count; i++)
        if (!affine_inverse(&g->l2w[12 * size_t(i)], &g->w2l[12 * size_t(i)])) {
            set_error("accel group: transform %u is singular", i);
            return MRB_E_ARG;
        }
    g->identity = identityIndex;
    if (group_set_device(g->sys)) return MRB_E_CUDA;
    return upload_transforms(g);
}

int mrb_accel_group_construct(mrb_accel_group* g, void* stream) {
    if (!g) return MRB_E_ARG;
    if (group_set_device(g->sys)) return MRB_E_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (const mrb_surface& s : g->surfaces)
        if (12 * size_t(s.transform_id) >= g->l2w.size()) {
            set_error("accel group: surface transform %u not attached", s.transform_id);
            return MRB_E_STATE;
        }
    int r;
    if (!g->dL2W.p && (r = upload_transforms(g))) return r;
    const uint32_t T = g->T, S = static_cast<uint32_t>(g->surfaces.size());
    uint32_t maxN = 0;
    for (const mrb_surface& s : g->surfaces) maxN = std::max(maxN, s.tri_end - s.tri_begin);
    // per surface: inner nodes n - 1 (the stored node arrays hold T entries)
    if ((r = g->triAabb.alloc(size_t(T) * 24)) || (r = g->extent.alloc(32 * size_t(S))) ||
        (r = g->codes.alloc(size_t(T) * 8)) || (r = g->sorted.alloc(size_t(T) * 4)) ||
        (r = g->left.alloc(size_t(T) * 4)) || (r = g->right.alloc(size_t(T) * 4)) ||
        (r = g->parent.alloc(size_t(2 * T) * 4)) || (r = g->inner.alloc(size_t(T) * 24)) ||
        (r = g->scratch.alloc(size_t(maxN) * 12 + 12)) || (r = g->root.alloc(4 * size_t(S))) ||
        (r = g->nodes.alloc(size_t(T) * sizeof(BvhNode))) || (r = g->tv0.alloc(size_t(T) * 16)) ||
        (r = g->te0.alloc(size_t(T) * 16)) || (r = g->te1.alloc(size_t(T) * 16)) ||
        (r = g->err.alloc(4)))
        return r;
    const size_t tb = radix_sort_temp_bytes(maxN, 8, 0, 63);
    if ((r = g->sortTemp.alloc(tb))) return r;
    MRB_CUDA(cudaMemsetAsync(g->err.p, 0, 4, st));
    std::vector<SurfaceDev> sd(S);
    std::vector<uint32_t> roots(S, 0);
    for (uint32_t si = 0; si < S; si++) {
        const uint32_t b = g->surfaces[si].tri_begin, n = g->surfaces[si].tri_end - b;
        const uint32_t* idx = g->dIdx.as<uint32_t>() + 3 * size_t(b);
        float* triAabb = g->triAabb.as<float>() + 6 * size_t(b);
        uint64_t* codes = g->codes.as<uint64_t>() + b;
        uint32_t* sorted = g->sorted.as<uint32_t>() + b;
        float* ext = g->extent.as<float>() + 8 * size_t(si);
        if ((r = lbvh_morton(g->dPos.as<float>(), idx, n, triAabb, ext, codes, nullptr, ext + 6,
                             st)))
            return r;
        if ((r = radix_sort_pairs<uint64_t>(codes, sorted, nullptr, n, 0, 63, false,
                                            g->sortTemp.p, tb, st, true)))
            return r;
        uint32_t* scr = g->scratch.as<uint32_t>();
        const size_t ni = n > 1 ? n - 1 : 1;
        LbvhArrays a{g->left.as<uint32_t>() + b, g->right.as<uint32_t>() + b,
                     g->parent.as<uint32_t>() + 2 * size_t(b), g->inner.as<float>() + 6 * size_t(b),
                     scr, scr + ni, scr + 2 * ni, g->root.as<uint32_t>() + si,
                     g->nodes.as<BvhNode>() + b};
        if ((r = lbvh_hierarchy(codes, sorted, triAabb, n, a, st))) return r;
        if ((r = lbvh_gather(g->dPos.as<float>(), idx, g->dKey.as<uint32_t>() + b,
                             g->dCull.as<uint8_t>() + b, sorted, n, g->tv0.as<float4>() + b,
                             g->te0.as<float4>() + b, g->te1.as<float4>() + b, st)))
            return r;
        uint32_t err = 0;
        MRB_CUDA(cudaMemcpyAsync(&roots[si], g->root.as<uint32_t>() + si, 4, cudaMemcpyDeviceToHost,
                                 st));
        MRB_CUDA(cudaMemcpyAsync(&err, radix_sort_error_flag(g->sortTemp.p, n), 4,
                                 cudaMemcpyDeviceToHost, st));
        MRB_CUDA(cudaStreamSynchronize(st));
        if (err) {
            set_error("accel group: radix sort look-back gave up");
            return MRB_E_DEVICE;
        }
        AccelDev acc{g->nodes.as<BvhNode>() + b, g->tv0.as<float4>() + b, g->te0.as<float4>() + b,
                     g->te1.as<float4>() + b, n > 1 ? int(roots[si]) - int(n) : ~0, n};
        sd[si] = SurfaceDev{acc, b, g->surfaces[si].transform_id};
    }
    if ((r = upload(g->surfDev, sd))) return r;
    // world AABB of each surface: the local box's eight corners transformed
    std::vector<float> ext(8 * size_t(S));
    MRB_CUDA(cudaMemcpy(ext.data(), g->extent.p, ext.size() * 4, cudaMemcpyDeviceToHost));
    g->surfAabbs.assign(6 * size_t(S), 0.0f);
    for (uint32_t si = 0; si < S; si++) {
        const float* e = &ext[8 * size_t(si)];
        const float* m = &g->l2w[12 * size_t(g->surfaces[si].transform_id)];
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = 0; k < 8; k++) {
            const float p[3] = {e[(k & 1) ? 3 : 0], e[(k & 2) ? 4 : 1], e[(k & 4) ? 5 : 2]};
            for (int row = 0; row < 3; row++) {
                const float w = ((m[4 * row] * p[0] + m[4 * row + 1] * p[1]) + m[4 * row + 2] * p[2]) +
                                m[4 * row + 3];
                lo[row] = std::min(lo[row], w);
                hi[row] = std::max(hi[row], w);
            }
        }
        for (int c = 0; c < 3; c++) {
            g->surfAabbs[6 * size_t(si) + c] = lo[c];
            g->surfAabbs[6 * size_t(si) + 3 + c] = hi[c];
        }
    }
    g->scratch.release();
    g->built = true;
    return 0;
}

int mrb_accel_group_hit(const mrb_accel_group* g, uint32_t* materialKeys, uint32_t* transformIds,
                        uint64_t* primitiveIds, void* hitStructs, uint32_t hitStride, void* rays,
                        const uint32_t* rayIds, const uint32_t* accelKeys, uint32_t rayCount,
                        void* stream) {
    if (!g || !g->built) {
        set_error("accel group: not constructed");
        return MRB_E_STATE;
    }
    if (rayCount == 0) return 0;
    if (!materialKeys || !transformIds || !primitiveIds || !hitStructs || !rays || !rayIds ||
        !accelKeys || hitStride < 8 || (hitStride & 3)) {
        set_error("accel group hit: invalid arguments (hit stride %u)", hitStride);
        return MRB_E_ARG;
    }
    if (group_set_device(g->sys)) return MRB_E_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_group_hit<<<blocks_for(rayCount, 128, 148 * 16), 128, 0, st>>>(
        g->surfDev.as<SurfaceDev>(), static_cast<uint32_t>(g->surfaces.size()), g->dW2L.as<float>(),
        g->dPrimId.as<unsigned long long>(), materialKeys, transformIds,
        reinterpret_cast<unsigned long long*>(primitiveIds), static_cast<char*>(hitStructs),
        hitStride, static_cast<float4*>(rays), rayIds, accelKeys, rayCount, g->err.as<uint32_t>());
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int mrb_accel_group_aabbs(const mrb_accel_group* g, float* aabbs, uint32_t capacity) {
    if (!g || !g->built) return MRB_E_STATE;
    const uint32_t S = static_cast<uint32_t>(g->surfaces.size());
    if (aabbs) std::memcpy(aabbs, g->surfAabbs.data(), 24 * size_t(std::min(S, capacity)));
    return static_cast<int>(S);
}

uint64_t mrb_accel_group_primitive_count(const mrb_accel_group* g) { return g ? g->T : 0; }

uint32_t mrb_accel_group_accelerator_count(const mrb_accel_group* g) {
    return g ? static_cast<uint32_t>(g->surfaces.size()) : 0u;
}

int mrb_accel_group_total_area(const mrb_accel_group* g, float* area, void* stream) {
    if (!g || !area) return MRB_E_ARG;
    if (!g->dL2W.p) return MRB_E_STATE;
    if (group_set_device(g->sys)) return MRB_E_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DBuf a;
    int r = a.alloc(size_t(g->T) * 4);
    if (r) return r;
    k_tri_areas<<<blocks_for(g->T, 256, 148 * 8), 256, 0, st>>>(
        g->dPos.as<float>(), g->dIdx.as<uint32_t>(), g->dTriXf.as<uint32_t>(), g->dL2W.as<float>(),
        g->T, a.as<float>());
    MRB_CUDA(cudaGetLastError());
    std::vector<float> h(g->T);
    MRB_CUDA(cudaMemcpyAsync(h.data(), a.p, h.size() * 4, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    double sum = 0.0;  // summed in triangle order
    for (float v : h) sum += v;
    *area = static_cast<float>(sum);
    return 0;
}

int mrb_accel_group_sample_points(const mrb_accel_group* g, float* positions, float* normals,
                                  uint32_t count, uint64_t seed, void* stream) {
    if (!g || !positions || !normals) return MRB_E_ARG;
    if (!g->dL2W.p) return MRB_E_STATE;
    if (count == 0) return 0;
    if (group_set_device(g->sys)) return MRB_E_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DBuf a, c;
    int r;
    if ((r = a.alloc(size_t(g->T) * 4)) || (r = c.alloc(size_t(g->T + 1) * 8))) return r;
    k_tri_areas<<<blocks_for(g->T, 256, 148 * 8), 256, 0, st>>>(
        g->dPos.as<float>(), g->dIdx.as<uint32_t>(), g->dTriXf.as<uint32_t>(), g->dL2W.as<float>(),
        g->T, a.as<float>());
    MRB_CUDA(cudaGetLastError());
    // the area CDF in double, on the host (its sums must not depend on a
    // reduction order)
    std::vector<float> h(g->T);
    MRB_CUDA(cudaMemcpyAsync(h.data(), a.p, h.size() * 4, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    std::vector<double> cdf(g->T + 1, 0.0);
    for (uint32_t t = 0; t < g->T; t++) cdf[t + 1] = cdf[t] + h[t];
    if (!(cdf[g->T] > 0.0)) {
        set_error("accel group: zero total area");
        return MRB_E_ARG;
    }
    MRB_CUDA(cudaMemcpyAsync(c.p, cdf.data(), cdf.size() * 8, cudaMemcpyHostToDevice, st));
    k_sample_points<<<blocks_for(count, 128, 148 * 16), 128, 0, st>>>(
        g->dPos.as<float>(), g->dIdx.as<uint32_t>(), g->dTbn.as<float4>(),
        g->dTriXf.as<uint32_t>(), g->dL2W.as<float>(), c.as<double>(), g->T, count,
        static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), positions, normals);
    MRB_CUDA(cudaGetLastError());
    MRB_CUDA(cudaStreamSynchronize(st));
    return 0;
}

static SvoParams octree_params(const float* box, uint32_t res) {
    SvoParams P{};
    for (int c = 0; c < 3; c++) {
        P.lo[c] = box[c];
        P.hi[c] = box[3 + c];
    }
    P.res = res;
    uint32_t d = 0;
    while ((1u << (d + 1)) <= res) d++;
    P.depth = d;
    P.leafVoxelSize = (box[3] - box[0]) / static_cast<float>(res);
    return P;
}

int mrb_accel_group_voxel_counts(const mrb_accel_group* g, uint64_t* counts, uint32_t resolution,
                                 const float* octreeAabb, void* stream) {
    if (!g || !counts || !octreeAabb || resolution == 0 || (resolution & (resolution - 1)))
        return MRB_E_ARG;
    if (!g->dL2W.p) return MRB_E_STATE;
    if (group_set_device(g->sys)) return MRB_E_CUDA;
    PrimVoxIn in{g->T, g->dPos.as<float>(), g->dIdx.as<uint32_t>(), g->dKey.as<uint32_t>(),
                 g->dTriXf.as<uint32_t>(), g->dL2W.as<float>()};
    return prim_voxel_count(in, octree_params(octreeAabb, resolution),
                            reinterpret_cast<unsigned long long*>(counts),
                            static_cast<cudaStream_t>(stream));
}

int mrb_accel_group_voxelize(const mrb_accel_group* g, uint64_t* voxels, uint32_t* voxelNormals,
                             uint32_t* voxelLightKeys, const uint64_t* voxelOffsets,
                             const uint32_t* sortedLightKeys, uint32_t lightCount,
                             uint32_t resolution, const float* octreeAabb, void* stream) {
    if (!g || !voxels || !voxelNormals || !voxelLightKeys || !voxelOffsets || !octreeAabb ||
        resolution == 0 || (resolution & (resolution - 1)) || (lightCount && !sortedLightKeys))
        return MRB_E_ARG;
    if (!g->dL2W.p) return MRB_E_STATE;
    if (group_set_device(g->sys)) return MRB_E_CUDA;
    PrimVoxIn in{g->T, g->dPos.as<float>(), g->dIdx.as<uint32_t>(), g->dKey.as<uint32_t>(),
                 g->dTriXf.as<uint32_t>(), g->dL2W.as<float>()};
    return prim_voxelize(in, octree_params(octreeAabb, resolution),
                         reinterpret_cast<const unsigned long long*>(voxelOffsets), voxels,
                         voxelNormals, voxelLightKeys, sortedLightKeys, lightCount,
                         static_cast<cudaStream_t>(stream));
}

// ---- base accelerator ------------------------------------------------------
int mrb_base_accel_create(mrb_system* sys, mrb_base_accel** out) {
    if (!sys || !out) return MRB_E_ARG;
    auto b = new mrb_base_accel();
    b->sys = sys;
    *out = b;
    return 0;
}

void mrb_base_accel_destroy(mrb_base_accel* b) { delete b; }

int mrb_base_accel_construct(mrb_base_accel* b, const float* aabbs, const uint32_t* accelKeys,
                             uint32_t count) {
    if (!b || !aabbs || !accelKeys || count == 0) return MRB_E_ARG;
    for (uint32_t i = 0; i < count; i++)
        if (accelKeys[i] == kBatchNull) {
            set_error("base accelerator: surface %u has the null key", i);
            return MRB_E_ARG;
        }
    if (group_set_device(b->sys)) return MRB_E_CUDA;
    std::vector<uint32_t> items(count);
    for (uint32_t i = 0; i < count; i++) items[i] = i;
    b->nodes.clear();
    base_build(b->nodes, items, 0, count, kDone, aabbs, accelKeys);
    for (int c = 0; c < 3; c++) {
        b->extent[c] = b->nodes[0].lo[c];
        b->extent[3 + c] = b->nodes[0].hi[c];
    }
    return upload(b->dNodes, b->nodes);
}

int mrb_base_accel_get_ready(mrb_base_accel* b, uint32_t rayCount, void* stream) {
    if (!b || b->nodes.empty()) return MRB_E_STATE;
    if (group_set_device(b->sys)) return MRB_E_CUDA;
    int r = b->states.alloc(size_t(std::max(rayCount, 1u)) * 4);
    if (r) return r;
    b->stateCount = rayCount;
    MRB_CUDA(cudaMemsetAsync(b->states.p, 0, size_t(rayCount) * 4,
                             static_cast<cudaStream_t>(stream)));  // every ray at the root
    return 0;
}

int mrb_base_accel_hit(const mrb_base_accel* b, uint32_t* accelKeys, const void* rays,
                       const uint32_t* rayIds, uint32_t rayCount, void* stream) {
    if (!b || b->nodes.empty() || !b->states.p) {
        set_error("base accelerator: construct and get ready first");
        return MRB_E_STATE;
    }
    if (rayCount == 0) return 0;
    if (!accelKeys || !rays || !rayIds) return MRB_E_ARG;
    if (group_set_device(b->sys)) return MRB_E_CUDA;
    k_base_hit<<<blocks_for(rayCount, 128, 148 * 16), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        b->dNodes.as<BaseNode>(), static_cast<uint32_t>(b->nodes.size()), b->states.as<uint32_t>(),
        accelKeys, static_cast<const float4*>(rays), rayIds, rayCount);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int mrb_base_accel_extents(const mrb_base_accel* b, float* aabb) {
    if (!b || !aabb || b->nodes.empty()) return MRB_E_STATE;
    std::memcpy(aabb, b->extent, 24);
    return 0;
}

}  // extern "C"
