// Shim that runs MRay's own sparse-voxel-octree code on the host, for golden
// vectors of the guided path:
//   - TriFunctions::Voxelize (GPUPrimitiveTriangle.h:384-620) driven as
//     KCGetVoxelCount / KCVoxelizePrims drive it (GPUAcceleratorCommonKC.cuh:
//     439-542): a counting pass, an exclusive scan, a writing pass;
//   - the octree level kernels KCMarkMortonChanges, KCMarkChild,
//     KCExtractChildrenCounts, KCSetChildrenPtrs, KCSetParentOf(Leaf)Children
//     (AnisoSVO.cu:58-222), launched in the order AnisoSVOctreeCPU::Constrcut
//     launches them (AnisoSVO.cu:916-1094);
//   - ray binning: AnisoSVOctreeGPU::NearestNodeIndex with neighbour search
//     (KCInitializeSVOBins, WFPGTracerKC.cuh:965-1018), SetLeafRayCount
//     (KCWriteLeafRayAmounts, :1020-1043), KCCollapseRayCountsLeaf /
//     KCCollapseRayCounts (AnisoSVO.cu:265-350) in CollapseRayCounts' order
//     (AnisoSVO.cu:1485-1528) and FindMarkedBin (KCCheckReducedSVOBins,
//     WFPGTracerKC.cuh:1045-1066);
//   - AnisoSVOctreeGPU::ConeTraceRay and ReadRadiance (AnisoSVO.cuh:767-1033,
//     1035-1055, VoxelPayload::ReadRadiance :433-470);
//   - the payload passes: KCAverageNormals (AnisoSVO.cu:418-517),
//     NormalizeAndFilterRadiance with its three kernels (AnisoSVO.cu:352-380,
//     519-654, 1415-1483) and DepositRadiance (AnisoSVO.cuh:1080-1098).
//
// TEST INFRASTRUCTURE ONLY (tests/golden/make_golden.py).  The reference
// headers are #included from REF_ROOT and the kernel bodies are cut out of
// AnisoSVO.cu by oracle/Makefile into oracle/_ref/ (git-ignored); nothing of
// the reference is copied into the repository.  CUB's sort, run-length
// encode and scan are replaced by the standard library with the semantics
// CUB documents (stable radix sort, run lengths of equal neighbours,
// exclusive sum).  Each simulated thread runs to completion before the next
// starts, so plain loads/stores stand in for the atomics; every kernel here
// is free of inter-thread ordering within a launch except through those
// atomics, whose sums are order-independent integers.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>
// unqualified math calls in the reference must pick the float overloads, as
// they do on the device (the C library's double nextafter would step tMin by
// a double ulp, which rounds back to the same float, and the cone loop would
// stop advancing)
using std::ceil;
using std::copysign;
using std::fabs;
using std::floor;
using std::isinf;
using std::isnan;
using std::max;
using std::min;
using std::nextafter;
using std::signbit;
using std::sqrt;

// ---- host stand-ins for the CUDA built-ins the reference code uses -------
static uint3 blockIdx, threadIdx;
static dim3 blockDim, gridDim;
template <class T, class U>
static inline T atomicAdd(T* a, U v) {
    T o = *a;
    *a = static_cast<T>(o + v);
    return o;
}
template <class T>
static inline T atomicOr(T* a, T v) {
    T o = *a;
    *a = o | v;
    return o;
}
template <class T>
static inline T atomicCAS(T* a, T c, T v) {
    T o = *a;
    if (o == c) *a = v;
    return o;
}
static inline int __popc(unsigned int x) { return __builtin_popcount(x); }
static inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }
static inline int __ffs(int x) { return __builtin_ffs(x); }
static inline int __clz(int x) { return x ? __builtin_clz(static_cast<unsigned>(x)) : 32; }
static inline unsigned long long __brevll(unsigned long long x) {
    unsigned long long r = 0;
    for (int i = 0; i < 64; i++)
        if ((x >> i) & 1ull) r |= 1ull << (63 - i);
    return r;
}
static inline float __int_as_float(int x) {
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}
static inline int __float_as_int(float x) {
    int i;
    std::memcpy(&i, &x, 4);
    return i;
}
static inline unsigned int __float_as_uint(float x) {
    unsigned int i;
    std::memcpy(&i, &x, 4);
    return i;
}
static inline float __uint_as_float(unsigned int x) {
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

#include "RayLib/Types.h"
#include "TracerCUDA/GPUPrimitiveTriangle.h"
// the octree's arrays are private members that only AnisoSVOctreeCPU sets;
// the shim stands in for that class, so it opens them up
#define private public
#define protected public
#include "TracerCUDA/AnisoSVO.cuh"
#undef private
#undef protected

#define CUDA_LAUNCH_BOUNDS_1D
// KCMarkMortonChanges .. KCSetParentOfLeafChildren (AnisoSVO.cu:58-222),
// KCCollapseRayCounts / KCCollapseRayCountsLeaf (AnisoSVO.cu:265-350),
// KCCCopyRadianceToHalfBufferLeaf (:352-380) and KCAverageNormals,
// KCBottomUpFilterIrradiance, KCTopDownFilterIrradiance (:418-654).  This
// file is compiled with -ftrivial-auto-var-init=zero: KCAverageNormals adds
// into its second k-means buffer before anything is written there, and
// zero is the start that clustering intends.
#include "svo_level_kernels.inc"
#include "svo_collapse_kernels.inc"
#include "svo_payload_kernels.inc"

namespace {

template <class F>
void launch(uint32_t threads, F f) {
    blockDim = dim3(256, 1, 1);
    gridDim = dim3((threads + 255) / 256, 1, 1);
    for (uint32_t b = 0; b < gridDim.x; b++)
        for (uint32_t t = 0; t < 256; t++) {
            blockIdx = make_uint3(b, 0, 0);
            threadIdx = make_uint3(t, 0, 0);
            f();
        }
}

// Identity GPUTransformI (what GPUTransformIdentity computes: the input)
struct HostIdentity final : public GPUTransformI {
    RayF WorldToLocal(const RayF& r, const uint32_t*, const float*, uint32_t) const override {
        return r;
    }
    Vector3 WorldToLocal(const Vector3& v, bool, const uint32_t*, const float*,
                         uint32_t) const override {
        return v;
    }
    AABB3f WorldToLocal(const AABB3f& a) const override { return a; }
    Vector3 LocalToWorld(const Vector3& v, bool, const uint32_t*, const float*,
                         uint32_t) const override {
        return v;
    }
    AABB3f LocalToWorld(const AABB3f& a) const override { return a; }
    QuatF ToLocalRotation(const uint32_t*, const float*, uint32_t) const override {
        return IdentityQuatF;
    }
    Vector3f ToWorldScale(const uint32_t*, const float*, uint32_t) const override {
        return Vector3f(1.0f);
    }
    Vector3f ToLocalScale(const uint32_t*, const float*, uint32_t) const override {
        return Vector3f(1.0f);
    }
    Matrix4x4 GetLocalToWorldAsMatrix() const override { return Indentity4x4; }
};

// The octree AABB of AnisoSVOctreeCPU::Constrcut (AnisoSVO.cu:670-679)
AABB3f svo_aabb(const AABB3f& sceneAABB, uint32_t res, float& leafSize, uint32_t& leafDepth) {
    Vector3f span = sceneAABB.Span();
    int maxDimIndex = span.Max();
    float worldSizeXYZ = span[maxDimIndex];
    float sizePadding = (worldSizeXYZ / static_cast<float>(res));
    leafDepth = Utility::FindLastSet(res);
    leafSize = (worldSizeXYZ + 2.0f * sizePadding) / static_cast<float>(res);
    return AABB3f(sceneAABB.Min() - Vector3f(sizePadding),
                  sceneAABB.Min() + Vector3f(sizePadding + worldSizeXYZ));
}

struct RefSvo {
    AnisoSVOctreeGPU tree;
    std::vector<uint64_t> nodes;
    std::vector<uint32_t> leafParents, levelOffsets, levelCounts;
    std::vector<uint64_t> leafCodes;
    std::vector<uint32_t> binInfo, leafBinInfo;
    std::vector<uint32_t> nodeNormSpec, leafNormSpec;
    std::vector<Vector2h> nodeAvg, leafAvg;
    std::vector<Vector2f> leafIrr;
    std::vector<Vector2ui> leafCnt;
    std::vector<uint32_t> shadowHit, shadowMiss;
    std::vector<half> nodeFactor;
};

}  // namespace

extern "C" {

// Voxelize every triangle: counts[ntri], then codes / normals (packed
// u16 | u16 << 16) in triangle order, at most `capacity` voxels.  The octree
// AABB is written to svo_aabb6 (min xyz, max xyz).  Returns the voxel count
// or -1 when `capacity` is too small.
int64_t ref_svo_voxelize(const float* pos, const uint32_t* idx, uint32_t ntri,
                         const float* scene_aabb6, uint32_t res, float* svo_aabb6,
                         uint64_t* counts, uint64_t* codes, uint32_t* normals, uint64_t capacity) {
    // the triangle group's data as the loader lays it out (GPUPrimitiveTriangle.h:41-56)
    uint32_t nv = 0;
    for (uint32_t i = 0; i < 3 * ntri; i++) nv = std::max(nv, idx[i] + 1);
    std::vector<Vector3f> P(nv);
    for (uint32_t v = 0; v < nv; v++) P[v] = Vector3f(pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]);
    std::vector<uint64_t> I(idx, idx + 3 * size_t(ntri));
    TriData data{};
    data.positions = P.data();
    data.indexList = I.data();
    HostIdentity ident;
    float leaf;
    uint32_t depth;
    const AABB3f aabb = svo_aabb(AABB3f(Vector3f(scene_aabb6[0], scene_aabb6[1], scene_aabb6[2]),
                                        Vector3f(scene_aabb6[3], scene_aabb6[4], scene_aabb6[5])),
                                 res, leaf, depth);
    for (int c = 0; c < 3; c++) {
        svo_aabb6[c] = aabb.Min()[c];
        svo_aabb6[3 + c] = aabb.Max()[c];
    }
    // KCGetVoxelCount
    for (uint32_t t = 0; t < ntri; t++)
        counts[t] = TriFunctions::Voxelize(nullptr, nullptr, 0, true, t, data, ident, aabb, res);
    // ExclusiveScanArrayGPU over the counts, then KCVoxelizePrims
    uint64_t total = 0;
    for (uint32_t t = 0; t < ntri; t++) total += counts[t];
    if (!codes) return static_cast<int64_t>(total);
    if (total > capacity) return -1;
    std::vector<Vector2us> nrm(total);
    uint64_t off = 0;
    for (uint32_t t = 0; t < ntri; t++) {
        TriFunctions::Voxelize(codes + off, nrm.data() + off, static_cast<uint32_t>(counts[t]),
                               false, t, data, ident, aabb, res);
        off += counts[t];
    }
    for (uint64_t i = 0; i < total; i++)
        normals[i] = uint32_t(nrm[i][0]) | (uint32_t(nrm[i][1]) << 16);
    return static_cast<int64_t>(total);
}

// AnisoSVOctreeCPU::Constrcut's structure from voxel Morton codes (octree
// box, leaf depth and leaf size derived from the scene AABB as Constrcut
// derives them): stable
// sort on bits [0, 3 * depth + 1), run-length encode, then per level
// KCMarkMortonChanges + reduce, and top-down KCMarkChild,
// KCExtractChildrenCounts, exclusive scan, KCSetChildrenPtrs and
// KCSetParentOf(Leaf)Children.  Returns a handle, or null with *status set
// (1: the scan of a level's child counts does not match the next level).
void* ref_svo_build(const uint64_t* voxels, uint64_t nvox, const float* scene_aabb6, uint32_t res,
                    int* status) {
    *status = 0;
    auto h = std::make_unique<RefSvo>();
    AnisoSVOctreeGPU& T = h->tree;
    T.svoAABB = svo_aabb(AABB3f(Vector3f(scene_aabb6[0], scene_aabb6[1], scene_aabb6[2]),
                                Vector3f(scene_aabb6[3], scene_aabb6[4], scene_aabb6[5])),
                         res, T.leafVoxelSize, T.leafDepth);
    T.voxelResolution = res;
    const uint32_t levelCount = T.leafDepth;
    // cub::DeviceRadixSort::SortPairs on bits [0, 3*depth+1) is stable; codes
    // never use bits at or above 3*depth, so this is a stable sort by value
    std::vector<uint64_t> sorted(voxels, voxels + nvox);
    std::stable_sort(sorted.begin(), sorted.end());
    // cub::DeviceRunLengthEncode::Encode: unique values in order
    std::vector<uint64_t> uniq;
    for (uint64_t i = 0; i < nvox; i++)
        if (i == 0 || sorted[i] != sorted[i - 1]) uniq.push_back(sorted[i]);
    const uint32_t U = static_cast<uint32_t>(uniq.size());
    uniq.push_back(0);  // KCMarkMortonChanges reads gVoxels[threadId + 1] up to U - 1
    std::vector<uint32_t> diff(U + 1, 0), childOffsets(U + 1, 0);
    std::vector<uint32_t>& counts = h->levelCounts;
    counts.assign(levelCount + 1, 0);
    counts[0] = 1;
    for (uint32_t i = 1; i <= levelCount; i++) {
        const uint32_t n = U - 1;
        launch(n, [&] { KCMarkMortonChanges(diff.data(), uniq.data(), n, i, levelCount); });
        uint32_t s = 0;
        for (uint32_t k = 0; k < n; k++) s += diff[k];
        counts[i] = s + 1;
    }
    std::vector<uint32_t>& offs = h->levelOffsets;
    offs.assign(levelCount + 2, 0);
    std::inclusive_scan(counts.cbegin(), counts.cend(), offs.begin() + 1);
    offs.front() = 0;
    const uint32_t nodeCount = offs[offs.size() - 2];
    T.nodeCount = nodeCount;
    T.leafCount = U;
    T.levelOffsetCount = static_cast<uint32_t>(offs.size());
    h->nodes.assign(nodeCount, AnisoSVOctreeGPU::INVALID_NODE);
    h->leafParents.assign(U, 0xFFFFFFFFu);
    uint64_t* N = h->nodes.data();
    for (uint32_t i = 0; i < levelCount; i++) {
        launch(U, [&] { KCMarkChild(N, uniq.data(), U, i, levelCount); });
        launch(counts[i], [&] { KCExtractChildrenCounts(diff.data(), N + offs[i], counts[i]); });
        // cub::DeviceScan::ExclusiveSum over counts[i] + 1 entries
        uint32_t run = 0;
        for (uint32_t k = 0; k <= counts[i]; k++) {
            childOffsets[k] = run;
            run += (k < counts[i]) ? diff[k] : 0u;
        }
        if (childOffsets[counts[i]] != counts[i + 1]) {
            *status = 1;
            return nullptr;
        }
        const bool last = (i == levelCount - 1);
        const uint32_t nextOff = last ? 0u : offs[i + 1];
        launch(counts[i], [&] {
            KCSetChildrenPtrs(N + offs[i], childOffsets.data(), nextOff, counts[i], last);
        });
        if (!last)
            launch(counts[i], [&] { KCSetParentOfChildren(N, N + offs[i], counts[i]); });
        else
            launch(counts[i], [&] {
                KCSetParentOfLeafChildren(h->leafParents.data(), N, N + offs[i], counts[i]);
            });
    }
    uniq.pop_back();
    h->leafCodes = std::move(uniq);
    h->binInfo.assign(nodeCount, 0);
    h->leafBinInfo.assign(U, 0);
    h->nodeNormSpec.assign(nodeCount, 0);
    h->leafNormSpec.assign(U, 0);
    h->nodeAvg.assign(nodeCount, Vector2h(0.0f, 0.0f));
    h->leafAvg.assign(U, Vector2h(0.0f, 0.0f));
    h->leafIrr.assign(U, Vector2f(0.0f, 0.0f));
    h->leafCnt.assign(U, Vector2ui(0u, 0u));
    h->shadowHit.assign(U, 0u);
    h->shadowMiss.assign(U, 0u);
    h->nodeFactor.assign(nodeCount, half(0.0f));
    T.dNodes = h->nodes.data();
    T.dLeafParents = h->leafParents.data();
    T.dLevelNodeOffsets = h->levelOffsets.data();
    T.dBinInfo = h->binInfo.data();
    T.dLeafBinInfo = h->leafBinInfo.data();
    T.payload.dNormalAndSpecNode = h->nodeNormSpec.data();
    T.payload.dNormalAndSpecLeaf = h->leafNormSpec.data();
    T.payload.dAvgIrradianceNode = h->nodeAvg.data();
    T.payload.dAvgIrradianceLeaf = h->leafAvg.data();
    T.payload.dTotalIrradianceLeaf = h->leafIrr.data();
    T.payload.dSampleCountLeaf = h->leafCnt.data();
    T.payload.dShadowRayHitLeaf = h->shadowHit.data();
    T.payload.dShadowRayMissLeaf = h->shadowMiss.data();
    T.payload.dGuidingFactorNode = h->nodeFactor.data();
    T.dBoundaryLight = nullptr;
    return h.release();
}

void ref_svo_destroy(void* p) { delete static_cast<RefSvo*>(p); }

// sizes[3]: nodes, leaves, level-offset entries
void ref_svo_sizes(const void* p, uint32_t* sizes) {
    const RefSvo* h = static_cast<const RefSvo*>(p);
    sizes[0] = h->tree.nodeCount;
    sizes[1] = h->tree.leafCount;
    sizes[2] = static_cast<uint32_t>(h->levelOffsets.size());
}

void ref_svo_get(const void* p, uint64_t* nodes, uint32_t* leaf_parents, uint64_t* leaf_codes,
                 uint32_t* level_offsets) {
    const RefSvo* h = static_cast<const RefSvo*>(p);
    std::copy(h->nodes.begin(), h->nodes.end(), nodes);
    std::copy(h->leafParents.begin(), h->leafParents.end(), leaf_parents);
    std::copy(h->leafCodes.begin(), h->leafCodes.end(), leaf_codes);
    std::copy(h->levelOffsets.begin(), h->levelOffsets.end(), level_offsets);
}

// Bin ids of n rays that hit at t along (o, d); valid[i] = 0 for the rays
// KCInitializeSVOBins skips (NEE rays, misses, the boundary material).  The
// bin words start at zero (the reference clears only their first halves,
// AnisoSVO.cu:1485-1489 with 16-bit sizes; a clean start is what the binning
// intends).  Output: 0xFFFFFFFF (no bin), leaf | 1 << 31, or a node index.
void ref_svo_bin_rays(void* p, const float* o, const float* d, const float* t,
                      const uint8_t* valid, uint32_t n, uint32_t min_level,
                      uint32_t min_ray_count, uint32_t* bin_out) {
    RefSvo* h = static_cast<RefSvo*>(p);
    AnisoSVOctreeGPU& T = h->tree;
    std::fill(h->binInfo.begin(), h->binInfo.end(), 0u);
    std::fill(h->leafBinInfo.begin(), h->leafBinInfo.end(), 0u);
    // KCInitializeSVOBins
    std::vector<uint32_t> leafRays(T.leafCount, 0);
    for (uint32_t i = 0; i < n; i++) {
        bin_out[i] = 0xFFFFFFFFu;
        if (!valid[i]) continue;
        RayF ray(Vector3f(d[3 * i], d[3 * i + 1], d[3 * i + 2]),
                 Vector3f(o[3 * i], o[3 * i + 1], o[3 * i + 2]));
        Vector3 position = ray.AdvancedPos(t[i]);
        uint32_t leafIndex;
        if (T.NearestNodeIndex(leafIndex, position, T.LeafDepth(), true)) {
            bin_out[i] = leafIndex | (1u << 31);
            leafRays[leafIndex]++;
        }
    }
    // sort + RLE of the leaf bins, then KCWriteLeafRayAmounts
    for (uint32_t l = 0; l < T.leafCount; l++)
        if (leafRays[l])
            T.SetLeafRayCount(l, static_cast<uint16_t>(std::min<uint32_t>(leafRays[l], UINT16_MAX)));
    // AnisoSVOctreeCPU::CollapseRayCounts
    launch(T.leafCount, [&] {
        KCCollapseRayCountsLeaf(T.dLeafBinInfo, T.dBinInfo, T.dLeafParents, T.leafCount,
                                T.leafDepth, min_level, min_ray_count);
    });
    for (int32_t i = static_cast<int32_t>(T.leafDepth) - 1; i >= static_cast<int32_t>(min_level);
         i--) {
        const Vector2ui range(h->levelOffsets[i], h->levelOffsets[i + 1]);
        launch(range[1] - range[0], [&] {
            KCCollapseRayCounts(T.dBinInfo, T.dNodes, range, static_cast<uint32_t>(i), min_level,
                                min_ray_count);
        });
    }
    // KCCheckReducedSVOBins
    for (uint32_t i = 0; i < n; i++) {
        if (bin_out[i] == 0xFFFFFFFFu) continue;
        bool isLeaf;
        const uint32_t nb = T.FindMarkedBin(isLeaf, bin_out[i] & 0x7FFFFFFFu);
        if (!isLeaf) bin_out[i] = nb;
    }
}

// Payload the cone reads need: normal/specular words and half2 averages
// (leaf and node), in the layout of VoxelPayload (AnisoSVO.cuh:23-114).
void ref_svo_set_payload(void* p, const uint32_t* leaf_norm_spec, const uint32_t* node_norm_spec,
                         const uint32_t* leaf_avg, const uint32_t* node_avg) {
    RefSvo* h = static_cast<RefSvo*>(p);
    std::copy(leaf_norm_spec, leaf_norm_spec + h->leafNormSpec.size(), h->leafNormSpec.begin());
    std::copy(node_norm_spec, node_norm_spec + h->nodeNormSpec.size(), h->nodeNormSpec.begin());
    static_assert(sizeof(Vector2h) == 4, "half2");
    std::memcpy(h->leafAvg.data(), leaf_avg, 4 * h->leafAvg.size());
    std::memcpy(h->nodeAvg.data(), node_avg, 4 * h->nodeAvg.size());
}

// ConeTraceRay + ReadRadiance for n cones: t_out (the returned tMin),
// id_out (node / leaf index, 0xFFFFFFFF for a miss), leaf_out, rad_out.
void ref_svo_cone_trace(const void* p, const float* o, const float* d, const float* tmin,
                        const float* tmax, const float* aperture, uint32_t max_query_offset,
                        uint32_t n, float* t_out, uint32_t* id_out, uint8_t* leaf_out,
                        float* rad_out) {
    const RefSvo* h = static_cast<const RefSvo*>(p);
    const AnisoSVOctreeGPU& T = h->tree;
    for (uint32_t i = 0; i < n; i++) {
        RayF ray(Vector3f(d[3 * i], d[3 * i + 1], d[3 * i + 2]),
                 Vector3f(o[3 * i], o[3 * i + 1], o[3 * i + 2]));
        bool isLeaf = false;
        uint32_t id = UINT32_MAX;
        const float t = T.ConeTraceRay(isLeaf, id, ray, tmin[i], tmax[i], aperture[i],
                                       max_query_offset);
        t_out[i] = t;
        id_out[i] = id;
        leaf_out[i] = isLeaf ? 1 : 0;
        rad_out[i] = T.ReadRadiance(ray.getDirection(), aperture[i], id, isLeaf);
    }
}

// KCAverageNormals bottom-up over the node levels (AnisoSVO.cu:1066-1088)
// from the given leaf normal words; node words out.
void ref_svo_average_normals(void* p, const uint32_t* leaf_norm_spec, uint32_t* node_norm_spec) {
    RefSvo* h = static_cast<RefSvo*>(p);
    AnisoSVOctreeGPU& T = h->tree;
    std::copy(leaf_norm_spec, leaf_norm_spec + h->leafNormSpec.size(), h->leafNormSpec.begin());
    const uint32_t levelCount = T.leafDepth;
    for (uint32_t i = 0; i < levelCount; i++) {
        const uint32_t levelIndex = levelCount - i - 1;
        const bool lastNonLeafLevel = (levelIndex == (levelCount - 1));
        const uint32_t count = h->levelCounts[levelIndex];
        launch(count, [&] {
            KCAverageNormals(T.payload, T.dNodes, T.dLevelNodeOffsets, levelIndex, count,
                             lastNonLeafLevel);
        });
    }
    std::copy(h->nodeNormSpec.begin(), h->nodeNormSpec.end(), node_norm_spec);
}

// AnisoSVOctreeCPU::NormalizeAndFilterRadiance (AnisoSVO.cu:1415-1483): leaf
// averages from the FP32 sums and counts, bottom-up node averages, top-down
// fill of the empty ones.  Uses the normal words set by ref_svo_set_payload;
// leaf / node half2 averages out (u16 | u16 << 16).
void ref_svo_normalize_filter(void* p, const float* leaf_irr2, const uint32_t* leaf_cnt2,
                              uint32_t* leaf_avg, uint32_t* node_avg) {
    RefSvo* h = static_cast<RefSvo*>(p);
    AnisoSVOctreeGPU& T = h->tree;
    for (size_t l = 0; l < h->leafIrr.size(); l++) {
        h->leafIrr[l] = Vector2f(leaf_irr2[2 * l], leaf_irr2[2 * l + 1]);
        h->leafCnt[l] = Vector2ui(leaf_cnt2[2 * l], leaf_cnt2[2 * l + 1]);
    }
    launch(T.leafCount, [&] {
        KCCCopyRadianceToHalfBufferLeaf(T.payload.dAvgIrradianceLeaf,
                                        T.payload.dTotalIrradianceLeaf,
                                        T.payload.dSampleCountLeaf, T.leafCount, 1.0f);
    });
    const uint32_t levelCount = T.leafDepth;
    const std::vector<uint32_t>& offs = h->levelOffsets;
    for (uint32_t i = 0; i < levelCount; i++) {
        const uint32_t levelIndex = levelCount - i - 1;
        const bool lastNonLeafLevel = (levelIndex == (levelCount - 1));
        const uint32_t count = offs[levelIndex + 1] - offs[levelIndex];
        launch(count, [&] {
            KCBottomUpFilterIrradiance(T.payload, T.dNodes, T.dLevelNodeOffsets, levelIndex,
                                       count, lastNonLeafLevel);
        });
    }
    for (uint32_t i = 1; i <= levelCount; i++) {
        const bool isLeafLevel = (i == levelCount);
        const uint32_t count = offs[i + 1] - offs[i];
        launch(count, [&] {
            KCTopDownFilterIrradiance(T.payload, T.dNodes, T.dLeafParents, T.dLevelNodeOffsets,
                                      i, count, isLeafLevel);
        });
    }
    std::memcpy(leaf_avg, h->leafAvg.data(), 4 * h->leafAvg.size());
    std::memcpy(node_avg, h->nodeAvg.data(), 4 * h->nodeAvg.size());
}

// AnisoSVOctreeGPU::DepositRadiance (AnisoSVO.cuh:1080-1098 with
// VoxelPayload::WriteLeafRadiance :490-537) for n path vertices, in order,
// over zeroed accumulators; leaf sums (2 floats) and counts (2) out.  The
// surface normal and wi the reference passes are not read by it.
void ref_svo_deposit(void* p, const float* pos, const float* wo, const float* lum, uint32_t n,
                     float* leaf_irr2, uint32_t* leaf_cnt2) {
    RefSvo* h = static_cast<RefSvo*>(p);
    AnisoSVOctreeGPU& T = h->tree;
    std::fill(h->leafIrr.begin(), h->leafIrr.end(), Vector2f(0.0f, 0.0f));
    std::fill(h->leafCnt.begin(), h->leafCnt.end(), Vector2ui(0u, 0u));
    for (uint32_t i = 0; i < n; i++) {
        const Vector3f w(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        T.DepositRadiance(Vector3f(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), w, w, w, lum[i]);
    }
    for (size_t l = 0; l < h->leafIrr.size(); l++) {
        leaf_irr2[2 * l] = h->leafIrr[l][0];
        leaf_irr2[2 * l + 1] = h->leafIrr[l][1];
        leaf_cnt2[2 * l] = h->leafCnt[l][0];
        leaf_cnt2[2 * l + 1] = h->leafCnt[l][1];
    }
}

// AnisoSVOctreeGPU::DepositNEEHitMiss (AnisoSVO.cuh:1101-1115 with
// VoxelPayload::WriteLeafNEEHitMiss :540-545) for n vertices, in order, over
// zeroed counters: is_hit[i] picks the hit or the miss counter; per-leaf
// hits and misses out.
void ref_svo_deposit_nee(void* p, const float* pos, const uint8_t* is_hit, uint32_t n,
                         uint32_t* hit_out, uint32_t* miss_out) {
    RefSvo* h = static_cast<RefSvo*>(p);
    AnisoSVOctreeGPU& T = h->tree;
    std::fill(h->shadowHit.begin(), h->shadowHit.end(), 0u);
    std::fill(h->shadowMiss.begin(), h->shadowMiss.end(), 0u);
    for (uint32_t i = 0; i < n; i++)
        T.DepositNEEHitMiss(Vector3f(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), 1.0f,
                            is_hit[i] != 0);
    std::copy(h->shadowHit.begin(), h->shadowHit.end(), hit_out);
    std::copy(h->shadowMiss.begin(), h->shadowMiss.end(), miss_out);
}

// The guiding factors of KCBottomUpFilterIrradiance (AnisoSVO.cu:520-615)
// over the given per-leaf shadow-ray counters, level by level from the
// deepest; binary16 node factors out.  Uses the normal and radiance payload
// already set (the factors do not depend on it).
void ref_svo_guiding_factors(void* p, const uint32_t* hit, const uint32_t* miss,
                             uint16_t* node_factor) {
    RefSvo* h = static_cast<RefSvo*>(p);
    AnisoSVOctreeGPU& T = h->tree;
    std::copy(hit, hit + h->shadowHit.size(), h->shadowHit.begin());
    std::copy(miss, miss + h->shadowMiss.size(), h->shadowMiss.begin());
    const uint32_t levelCount = T.leafDepth;
    const std::vector<uint32_t>& offs = h->levelOffsets;
    for (uint32_t i = 0; i < levelCount; i++) {
        const uint32_t levelIndex = levelCount - i - 1;
        const bool lastNonLeafLevel = (levelIndex == (levelCount - 1));
        const uint32_t count = offs[levelIndex + 1] - offs[levelIndex];
        launch(count, [&] {
            KCBottomUpFilterIrradiance(T.payload, T.dNodes, T.dLevelNodeOffsets, levelIndex,
                                       count, lastNonLeafLevel);
        });
    }
    static_assert(sizeof(half) == 2, "half");
    std::memcpy(node_factor, h->nodeFactor.data(), 2 * h->nodeFactor.size());
}

}  // extern "C"
