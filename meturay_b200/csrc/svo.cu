// Sparse voxel octree of the scene (the path-guiding radiance cache):
// conservative voxelisation of every triangle and the level-by-level octree
// build, as AnisoSVOctreeCPU::Constrcut (AnisoSVO.cu:657-1188) with
// TriFunctions::Voxelize (GPUPrimitiveTriangle.h:385-620) and the
// KCGetVoxelCount / KCVoxelizePrims kernels (GPUAcceleratorCommonKC.cuh:440-542).
//
// The node array is canonical: level by level, and inside a level the nodes
// in Morton order of their prefixes.  The reference reaches that layout with
// per-level child marking, a scan of child counts and parent fix-ups
// (KCMarkChild / KCExtractChildrenCounts / KCSetChildrenPtrs /
// KCSetParentOf(Leaf)Children, AnisoSVO.cu:58-222).  Here each level's
// nodes are the distinct prefixes of the sorted unique voxel codes: a head
// flag per voxel and a prefix sum give every voxel its ancestor's rank at
// every level, and one pass per level writes the packed nodes from those
// ranks.  Packed node (AnisoSVO.cuh:125-151): child index bits 0-26, parent
// bits 27-54, child mask bits 55-62, "children are leaves" bit 63.
#include "../../include/mrb200.h"
#include "common.cuh"
#include "scan.cuh"
#include "sort.cuh"
#include "svo.cuh"
#include "svo_dev.cuh"

namespace mrb {
namespace {

constexpr uint64_t kInvalidNode = 0x007FFFFFFFFFFFFFull;

__device__ __forceinline__ uint64_t expand3d(uint32_t val) {
    uint64_t x = val;
    x &= 0x1fffff;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

struct V2 {
    float x, y;
};
__device__ __forceinline__ V3 cross3(V3 a, V3 b) { return cross(a, b); }

// TriFunctions::Voxelize (GPUPrimitiveTriangle.h:385-620), split into the
// per-triangle setup and one raster row, so that the rows of a large
// triangle run on separate threads.  Voxels of a triangle come out in the
// reference's order, rows bottom-up and pixels left to right; the row
// offsets of the build keep that order in the voxel array.
struct TriRaster {
    V2 q2[3], c0, ec0, ec1, e0, e1;
    V3 p0, p1, p2;
    float denomC, denom, deltaPix, res;
    uint32_t packedNormal;
    int x0, x1, y0, y1;
};

__device__ TriRaster tri_setup(const SvoParams& P, V3 p0, V3 p1, V3 p2) {
    const V3 pos[3] = {p0, p1, p2};
    const V3 normal = normalize(cross(p1 - p0, p2 - p0));
    const float an[3] = {fabsf(normal.x), fabsf(normal.y), fabsf(normal.z)};
    int dom = 0;
    float mx = an[0];
    if (an[1] > mx) { mx = an[1]; dom = 1; }
    if (an[2] > mx) { mx = an[2]; dom = 2; }
    const float nd = dom == 0 ? normal.x : (dom == 1 ? normal.y : normal.z);
    const bool neg = signbit(nd);
    const float domSign = neg ? -1.0f : 1.0f;
    // spherical coordinates of the normal packed to 2 x 16 bit
    const float az = pm_atan2(normal.y, normal.x);
    const float incl = pm_acos(fminf(fmaxf(normal.z, -1.0f), 1.0f));
    const float s0 = (az + kPiF) * kInvPiF * 0.5f;
    const float s1 = incl * kInvPiF;
    int u = static_cast<int>(s0 * 65535.0f), v = static_cast<int>(s1 * 65535.0f);
    u = u < 0 ? 0 : (u > 65535 ? 65535 : u);
    v = v < 0 ? 0 : (v > 65535 ? 65535 : v);
    const uint32_t packedNormal = uint32_t(u) | (uint32_t(v) << 16);
    // rotation that looks down the dominant axis: QuatF(angle, axis).  The
    // half angle is float(pi)/4 or float(pi)/2, whose sin and cos are taken
    // correctly rounded (the portable polynomials are an ulp off at pi/4,
    // which moves the conservative edges and with them whole voxel rows)
    Q4 rot = {1.0f, 0.0f, 0.0f, 0.0f};
    if (dom != 2 || neg) {
        const bool halfPi = (dom == 2);
        const float sn = halfPi ? 1.0f : 0x1.6a09e6p-1f;
        const float cs = halfPi ? -0x1.777a5cp-25f : 0x1.6a09e6p-1f;
        V3 axis;
        if (dom == 0) axis = v3(-domSign * 0.0f, -domSign * 1.0f, -domSign * 0.0f);
        else if (dom == 1) axis = v3(domSign * 1.0f, domSign * 0.0f, domSign * 0.0f);
        else axis = v3(0.0f, 1.0f, 0.0f);
        rot = Q4{cs, axis.x * sn, axis.y * sn, axis.z * sn};
    }
    // orthographic projection to NDC (TransformGen::Ortogonal, Matrix.hpp:1021-1039)
    const float l = P.lo[0], r = P.hi[0], t = P.hi[1], b = P.lo[1], nn = P.lo[2], f = P.hi[2];
    const float xt = -((r + l) / (r - l)), yt = -((t + b) / (t - b)), zt = -((f + nn) / (f - nn));
    const float xs = 2.0f / (r - l), ys = 2.0f / (t - b), zs = 2.0f / (f - nn);
    V2 q2[3];
    float amnx = kFltMax, amny = kFltMax, amxx = -kFltMax, amxy = -kFltMax;
    for (int i = 0; i < 3; i++) {
        V3 pt = {xs * pos[i].x + xt, ys * pos[i].y + yt, zs * pos[i].z + zt};
        pt = qrotate(rot, pt);
        q2[i] = V2{pt.x, pt.y};
        amnx = fminf(amnx, pt.x);
        amny = fminf(amny, pt.y);
        amxx = fmaxf(amxx, pt.x);
        amxy = fmaxf(amxy, pt.y);
    }
    const float res = static_cast<float>(P.res);
    int x0 = static_cast<int>(floorf((0.5f + 0.5f * amnx) * res));
    int x1 = static_cast<int>(ceilf((0.5f + 0.5f * amxx) * res));
    int y0 = static_cast<int>(floorf((0.5f + 0.5f * amny) * res));
    int y1 = static_cast<int>(ceilf((0.5f + 0.5f * amxy) * res));
    const int ri = static_cast<int>(P.res);
    x0 = min(max(x0, 0), ri);
    x1 = min(max(x1, 0), ri);
    y0 = min(max(y0, 0), ri);
    y1 = min(max(y1, 0), ri);
    // conservative rasterisation: edges moved out by half a pixel
    const float half = 1.0f / res;
    const float deltaPix = 2.0f * half;
    V3 pl[3];
    for (int i = 0; i < 3; i++) {
        const V2 a = q2[i], c = q2[(i + 1) % 3];
        pl[i] = cross3(v3(c.x - a.x, c.y - a.y, 0.0f), v3(a.x, a.y, 1.0f));
        pl[i].z -= half * fabsf(pl[i].x) + half * fabsf(pl[i].y);
    }
    const V3 pc0 = cross3(pl[0], pl[2]), pc1 = cross3(pl[0], pl[1]), pc2 = cross3(pl[1], pl[2]);
    const V2 c0 = {pc0.x / pc0.z, pc0.y / pc0.z}, c1 = {pc1.x / pc1.z, pc1.y / pc1.z},
             c2 = {pc2.x / pc2.z, pc2.y / pc2.z};
    const V2 ec0 = {c1.x - c0.x, c1.y - c0.y}, ec1 = {c2.x - c0.x, c2.y - c0.y};
    const float denomC = 1.0f / (ec0.x * ec1.y - ec1.x * ec0.y);
    const V2 e0 = {q2[1].x - q2[0].x, q2[1].y - q2[0].y}, e1 = {q2[2].x - q2[0].x, q2[2].y - q2[0].y};
    const float denom = 1.0f / (e0.x * e1.y - e1.x * e0.y);
    TriRaster R;
    for (int i = 0; i < 3; i++) R.q2[i] = q2[i];
    R.c0 = c0;
    R.ec0 = ec0;
    R.ec1 = ec1;
    R.e0 = e0;
    R.e1 = e1;
    R.p0 = p0;
    R.p1 = p1;
    R.p2 = p2;
    R.denomC = denomC;
    R.denom = denom;
    R.deltaPix = deltaPix;
    R.res = res;
    R.packedNormal = packedNormal;
    R.x0 = x0;
    R.x1 = x1;
    R.y0 = y0;
    R.y1 = y1;
    return R;
}

// Rows of the triangle's pixel rectangle (0 when it has no columns).
__device__ __forceinline__ uint32_t tri_rows(const TriRaster& R) {
    return (R.x1 > R.x0 && R.y1 > R.y0) ? uint32_t(R.y1 - R.y0) : 0u;
}

// Row y of the triangle: writes up to `maxOut` voxels when codes !=
// nullptr; returns the row's count.
__device__ uint32_t tri_row(const SvoParams& P, const TriRaster& R, int y, uint64_t* codes,
                            uint32_t* normals, uint32_t maxOut) {
    const V2 c0 = R.c0, ec0 = R.ec0, ec1 = R.ec1, e0 = R.e0, e1 = R.e1;
    const float denomC = R.denomC, denom = R.denom, deltaPix = R.deltaPix, res = R.res;
    uint32_t w = 0;
    for (int x = R.x0; x < R.x1; x++) {
        const V2 p = {(static_cast<float>(x) + 0.5f) * deltaPix - 1.0f,
                      (static_cast<float>(y) + 0.5f) * deltaPix - 1.0f};
        const V2 ec2 = {p.x - c0.x, p.y - c0.y};
        const float bb = (ec2.x * ec1.y - ec1.x * ec2.y) * denomC;
        const float cc = (ec0.x * ec2.y - ec2.x * ec0.y) * denomC;
        const float aa = 1.0f - bb - cc;
        if (!(bb >= 0.0f && bb <= 1.0f && cc >= 0.0f && cc <= 1.0f && aa >= 0.0f && aa <= 1.0f))
            continue;
        if (codes && w < maxOut) {
            const V2 e2 = {p.x - R.q2[0].x, p.y - R.q2[0].y};
            const float ab = (e2.x * e1.y - e1.x * e2.y) * denom;
            const float ac = (e0.x * e2.y - e2.x * e0.y) * denom;
            const float aA = 1.0f - ab - ac;
            const V3 vp = (R.p0 * aA + R.p1 * ab) + R.p2 * ac;
            uint32_t vi[3];
            const float vpc[3] = {vp.x, vp.y, vp.z};
            for (int k = 0; k < 3; k++) {
                float fi = (vpc[k] - P.lo[k]) / (P.hi[k] - P.lo[k]);
                fi *= res;
                uint32_t q = fi > 0.0f ? static_cast<uint32_t>(fi) : 0u;
                vi[k] = q > P.res - 1 ? P.res - 1 : q;
            }
            codes[w] = expand3d(vi[0]) | (expand3d(vi[1]) << 1) | (expand3d(vi[2]) << 2);
            normals[w] = R.packedNormal;
        }
        w++;
    }
    return w;
}

__device__ __forceinline__ void tri_pos(const SvoBuildIn& in, uint32_t t, V3& a, V3& b, V3& c) {
    const uint32_t i0 = in.idx[3 * size_t(t)], i1 = in.idx[3 * size_t(t) + 1],
                   i2 = in.idx[3 * size_t(t) + 2];
    a = ld3(in.pos + 3 * size_t(i0));
    b = ld3(in.pos + 3 * size_t(i1));
    c = ld3(in.pos + 3 * size_t(i2));
}

__global__ void __launch_bounds__(128) k_tri_rows(SvoBuildIn in, SvoParams P, uint32_t* rows) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < in.triCount;
         t += gridDim.x * blockDim.x) {
        V3 a, b, c;
        tri_pos(in, t, a, b, c);
        rows[t] = tri_rows(tri_setup(P, a, b, c));
    }
}

// The triangle of every row: row r of the flat list belongs to triangle t
// for rowStart[t] <= r < rowStart[t + 1].
__global__ void __launch_bounds__(256) k_row_tri(const uint32_t* __restrict__ rowStart, uint32_t T,
                                                 uint32_t* __restrict__ rowTri) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x)
        for (uint32_t r = rowStart[t]; r < rowStart[t + 1]; r++) rowTri[r] = t;
}

__global__ void __launch_bounds__(128) k_row_count(SvoBuildIn in, SvoParams P,
                                                   const uint32_t* __restrict__ rowStart,
                                                   const uint32_t* __restrict__ rowTri,
                                                   uint32_t rowsTotal, uint32_t* counts) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rowsTotal;
         r += gridDim.x * blockDim.x) {
        const uint32_t t = rowTri[r];
        V3 a, b, c;
        tri_pos(in, t, a, b, c);
        const TriRaster R = tri_setup(P, a, b, c);
        counts[r] = tri_row(P, R, R.y0 + int(r - rowStart[t]), nullptr, nullptr, 0);
    }
}

__global__ void __launch_bounds__(128) k_row_voxelize(SvoBuildIn in, SvoParams P,
                                                      const uint32_t* __restrict__ rowStart,
                                                      const uint32_t* __restrict__ rowTri,
                                                      uint32_t rowsTotal,
                                                      const uint32_t* __restrict__ offsets,
                                                      uint64_t* codes, uint32_t* normals,
                                                      uint32_t* lightKeys) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rowsTotal;
         r += gridDim.x * blockDim.x) {
        const uint32_t t = rowTri[r];
        V3 a, b, c;
        tri_pos(in, t, a, b, c);
        const TriRaster R = tri_setup(P, a, b, c);
        const uint32_t o = offsets[r], cnt = offsets[r + 1] - o;
        tri_row(P, R, R.y0 + int(r - rowStart[t]), codes + o, normals + o, cnt);
        const uint32_t key = in.key[t];
        const uint32_t lk = ((key >> kIdBits) == kBatchLight) ? key : 0u;
        for (uint32_t i = 0; i < cnt; i++) lightKeys[o + i] = lk;
    }
}

// EachPrimVoxelCount / VoxelizeSurfaces of an accelerator group
// (GPUAcceleratorI.h:113-133; KCGetVoxelCount / KCVoxelizePrims,
// GPUAcceleratorCommonKC.cuh:439-542): one thread per primitive, its
// vertices taken to world space by its surface's local-to-world matrix.
__device__ __forceinline__ void prim_world_pos(const PrimVoxIn& in, uint32_t t, V3& a, V3& b,
                                               V3& c) {
    const uint32_t i0 = in.idx[3 * size_t(t)], i1 = in.idx[3 * size_t(t) + 1],
                   i2 = in.idx[3 * size_t(t) + 2];
    a = ld3(in.pos + 3 * size_t(i0));
    b = ld3(in.pos + 3 * size_t(i1));
    c = ld3(in.pos + 3 * size_t(i2));
    if (in.triTransform) {
        const float* m = in.transforms + 12 * size_t(in.triTransform[t]);
        a = xform_point(m, a);
        b = xform_point(m, b);
        c = xform_point(m, c);
    }
}

__global__ void __launch_bounds__(128) k_prim_voxel_count(PrimVoxIn in, SvoParams P,
                                                          unsigned long long* counts) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < in.triCount;
         t += gridDim.x * blockDim.x) {
        V3 a, b, c;
        prim_world_pos(in, t, a, b, c);
        const TriRaster R = tri_setup(P, a, b, c);
        unsigned long long n = 0;
        if (tri_rows(R))
            for (int y = R.y0; y < R.y1; y++) n += tri_row(P, R, y, nullptr, nullptr, 0);
        counts[t] = n;
    }
}

__global__ void __launch_bounds__(128) k_prim_voxelize(PrimVoxIn in, SvoParams P,
                                                       const unsigned long long* __restrict__ offs,
                                                       uint64_t* codes, uint32_t* normals,
                                                       uint32_t* lightKeys,
                                                       const uint32_t* __restrict__ sortedLights,
                                                       uint32_t lightCount) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < in.triCount;
         t += gridDim.x * blockDim.x) {
        V3 a, b, c;
        prim_world_pos(in, t, a, b, c);
        const TriRaster R = tri_setup(P, a, b, c);
        const unsigned long long o = offs[t], cnt = offs[t + 1] - o;
        unsigned long long w = 0;
        if (tri_rows(R))
            for (int y = R.y0; y < R.y1 && w < cnt; y++)
                w += tri_row(P, R, y, codes + o + w, normals + o + w, uint32_t(cnt - w));
        // the primitive's work key if it is one of the (sorted) light keys
        const uint32_t key = in.key[t];
        uint32_t lo = 0, hi = lightCount;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sortedLights[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        const uint32_t lk = (lo < lightCount && sortedLights[lo] == key) ? key : 0u;
        for (unsigned long long i = 0; i < cnt; i++) lightKeys[o + i] = lk;
    }
}

__global__ void k_iota(uint32_t* v, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v[i] = i;
}

// head flag: the value differs from its predecessor after a right shift
__global__ void k_heads(const uint64_t* __restrict__ v, uint32_t n, uint32_t shift,
                        uint32_t* __restrict__ heads) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        heads[i] = (i == 0 || (v[i] >> shift) != (v[i - 1] >> shift)) ? 1u : 0u;
}

// unique voxel codes (RLE of the sorted codes) and run starts
__global__ void k_compact_unique(const uint64_t* __restrict__ sorted, uint32_t n,
                                 const uint32_t* __restrict__ heads,
                                 const uint32_t* __restrict__ rank, uint64_t* uniq,
                                 uint32_t* runStart) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (heads[i]) {
            uniq[rank[i]] = sorted[i];
            runStart[rank[i]] = i;
        }
    if (blockIdx.x == 0 && threadIdx.x == 0) runStart[rank[n]] = n;
}

__global__ void k_fill_u64(uint64_t* p, uint64_t v, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        p[i] = v;
}

// Rank of voxel j's ancestor group from an exclusive scan of head flags:
// the inclusive count at j, minus one.
__device__ __forceinline__ uint32_t anc(const uint32_t* __restrict__ scan, uint32_t j) {
    return scan[j + 1] - 1u;
}

// Nodes of level L: one writer per distinct prefix (its first voxel).
__global__ void k_level_nodes(const uint32_t* __restrict__ headsL,
                              const uint32_t* __restrict__ rankL,
                              const uint32_t* __restrict__ rankNext,
                              const uint32_t* __restrict__ rankPrev, uint32_t U,
                              uint32_t levelOffset, uint32_t nextOffset, uint32_t prevOffset,
                              int lastNodeLevel, int isRoot, uint64_t* nodes) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < U; j += gridDim.x * blockDim.x) {
        if (!headsL[j]) continue;
        const uint32_t node = levelOffset + anc(rankL, j);
        const uint32_t child = lastNodeLevel ? j : (nextOffset + anc(rankNext, j));
        const uint64_t parent = isRoot ? 0xFFFFFFFull : uint64_t(prevOffset + anc(rankPrev, j));
        uint64_t packed = uint64_t(child & 0x7FFFFFFu) | ((parent & 0xFFFFFFFull) << 27);
        if (lastNodeLevel) packed |= (1ull << 63);
        // the child mask (bits 55-62) is OR-ed in by k_child_mask
        nodes[node] = packed | (nodes[node] & (0xFFull << 55));
    }
}

// Child mask: every distinct prefix at level L+1 sets its bit in its parent.
__global__ void k_child_mask(const uint64_t* __restrict__ uniq,
                             const uint32_t* __restrict__ headsNext,
                             const uint32_t* __restrict__ rankL, uint32_t U, uint32_t levelOffset,
                             uint32_t shiftNext, unsigned long long* nodes) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < U; j += gridDim.x * blockDim.x) {
        if (!headsNext[j]) continue;
        const uint32_t childId = static_cast<uint32_t>(uniq[j] >> shiftNext) & 7u;
        atomicOr(nodes + levelOffset + anc(rankL, j), (1ull << (55 + childId)));
    }
}

__global__ void k_leaf_parents(const uint32_t* __restrict__ rankLast, uint32_t U,
                               uint32_t lastOffset, uint32_t* leafParents) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < U; j += gridDim.x * blockDim.x)
        leafParents[j] = lastOffset + anc(rankLast, j);
}

// Leaf payload, KCReduceVoxelPayload (AnisoSVOKC.cuh:8-320) with one thread
// per unique voxel: 2-means clustering of the voxel normals (4 passes;
// initial means n0 and -n0; the means are normalised at the start of each
// pass; a normal joins mean 0 when its angular distance to mean 0 is >= the
// distance to mean 1, as the reference compares), the larger cluster's mean
// becomes the leaf normal, and light voxels start with luminance x 10000
// samples on both sides (AnisoSVO.cuh SetLeafRadiance / SetLeafNormal).
// Sums run over the voxel's duplicates in sorted order; the reference's
// warp reductions add the same terms in a tree order.
__global__ void k_leaf_payload(const uint32_t* __restrict__ runStart,
                               const uint32_t* __restrict__ sortedIdx,
                               const uint32_t* __restrict__ normals,
                               const uint32_t* __restrict__ lightKeys,
                               const float* __restrict__ lightRad, uint32_t omitDirect,
                               uint32_t U, uint32_t* leafNormSpec, unsigned long long* leafIrr,
                               uint32_t* leafCnt, uint32_t* leafLight) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < U; j += gridDim.x * blockDim.x) {
        const uint32_t b = runStart[j], e = runStart[j + 1], dup = e - b;
        const V3 n0 = unpack_normal16(normals[sortedIdx[b]]);
        V3 m0 = n0, m1 = -n0;
        uint32_t c0 = 0, c1 = 0;
        for (int it = 0; it < 4; it++) {
            m0 = normalize(m0);
            m1 = normalize(m1);
            V3 a0 = v3(0.0f, 0.0f, 0.0f), a1 = v3(0.0f, 0.0f, 0.0f);
            uint32_t k0 = 0, k1 = 0;
            for (uint32_t i = b; i < e; i++) {
                const V3 n = unpack_normal16(normals[sortedIdx[i]]);
                if (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f) continue;
                const float d0 = 1.0f - dot(m0, n), d1 = 1.0f - dot(m1, n);
                if (d0 >= d1) {
                    a0 = a0 + n;
                    k0++;
                } else {
                    a1 = a1 + n;
                    k1++;
                }
            }
            m0 = a0;
            m1 = a1;
            c0 = k0;
            c1 = k1;
        }
        V3 mean = (c0 >= c1) ? m0 * (1.0f / static_cast<float>(c0)) : m1 * (1.0f / static_cast<float>(c1));
        float lum = 0.0f;
        uint32_t lk = 0;
        const uint32_t passes = (dup + 63u) / 64u;
        for (uint32_t pass = 0; pass < passes; pass++) {
            mean = normalize(mean);
            const uint32_t pe = min(e, b + (pass + 1) * 64u);
            for (uint32_t i = b + pass * 64u; i < pe; i++) {
                const uint32_t key = lightKeys[sortedIdx[i]];
                if (!key) continue;
                if (!lk) lk = key;
                const uint32_t li = key & kIdMask;
                const V3 r = ld3(lightRad + 3 * li);
                lum = lum + (0.2120f * r.x + 0.7150f * r.y + 0.0722f * r.z);
            }
        }
        unsigned long long fx = 0;
        uint32_t cnt = 0;
        if (lum != 0.0f) {
            lum /= static_cast<float>(dup);
            lum *= 10000.0f;
            if (omitDirect) lum = 0.0f;
            fx = (lum > 0.0f) ? __double2ull_rn(static_cast<double>(lum) * kFixScale) : 0ull;
            cnt = 10000u;
        }
        leafIrr[2 * j] = fx;
        leafIrr[2 * j + 1] = fx;
        leafCnt[2 * j] = cnt;
        leafCnt[2 * j + 1] = cnt;
        leafNormSpec[j] = write_normal_spec(mean, 0.0f);
        leafLight[j] = lk;
    }
}

inline uint32_t grid_of(uint32_t n) {
    uint32_t g = (n + 255) / 256;
    return g < 1 ? 1 : (g > 148u * 16u ? 148u * 16u : g);
}

}  // namespace

SvoParams svo_params(const float extent[6], uint32_t res) {
    // AnisoSVO.cu:669-680: a cube padded by one leaf voxel
    SvoParams P{};
    float span[3] = {extent[3] - extent[0], extent[4] - extent[1], extent[5] - extent[2]};
    int md = 0;
    if (span[1] > span[md]) md = 1;
    if (span[2] > span[md]) md = 2;
    const float world = span[md];
    const float pad = world / static_cast<float>(res);
    for (int c = 0; c < 3; c++) {
        P.lo[c] = extent[c] - pad;
        P.hi[c] = extent[c] + (pad + world);
    }
    P.res = res;
    uint32_t d = 0;
    while ((1u << (d + 1)) <= res) d++;
    P.depth = d;
    P.leafVoxelSize = (world + 2.0f * pad) / static_cast<float>(res);
    return P;
}

int svo_build(const SvoBuildIn& in, const SvoParams& P, SvoResult& out, cudaStream_t st) {
    const uint32_t T = in.triCount;
    if (T == 0 || P.depth == 0 || P.depth > 10) {
        set_error("SVO: need triangles and a resolution between 2 and 1024");
        return MRB_E_ARG;
    }
    auto alloc = [](void** p, size_t bytes) -> int {
        cudaError_t e = cudaMalloc(p, bytes ? bytes : 4);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("SVO: cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
            return MRB_E_OOM;
        }
        return 0;
    };
    std::vector<void*> temps;
    auto tmp = [&](size_t bytes) -> void* {
        void* p = nullptr;
        if (alloc(&p, bytes)) return nullptr;
        temps.push_back(p);
        return p;
    };
    auto cleanup = [&]() {
        for (void* p : temps) cudaFree(p);
        temps.clear();
    };
    int r = 0;
    // 1. raster rows of every triangle, voxel counts per row, voxelisation
    // (rows in triangle order, so the voxel array keeps the per-triangle
    // order of the reference)
    uint32_t* rows = static_cast<uint32_t*>(tmp(size_t(T) * 4));
    uint32_t* rowStart = static_cast<uint32_t*>(tmp((size_t(T) + 1) * 4));
    void* scanTmp = tmp(exclusive_scan_temp_bytes(T + 1));
    if (!rows || !rowStart || !scanTmp) { cleanup(); return MRB_E_OOM; }
    k_tri_rows<<<grid_of(T), 128, 0, st>>>(in, P, rows);
    if ((r = exclusive_scan_u32(rows, rowStart, T, scanTmp, st))) { cleanup(); return r; }
    uint32_t rowsTotal = 0;
    MRB_CUDA(cudaMemcpyAsync(&rowsTotal, rowStart + T, 4, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    if (rowsTotal == 0) { cleanup(); set_error("SVO: no voxels"); return MRB_E_ARG; }
    uint32_t* rowTri = static_cast<uint32_t*>(tmp(size_t(rowsTotal) * 4));
    uint32_t* counts = static_cast<uint32_t*>(tmp(size_t(rowsTotal) * 4));
    uint32_t* offsets = static_cast<uint32_t*>(tmp((size_t(rowsTotal) + 1) * 4));
    void* scanRows = tmp(exclusive_scan_temp_bytes(rowsTotal + 1));
    if (!rowTri || !counts || !offsets || !scanRows) { cleanup(); return MRB_E_OOM; }
    k_row_tri<<<grid_of(T), 256, 0, st>>>(rowStart, T, rowTri);
    k_row_count<<<grid_of(rowsTotal), 128, 0, st>>>(in, P, rowStart, rowTri, rowsTotal, counts);
    if ((r = exclusive_scan_u32(counts, offsets, rowsTotal, scanRows, st))) { cleanup(); return r; }
    uint32_t total = 0;
    MRB_CUDA(cudaMemcpyAsync(&total, offsets + rowsTotal, 4, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    if (total == 0) { cleanup(); set_error("SVO: no voxels"); return MRB_E_ARG; }
    if (total > (1u << 27)) { cleanup(); set_error("SVO: %u voxels exceed 2^27", total); return MRB_E_ARG; }
    uint64_t* codes = static_cast<uint64_t*>(tmp(size_t(total) * 8));
    uint32_t* vnorm = static_cast<uint32_t*>(tmp(size_t(total) * 4));
    uint32_t* vlight = static_cast<uint32_t*>(tmp(size_t(total) * 4));
    uint32_t* vidx = static_cast<uint32_t*>(tmp(size_t(total) * 4));
    const size_t sortBytes = radix_sort_temp_bytes(total, 8, 0, int(3 * P.depth + 1));
    void* sortTmp = tmp(sortBytes);
    uint32_t* heads = static_cast<uint32_t*>(tmp((size_t(total) + 1) * 4));
    uint32_t* rank = static_cast<uint32_t*>(tmp((size_t(total) + 1) * 4));
    void* scanTmp2 = tmp(exclusive_scan_temp_bytes(total + 1));
    if (!codes || !vnorm || !vlight || !vidx || !sortTmp || !heads || !rank || !scanTmp2) {
        cleanup();
        return MRB_E_OOM;
    }
    k_row_voxelize<<<grid_of(rowsTotal), 128, 0, st>>>(in, P, rowStart, rowTri, rowsTotal, offsets,
                                                       codes, vnorm, vlight);
    k_iota<<<grid_of(total), 256, 0, st>>>(vidx, total);
    // 2. sort on bits [0, 3*depth + 1) and run-length encode
    if ((r = radix_sort_pairs<uint64_t>(codes, vidx, nullptr, total, 0, int(3 * P.depth + 1), false,
                                        sortTmp, sortBytes, st, false))) {
        cleanup();
        return r;
    }
    k_heads<<<grid_of(total), 256, 0, st>>>(codes, total, 0, heads);
    if ((r = exclusive_scan_u32(heads, rank, total, scanTmp2, st))) { cleanup(); return r; }
    uint32_t U = 0;
    MRB_CUDA(cudaMemcpyAsync(&U, rank + total, 4, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    out.voxelCount = total;
    out.leafCount = U;
    if ((r = alloc(reinterpret_cast<void**>(&out.leafCodes), size_t(U) * 8)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafRunStart), (size_t(U) + 1) * 4))) {
        cleanup();
        return r;
    }
    k_compact_unique<<<grid_of(total), 256, 0, st>>>(codes, total, heads, rank, out.leafCodes,
                                                     out.leafRunStart);
    // 3. ranks of every voxel's ancestor at every level
    const uint32_t D = P.depth;
    std::vector<uint32_t*> lh(D + 1), lr(D + 1);
    for (uint32_t L = 0; L <= D; L++) {
        lh[L] = static_cast<uint32_t*>(tmp((size_t(U) + 1) * 4));
        lr[L] = static_cast<uint32_t*>(tmp((size_t(U) + 1) * 4));
        if (!lh[L] || !lr[L]) { cleanup(); return MRB_E_OOM; }
        k_heads<<<grid_of(U), 256, 0, st>>>(out.leafCodes, U, 3 * (D - L), lh[L]);
        if ((r = exclusive_scan_u32(lh[L], lr[L], U, scanTmp2, st))) { cleanup(); return r; }
    }
    std::vector<uint32_t> counts_(D + 1);
    for (uint32_t L = 0; L <= D; L++)
        MRB_CUDA(cudaMemcpyAsync(&counts_[L], lr[L] + U, 4, cudaMemcpyDeviceToHost, st));
    MRB_CUDA(cudaStreamSynchronize(st));
    out.levelOffsets.assign(D + 2, 0);
    for (uint32_t L = 0; L <= D; L++) out.levelOffsets[L + 1] = out.levelOffsets[L] + counts_[L];
    out.nodeCount = out.levelOffsets[D];
    if ((r = alloc(reinterpret_cast<void**>(&out.nodes), size_t(out.nodeCount) * 8)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafParents), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafNormSpec), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafLight), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&out.nodeNormSpec), size_t(out.nodeCount) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafIrr), size_t(U) * 16)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafCnt), size_t(U) * 8)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafAvg), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&out.nodeAvg), size_t(out.nodeCount) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafShadow), size_t(U) * 8)) ||
        (r = alloc(reinterpret_cast<void**>(&out.nodeFactor), size_t(out.nodeCount) * 2)) ||
        (r = alloc(reinterpret_cast<void**>(&out.leafBin), size_t(U) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&out.nodeBin), size_t(out.nodeCount) * 4)) ||
        (r = alloc(reinterpret_cast<void**>(&out.dLevelOffsets), out.levelOffsets.size() * 4))) {
        cleanup();
        return r;
    }
    // nodes start as INVALID_NODE with an empty child mask
    k_fill_u64<<<grid_of(out.nodeCount), 256, 0, st>>>(out.nodes, kInvalidNode & ~(0xFFull << 55),
                                                       out.nodeCount);
    for (uint32_t L = 0; L < D; L++) {
        k_child_mask<<<grid_of(U), 256, 0, st>>>(out.leafCodes, lh[L + 1], lr[L], U,
                                                 out.levelOffsets[L], 3 * (D - L - 1),
                                                 reinterpret_cast<unsigned long long*>(out.nodes));
    }
    for (uint32_t L = 0; L < D; L++) {
        const bool last = (L == D - 1);
        k_level_nodes<<<grid_of(U), 256, 0, st>>>(
            lh[L], lr[L], lr[L + 1], L ? lr[L - 1] : lr[L], U, out.levelOffsets[L],
            last ? 0u : out.levelOffsets[L + 1], L ? out.levelOffsets[L - 1] : 0u, last ? 1 : 0,
            L == 0 ? 1 : 0, out.nodes);
    }
    k_leaf_parents<<<grid_of(U), 256, 0, st>>>(lr[D - 1], U, out.levelOffsets[D - 1],
                                              out.leafParents);
    k_leaf_payload<<<grid_of(U), 256, 0, st>>>(out.leafRunStart, vidx, vnorm, vlight, in.lightRad,
                                              in.omitDirect, U, out.leafNormSpec, out.leafIrr,
                                              out.leafCnt, out.leafLight);
    // shadow-ray counters start at zero (AnisoSVO.cu:1029-1030)
    MRB_CUDA(cudaMemsetAsync(out.leafShadow, 0, size_t(U) * 8, st));
    MRB_CUDA(cudaMemcpyAsync(out.dLevelOffsets, out.levelOffsets.data(),
                             out.levelOffsets.size() * 4, cudaMemcpyHostToDevice, st));
    MRB_CUDA(cudaGetLastError());
    MRB_CUDA(cudaStreamSynchronize(st));
    cleanup();
    return 0;
}

void svo_free(SvoResult& r) {
    cudaFree(r.nodes);
    cudaFree(r.leafParents);
    cudaFree(r.leafCodes);
    cudaFree(r.leafRunStart);
    cudaFree(r.leafLight);
    cudaFree(r.leafNormSpec);
    cudaFree(r.nodeNormSpec);
    cudaFree(r.leafIrr);
    cudaFree(r.leafCnt);
    cudaFree(r.leafAvg);
    cudaFree(r.nodeAvg);
    cudaFree(r.leafShadow);
    cudaFree(r.nodeFactor);
    cudaFree(r.leafBin);
    cudaFree(r.nodeBin);
    cudaFree(r.dLevelOffsets);
    r = SvoResult{};
}

int prim_voxel_count(const PrimVoxIn& in, const SvoParams& P, unsigned long long* counts,
                     cudaStream_t st) {
    if (in.triCount == 0) return 0;
    const uint32_t blocks = std::min((in.triCount + 127) / 128, 148u * 16u);
    k_prim_voxel_count<<<blocks, 128, 0, st>>>(in, P, counts);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

int prim_voxelize(const PrimVoxIn& in, const SvoParams& P, const unsigned long long* offsets,
                  uint64_t* codes, uint32_t* normals, uint32_t* lightKeys,
                  const uint32_t* sortedLights, uint32_t lightCount, cudaStream_t st) {
    if (in.triCount == 0) return 0;
    const uint32_t blocks = std::min((in.triCount + 127) / 128, 148u * 16u);
    k_prim_voxelize<<<blocks, 128, 0, st>>>(in, P, offsets, codes, normals, lightKeys,
                                            sortedLights, lightCount);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

}  // namespace mrb
