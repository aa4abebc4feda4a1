// Device-side view of the sparse voxel octree radiance cache used by the
// path guider: packing helpers, tree queries (descend, nearest leaf,
// marked-bin search), the stackless cone trace and the radiance read.
//
// Reference: AnisoSVO.cuh (AnisoSVOctreeGPU, VoxelPayload) and
// RayLib/CoordinateConversion.h of yalcinerbora/meturay.  Every routine
// keeps the reference's operation order; the oracle restates the same
// steps on the host.  Conversions that C leaves undefined for NaN or
// out-of-range values go through explicit saturating helpers so both
// sides agree.
#pragma once
#include "common.cuh"

namespace mrb {

// ---------------------------------------------------------------------------
// conversions
// ---------------------------------------------------------------------------
// float -> uint32 toward zero, NaN and negatives to 0, saturating above
__host__ __device__ __forceinline__ uint32_t f2u_sat(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967040.0f) return 0xFFFFFFFFu;
    return static_cast<uint32_t>(x);
}
// float -> int32 toward zero, NaN to 0, saturating
__host__ __device__ __forceinline__ int32_t f2i_sat(float x) {
    if (x != x) return 0;
    if (x >= 2147483520.0f) return 0x7FFFFFFF;
    if (x <= -2147483648.0f) return static_cast<int32_t>(0x80000000u);
    return static_cast<int32_t>(x);
}

__host__ __device__ __forceinline__ uint32_t fbits(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
    return u;
#endif
}
__host__ __device__ __forceinline__ float bitsf(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}

// IEEE binary32 -> binary16, round to nearest even (NaN kept quiet)
__host__ __device__ __forceinline__ uint16_t f2h(float f) {
    const uint32_t x = fbits(f);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t ax = x & 0x7FFFFFFFu;
    if (ax > 0x7F800000u) return static_cast<uint16_t>(sign | 0x7E00u);
    if (ax >= 0x47800000u) return static_cast<uint16_t>(sign | 0x7C00u);
    if (ax < 0x38800000u) {  // half subnormal or zero
        const uint32_t e = ax >> 23;
        if (e == 0) return static_cast<uint16_t>(sign);
        const uint32_t m = (ax & 0x7FFFFFu) | 0x800000u;
        const uint32_t s = 126u - e;  // >= 14
        if (s > 24u) return static_cast<uint16_t>(sign);
        uint32_t q = m >> s;
        const uint32_t rem = m & ((1u << s) - 1u), halfway = 1u << (s - 1u);
        if (rem > halfway || (rem == halfway && (q & 1u))) q++;
        return static_cast<uint16_t>(sign | q);
    }
    uint32_t h = (((ax >> 23) - 112u) << 10) | ((ax & 0x7FFFFFu) >> 13);
    const uint32_t rem = ax & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
    return static_cast<uint16_t>(sign | h);
}
__host__ __device__ __forceinline__ float h2f(uint16_t h) {
    const uint32_t sign = (uint32_t(h) & 0x8000u) << 16;
    const uint32_t e = (h >> 10) & 0x1Fu, m = h & 0x3FFu;
    if (e == 0) {
        if (m == 0) return bitsf(sign);
        // subnormal: m * 2^-24
        const float v = static_cast<float>(m) * 0x1p-24f;
        return sign ? -v : v;
    }
    if (e == 31) return bitsf(sign | 0x7F800000u | (m << 13));
    return bitsf(sign | ((e + 112u) << 23) | (m << 13));
}

// next float toward +inf (nextafter(x, INFINITY) for finite x)
__host__ __device__ __forceinline__ float next_up(float x) {
    if (x != x || x == bitsf(0x7F800000u)) return x;
    if (x == 0.0f) return bitsf(1u);
    const uint32_t b = fbits(x);
    return bitsf(x > 0.0f ? b + 1u : b - 1u);
}

// 32-bit integer hash "lowbias32" (C. Wellons, hash-prospector)
__host__ __device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// ---------------------------------------------------------------------------
// co-centric octahedral map (RayLib/CoordinateConversion.h:112-233)
// ---------------------------------------------------------------------------
constexpr float kTwoOvrPiF = 0x1.45f306p-1f;  // float(2 / pi)
constexpr float kPiOvr4F = 0x1.921fb6p-1f;    // float(pi / 4)

// DirectionToCocentricOctohedral (:112-146); atan(y/x) for x, y >= 0 is
// the portable atan2.  An exact pole direction maps to (0, 0) as in the
// reference.
__device__ __forceinline__ void dir_to_octa(V3 d, float& s, float& t) {
    if (d.x == 0.0f && d.y == 0.0f) {
        s = 0.0f;
        t = 0.0f;
        return;
    }
    const float xAbs = fabsf(d.x), yAbs = fabsf(d.y);
    const float phiPrime = pm_atan2(yAbs, xAbs);
    const float radius = sqrtf(1.0f - fabsf(d.z));
    float v = radius * kTwoOvrPiF * phiPrime;
    float u = radius - v;
    if (d.z < 0.0f) {
        const float up = 1.0f - v, vp = 1.0f - u;
        u = up;
        v = vp;
    }
    u *= signbit(d.x) ? -1.0f : 1.0f;
    v *= signbit(d.y) ? -1.0f : 1.0f;
    s = (u + 1.0f) * 0.5f;
    t = (v + 1.0f) * 0.5f;
}
// CocentricOctohedralToDirection (:148-183)
__device__ __forceinline__ V3 octa_to_dir(float s, float t) {
    const float u = s * 2.0f - 1.0f, v = t * 2.0f - 1.0f;
    const float ua = fabsf(u), va = fabsf(v);
    const float d = 1.0f - (ua + va);
    const float radius = 1.0f - fabsf(d);
    float phiPrime = 0.0f;
    if (radius != 0.0f) phiPrime = ((va - ua) / radius + 1.0f) * kPiOvr4F;
    float sp, cp;
    pm_sincos(phiPrime, sp, cp);
    const float cosPhi = (signbit(u) ? -1.0f : 1.0f) * cp;
    const float sinPhi = (signbit(v) ? -1.0f : 1.0f) * sp;
    const float z = (signbit(d) ? -1.0f : 1.0f) * (1.0f - radius * radius);
    const float xyFactor = radius * sqrtf(2.0f - radius * radius);
    return v3(cosPhi * xyFactor, sinPhi * xyFactor, z);
}
// the guider's frames are y-up: (x, y, z) of the map -> (y, z, x)
__device__ __forceinline__ V3 octa_to_dir_yup(float s, float t) {
    const V3 r = octa_to_dir(s, t);
    return v3(r.y, r.z, r.x);
}
__device__ __forceinline__ void dir_yup_to_octa(V3 d, float& s, float& t) {
    dir_to_octa(v3(d.z, d.x, d.y), s, t);
}
// CocentricOctohedralWrap (:185-213) for st in any range
__device__ __forceinline__ void octa_wrap(float& s, float& t) {
    float a = s, b = t;
    if (s < 0.0f) a = -2.0f - s;
    if (t < 0.0f) b = -2.0f - t;
    const float ia = truncf(a), ib = truncf(b);
    float fa = fabsf(a - ia), fb = fabsf(b - ib);
    const int32_t ii = f2i_sat(ia), ij = f2i_sat(ib);
    if ((ii & 1) ^ (ij & 1)) {
        fa = 1.0f - fa;
        fb = 1.0f - fb;
    }
    s = fa;
    t = fb;
}
// CocentricOctohedralWrapInt (:215-233)
__host__ __device__ __forceinline__ void octa_wrap_int(int32_t& x, int32_t& y, int32_t dimX,
                                                       int32_t dimY) {
    int32_t a = x, b = y;
    if (x < 0) a = -2 * dimX - x;
    if (y < 0) b = -2 * dimY - y;
    const int32_t ia = a / dimX, ib = b / dimY;
    int32_t fa = a % dimX, fb = b % dimY;
    fa = fa < 0 ? -fa : fa;
    fb = fb < 0 ? -fb : fb;
    if ((ia & 1) ^ (ib & 1)) {
        fa = (dimX - 1) - fa;
        fb = (dimY - 1) - fb;
    }
    x = fa;
    y = fb;
}

// Utility::SphericalToCartesianUnit / CartesianToSphericalUnit with the
// 2 x 16-bit UNORM packing of voxel and path-node normals
// (PathNode.cuh WFPGPathNode::Normal / SetNormal)
__device__ __forceinline__ uint32_t pack_normal16(V3 n) {
    const float az = pm_atan2(n.y, n.x);
    const float incl = pm_acos(fminf(fmaxf(n.z, -1.0f), 1.0f));
    const float s0 = (az + kPiF) * kInvPiF * 0.5f;
    const float s1 = incl * kInvPiF;
    int u = f2i_sat(s0 * 65535.0f), v = f2i_sat(s1 * 65535.0f);
    u = u < 0 ? 0 : (u > 65535 ? 65535 : u);
    v = v < 0 ? 0 : (v > 65535 ? 65535 : v);
    return uint32_t(u) | (uint32_t(v) << 16);
}
__device__ __forceinline__ V3 unpack_normal16(uint32_t pn) {
    const float az = static_cast<float>(pn & 0xFFFFu) / 65535.0f * (kPiF * 2.0f) - kPiF;
    const float in = static_cast<float>(pn >> 16) / 65535.0f * kPiF;
    float sa, ca, si, ci;
    pm_sincos(az, sa, ca);
    pm_sincos(in, si, ci);
    return normalize(v3(ca * si, sa * si, ci));
}

// ---------------------------------------------------------------------------
// octree and payload
// ---------------------------------------------------------------------------
constexpr uint32_t kSvoInvalidParent = 0xFFFFFFFu;  // 28 parent bits
constexpr uint32_t kBinMark = 0x80000000u;          // bin word: mark bit | ray count
constexpr uint32_t kBinLeaf = 0x80000000u;          // bin id: leaf flag | index
constexpr uint32_t kBinInvalid = 0xFFFFFFFFu;
constexpr uint16_t kHalfMax = 0x7BFFu;              // 65504
constexpr uint16_t kFactorNone = 0x7FFFu;           // guiding factor without data: the binary16
                                                    // NaN the reference's conversion of NaN gives
constexpr double kFixScale = 16777216.0;            // radiance sums: 2^24 fixed point

struct GuideDev {
    const uint64_t* nodes;
    const uint32_t* leafParents;
    const uint32_t* levelOffsets;  // leafDepth + 2 entries
    uint32_t nodeCount, leafCount, leafDepth, res;
    float lo[3], hi[3];
    float leafVoxelSize;
    // payload
    uint32_t* leafNormSpec;        // VoxelPayload normal/specular word
    uint32_t* nodeNormSpec;
    unsigned long long* leafIrr;   // 2 per leaf: fixed-point radiance sums (front, back)
    uint32_t* leafCnt;             // 2 per leaf: sample counts
    uint32_t* leafAvg;             // half2: averaged radiance (front | back << 16)
    uint32_t* nodeAvg;
    uint32_t* leafShadow;          // 2 per leaf: NEE shadow rays that reached / missed their light
    uint16_t* nodeFactor;          // half: mean miss ratio of the children (kFactorNone: no data)
    // ray bins
    uint32_t* leafBin;
    uint32_t* nodeBin;
};

__device__ __forceinline__ uint32_t svo_child_index(uint64_t n) { return uint32_t(n & 0x7FFFFFFull); }
__device__ __forceinline__ uint32_t svo_parent(uint64_t n) { return uint32_t((n >> 27) & 0xFFFFFFFull); }
__device__ __forceinline__ uint32_t svo_mask(uint64_t n) { return uint32_t((n >> 55) & 0xFFull); }
__device__ __forceinline__ bool svo_children_leaf(uint64_t n) { return (n >> 63) != 0; }
__device__ __forceinline__ uint32_t svo_child_offset(uint64_t n, uint32_t c) {
    return __popc(((1u << c) - 1u) & svo_mask(n));
}

__device__ __forceinline__ float level_voxel_size(const GuideDev& g, uint32_t level) {
    return g.leafVoxelSize * static_cast<float>(1u << (g.leafDepth - level));
}

__device__ __forceinline__ uint64_t expand3(uint32_t val) {
    uint64_t x = val & 0x1fffffu;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

// AnisoSVOctreeGPU::Descend (AnisoSVO.cuh:1128-1155)
__device__ __forceinline__ bool svo_descend(const GuideDev& g, uint32_t& index, uint64_t code,
                                            uint32_t depth) {
    uint32_t shift = (g.leafDepth - 1) * 3;
    uint32_t cur = 0;
    for (uint32_t i = 0; i < depth; i++) {
        const uint64_t node = g.nodes[cur];
        const uint32_t childId = uint32_t(code >> shift) & 7u;
        if (!((svo_mask(node) >> childId) & 1u)) return false;
        cur = svo_child_index(node) + svo_child_offset(node, childId);
        shift -= 3;
    }
    index = cur;
    return true;
}

// AnisoSVOctreeGPU::NearestNodeIndex (AnisoSVO.cuh:1171-1242): the voxel of
// the point, then its 7 neighbours toward the nearest faces
__device__ __forceinline__ bool svo_nearest(const GuideDev& g, uint32_t& index, V3 p,
                                            uint32_t depth) {
    index = kInvalid;
    if (!(p.x >= g.lo[0] && p.x <= g.hi[0] && p.y >= g.lo[1] && p.y <= g.hi[1] &&
          p.z >= g.lo[2] && p.z <= g.hi[2]))
        return false;
    const float vs = level_voxel_size(g, depth);
    const float li[3] = {(p.x - g.lo[0]) / vs, (p.y - g.lo[1]) / vs, (p.z - g.lo[2]) / vs};
    float fr[3], fl[3];
    uint32_t inc[3];
    for (int c = 0; c < 3; c++) {
        const float ip = truncf(li[c]);
        fr[c] = li[c] - ip;
        fl[c] = floorf(li[c]);
        inc[c] = (fr[c] < 0.5f) ? 0xFFFFFFFFu : 1u;
        fr[c] = 0.5f - fabsf(fr[c] - 0.5f);
    }
    int m0 = 0;
    if (fr[1] < fr[m0]) m0 = 1;
    if (fr[2] < fr[m0]) m0 = 2;
    const float a = fr[(m0 + 1) % 3], b = fr[(m0 + 2) % 3];
    int m1 = (b < a) ? 1 : 0;
    m1 = (m0 + m1 + 1) % 3;
    const int m2 = 3 - m0 - m1;
    const uint32_t dense[3] = {f2u_sat(fl[0]), f2u_sat(fl[1]), f2u_sat(fl[2])};
    for (uint32_t i = 0; i < 8; i++) {
        uint32_t sh[3];
        sh[m0] = i & 1u;
        sh[m1] = (i >> 1) & 1u;
        sh[m2] = (i >> 2) & 1u;
        const uint32_t vx = dense[0] + sh[0] * inc[0], vy = dense[1] + sh[1] * inc[1],
                       vz = dense[2] + sh[2] * inc[2];
        const uint64_t code = expand3(vx) | (expand3(vy) << 1) | (expand3(vz) << 2);
        if (svo_descend(g, index, code, depth)) return true;
    }
    return false;
}

// VoxelPayload::ReadNormalAndSpecular (AnisoSVO.cuh:396-432)
__device__ __forceinline__ V3 read_normal_spec(uint32_t packed, float& stdDev, float& spec) {
    const float kx = (1.0f / 511.0f) * 2.0f;
    float nx = static_cast<float>(packed & 511u) * kx;
    float ny = static_cast<float>((packed >> 9) & 511u) * kx;
    nx -= 1.0f;
    ny -= 1.0f;
    const float nz = sqrtf(fmaxf(0.0f, 1.0f - nx * nx - ny * ny));
    V3 n = normalize(v3(nx, ny, nz));
    if ((packed >> 31) & 1u) n.z *= -1.0f;
    const float len = static_cast<float>((packed >> 18) & 127u) * (1.0f / 127.0f);
    // the reference scales the 6 specular bits by 1 / 6 (its bit count)
    spec = static_cast<float>((packed >> 25) & 63u) * (1.0f / 6.0f);
    stdDev = (1.0f - len) / len;
    return n;
}
// VoxelPayload::WriteNormalAndSpecular (AnisoSVO.cuh:542-580)
__device__ __forceinline__ uint32_t write_normal_spec(V3 n, float spec) {
    const float length = sqrtf(dot(n, n));
    const float il = 1.0f / length;
    float x = n.x * il, y = n.y * il;
    x += 1.0f;
    y += 1.0f;
    x *= 0.5f;
    y *= 0.5f;
    x *= 511.0f;
    y *= 511.0f;
    const uint32_t px = f2u_sat(x), py = f2u_sat(y);
    const uint32_t pl = f2u_sat(length * 127.0f);
    const uint32_t ps = f2u_sat(spec * 63.0f);
    const uint32_t sz = signbit(n.z) ? 1u : 0u;
    return (px & 511u) | ((py & 511u) << 9) | ((pl & 127u) << 18) | ((ps & 63u) << 25) | (sz << 31);
}

// AnisoSVOctreeGPU::ReadRadiance + VoxelPayload::ReadRadiance
// (AnisoSVO.cuh:434-478,1040-1055): the side of the surface facing the
// cone origin.  No boundary light: a cone that leaves the octree reads 0.
__device__ __forceinline__ float read_radiance(const GuideDev& g, V3 coneDir, uint32_t id,
                                               bool isLeaf) {
    if (id == kInvalid) return 0.0f;
    float sd, sp;
    const V3 n = read_normal_spec(isLeaf ? g.leafNormSpec[id] : g.nodeNormSpec[id], sd, sp);
    const bool towardsNormal = dot(n, -coneDir) >= 0.0f;
    const uint32_t w = isLeaf ? g.leafAvg[id] : g.nodeAvg[id];
    return h2f(static_cast<uint16_t>(towardsNormal ? (w & 0xFFFFu) : (w >> 16)));
}

// AnisoSVOctreeGPU::ConeTraceRay (AnisoSVO.cuh:767-1000): stackless
// traversal of the [0,1]^3-normalised octree with the ray mirrored to the
// positive octant and a 3-bit-per-level Morton stack.  Stops at a leaf, or
// at the first node whose size is below the cone's footprint.  The loop is
// bounded (kConeTraceMaxSteps); a ray that needs more steps reports a miss.
constexpr uint32_t kConeTraceMaxSteps = 1u << 16;

__device__ __forceinline__ float neg_exp2i(uint32_t p) {  // 2^-p for p <= 126
    return (p == 0) ? 1.0f : bitsf((127u - p) << 23);
}

// The reference steps into an empty child, then on the next iteration
// computes that child's exit, moves tMin past it and pops.  Here that pair
// of iterations is one: the empty child's exit is computed in place.  The
// corner moves by powers of two and stays exactly representable, so the
// add/subtract pair of the reference changes nothing and the operations
// that reach tMin are the same.  The voxel size test uses a per-level
// table of the same products.
// The descent that every cone from one origin shares.  At the start of a
// trace, tMin moves only when a cone skips an empty child, so while the
// point origin + dir * tMin lies on the same side of each centre plane for
// every direction, each cone takes the same children as a descent by the
// origin alone.  "Same side for every direction" means the origin is
// farther than |dir| * tMin from each plane in the normalised frame (|dir|
// at most the largest axis scale), plus a slack far above the rounding of
// the cone's own plane crossings (a few ulps of values in [0, 1]).  The
// prefix stops before the first level where that fails, where the child is
// empty, or where the descent would terminate.  A termination that every
// cone reaches on the shared path (leaf child, or a voxel smaller than the
// cone's footprint at the common tMin) is recorded as the result of every
// cone.  The cone then starts at the prefix's node with the corner and
// Morton stack its own descent would have built (mirrored per direction:
// the corner 1 - c - span, the stack bits xor the mirror mask), both exact
// in binary32 since they are dyadic with at most leafDepth bits.
struct ConePrefix {
    uint32_t nodeId;     // node reached (0: no shared descent)
    uint32_t depth;      // its level
    uint32_t stack;      // child ids on the way down, unmirrored, 3 bits each
    float corner[3];     // its minimum corner in the normalised frame
    uint32_t termId;     // with `term`: the node every cone stops at
    uint32_t term;       // 1: every cone stops at termId
    uint32_t termLeaf;   // ... which is a leaf
};

__device__ __forceinline__ float level_voxel_size_sqr(const GuideDev& g, uint32_t level) {
    const uint32_t sh = (level <= g.leafDepth) ? g.leafDepth - level : 0u;
    const float vs = g.leafVoxelSize * static_cast<float>(1u << sh);
    return vs * vs;
}

__device__ __forceinline__ ConePrefix cone_prefix(const GuideDev& g, V3 pos, float tMin,
                                                  float aperture, uint32_t maxQueryLevelOffset) {
    ConePrefix P{};
    const V3 sc = v3(1.0f / (g.hi[0] - g.lo[0]), 1.0f / (g.hi[1] - g.lo[1]),
                     1.0f / (g.hi[2] - g.lo[2]));
    const V3 p = (pos + v3(-g.lo[0], -g.lo[1], -g.lo[2])) * sc;
    const float pa[3] = {p.x, p.y, p.z};
    const float scMax = fmaxf(fmaxf(sc.x, sc.y), sc.z);
    const float margin = tMin * scMax * 1.0001f + 4.0e-6f;
    if (!(margin < 0.25f)) return P;
    for (int a = 0; a < 3; a++)
        if (!(pa[a] > margin && pa[a] < 1.0f - margin)) return P;
    float corner[3] = {0.0f, 0.0f, 0.0f};
    uint32_t nodeId = 0, stack = 0;
    const float area = tMin * tMin * aperture;
    const float diam2 = 4.0f * (area * kInvPiF);
    for (uint32_t level = 0; level < g.leafDepth; level++) {
        const float half = neg_exp2i(level + 1);
        uint32_t c = 0;
        for (int a = 0; a < 3; a++) {
            const float ctr = corner[a] + half;
            if (!(fabsf(pa[a] - ctr) > margin)) return P;
            if (pa[a] > ctr) c |= 1u << a;
        }
        const uint64_t node = g.nodes[nodeId];
        if (!((svo_mask(node) >> c) & 1u)) return P;
        const uint32_t child = svo_child_index(node) + svo_child_offset(node, c);
        const uint32_t lvl = level + 1;
        const bool childLeaf = svo_children_leaf(node);
        const bool term = diam2 > level_voxel_size_sqr(g, lvl) ||
                          (g.leafDepth - lvl) <= maxQueryLevelOffset;
        if (childLeaf || term) {
            P.term = 1;
            P.termLeaf = childLeaf ? 1u : 0u;
            P.termId = child;
            return P;
        }
        for (int a = 0; a < 3; a++)
            if ((c >> a) & 1u) corner[a] += half;
        stack = (stack << 3) | c;
        nodeId = child;
        P.nodeId = nodeId;
        P.depth = lvl;
        P.stack = stack;
        P.corner[0] = corner[0];
        P.corner[1] = corner[1];
        P.corner[2] = corner[2];
    }
    return P;
}

// The trace in two parts: cone_begin is the setup before the loop,
// cone_step one iteration of it.  The Morton stack holds at
// most leafDepth <= 10 levels of 3 bits.
struct ConeState {
    V3 dc, pb, corner;
    float tMin;
    uint32_t mirror, stack, depth, nodeId, step;
};

// True when the trace has already ended (NaN input, or a termination that
// the prefix shares); isLeaf / leafId then hold the result.
__device__ __forceinline__ bool cone_begin(const GuideDev& g, V3 pos, V3 dir, float tMin,
                                           const ConePrefix* pre, ConeState& s, bool& isLeaf,
                                           uint32_t& leafId) {
    const float EPS = 1.0e-5f;
    leafId = kInvalid;
    isLeaf = false;
    if (fabsf(dir.x) < EPS) dir.x = copysignf(EPS, dir.x);
    if (fabsf(dir.y) < EPS) dir.y = copysignf(EPS, dir.y);
    if (fabsf(dir.z) < EPS) dir.z = copysignf(EPS, dir.z);
    const V3 sc = v3(1.0f / (g.hi[0] - g.lo[0]), 1.0f / (g.hi[1] - g.lo[1]),
                     1.0f / (g.hi[2] - g.lo[2]));
    V3 d = dir * sc;
    V3 p = (pos + v3(-g.lo[0], -g.lo[1], -g.lo[2])) * sc;
    s.tMin = tMin;
    if (!(d.x == d.x && d.y == d.y && d.z == d.z && p.x == p.x && p.y == p.y && p.z == p.z))
        return true;
    p.x = (d.x < 0.0f) ? (1.0f - p.x) : p.x;
    p.y = (d.y < 0.0f) ? (1.0f - p.y) : p.y;
    p.z = (d.z < 0.0f) ? (1.0f - p.z) : p.z;
    uint32_t mirror = 0;
    if (d.x < 0.0f) mirror |= 1u;
    if (d.y < 0.0f) mirror |= 2u;
    if (d.z < 0.0f) mirror |= 4u;
    s.mirror = mirror;
    s.dc = v3(1.0f / fabsf(d.x), 1.0f / fabsf(d.y), 1.0f / fabsf(d.z));
    s.pb = p * s.dc;
    {
        const V3 t0 = -s.pb;
        const float tSvo = fmaxf(fmaxf(t0.x, t0.y), t0.z);
        if (!(t0.x < s.tMin && t0.y < s.tMin && t0.z < s.tMin)) s.tMin = next_up(tSvo);
    }
    s.stack = 0;
    s.depth = 0;
    s.nodeId = 0;
    s.step = 0;
    s.corner = v3(0.0f, 0.0f, 0.0f);
    if (pre) {
        if (pre->term) {
            isLeaf = pre->termLeaf != 0;
            leafId = pre->termId;
            return true;
        }
        if (pre->depth) {
            const float span = neg_exp2i(pre->depth);
            s.corner = v3((mirror & 1u) ? 1.0f - pre->corner[0] - span : pre->corner[0],
                          (mirror & 2u) ? 1.0f - pre->corner[1] - span : pre->corner[1],
                          (mirror & 4u) ? 1.0f - pre->corner[2] - span : pre->corner[2]);
            uint32_t pattern = 0;
            for (uint32_t j = 0; j < pre->depth; j++) pattern = (pattern << 3) | mirror;
            s.stack = pre->stack ^ pattern;
            s.depth = pre->depth;
            s.nodeId = pre->nodeId;
            s.step = pre->depth;
        }
    }
    return false;
}

// Per-level constants of the cone loop, computed once per block: span[L] =
// 2^-L (neg_exp2i) and vs2[L] = the squared voxel size of level L
// (level_voxel_size_sqr).  Same values as computing them in the loop.
struct ConeTables {
    const float* span;  // 12 entries (levels 0..11)
    const float* vs2;   // 11 entries (levels 0..10)
};

// One iteration of the reference's loop.  The empty-child skip takes the
// child's exit crossings from values the iteration already has: per axis
// the child's far plane is the node's far plane (child bit set: corner +
// span/2 + span/2 = corner + span, exact for these dyadic corners) or its
// centre plane, so the crossings are tm or tc, value for value.  True when
// the trace has ended.
__device__ __forceinline__ bool cone_step(const GuideDev& g, float aperture,
                                          uint32_t maxQueryLevelOffset, ConeState& s,
                                          bool& isLeaf, uint32_t& leafId,
                                          const ConeTables* tab = nullptr) {
    if (s.step == kConeTraceMaxSteps) {
        leafId = kInvalid;
        isLeaf = false;
        return true;
    }
    s.step++;
    const float childSpan = tab ? tab->span[s.depth + 1] : neg_exp2i(s.depth + 1);
    const float curSpan = tab ? tab->span[s.depth] : neg_exp2i(s.depth);
    const V3 topRight = s.corner + v3(curSpan, curSpan, curSpan);
    const V3 tm = topRight * s.dc - s.pb;
    const float tMax = fminf(fminf(tm.x, tm.y), tm.z);
    const uint64_t node = g.nodes[s.nodeId];
    if (tMax < s.tMin) {
        const uint32_t b = s.stack & 7u;
        s.corner = s.corner - v3((b & 1u) ? curSpan : 0.0f, (b & 2u) ? curSpan : 0.0f,
                                 (b & 4u) ? curSpan : 0.0f);
        s.stack >>= 3;
        s.depth -= 1;
        s.nodeId = svo_parent(node);
        return s.nodeId == kSvoInvalidParent;  // left the tree: a miss
    }
    const V3 center = s.corner + v3(childSpan, childSpan, childSpan);
    const V3 tc = center * s.dc - s.pb;
    uint32_t childId = 0;
    if (tc.x < s.tMin) childId |= 1u;
    if (tc.y < s.tMin) childId |= 2u;
    if (tc.z < s.tMin) childId |= 4u;
    const uint32_t mir = childId ^ s.mirror;
    if (!((svo_mask(node) >> mir) & 1u)) {
        // empty child: leave it at once
        const float ex = (childId & 1u) ? tm.x : tc.x;
        const float ey = (childId & 2u) ? tm.y : tc.y;
        const float ez = (childId & 4u) ? tm.z : tc.z;
        s.tMin = next_up(fminf(fminf(ex, ey), ez));
        return false;
    }
    const uint32_t child = svo_child_index(node) + svo_child_offset(node, mir);
    const uint32_t level = s.depth + 1;
    const float area = s.tMin * s.tMin * aperture;
    const float diam2 = 4.0f * (area * kInvPiF);
    bool term = diam2 > (tab ? tab->vs2[level] : level_voxel_size_sqr(g, level));
    const bool childLeaf = svo_children_leaf(node);
    term |= (g.leafDepth - level) <= maxQueryLevelOffset;
    if (childLeaf || term) {
        isLeaf = childLeaf;
        leafId = child;
        return true;
    }
    s.nodeId = child;
    s.corner = s.corner + v3((childId & 1u) ? childSpan : 0.0f, (childId & 2u) ? childSpan : 0.0f,
                             (childId & 4u) ? childSpan : 0.0f);
    s.stack = (s.stack << 3) | childId;
    s.depth = level;
    return false;
}

__device__ __forceinline__ float cone_trace(const GuideDev& g, V3 pos, V3 dir, float tMin,
                                            float aperture, uint32_t maxQueryLevelOffset,
                                            bool& isLeaf, uint32_t& leafId,
                                            const ConePrefix* pre = nullptr,
                                            const ConeTables* tab = nullptr) {
    ConeState s;
    if (cone_begin(g, pos, dir, tMin, pre, s, isLeaf, leafId)) return s.tMin;
    while (!cone_step(g, aperture, maxQueryLevelOffset, s, isLeaf, leafId, tab)) {
    }
    return s.tMin;
}

// AnisoSVOctreeGPU::FindMarkedBin (AnisoSVO.cuh:1244-1262): walk up from
// the leaf to the first marked bin
__device__ __forceinline__ uint32_t svo_marked_bin(const GuideDev& g, uint32_t leaf, bool& isLeaf) {
    isLeaf = true;
    uint32_t bin = g.leafBin[leaf];
    uint32_t parent = g.leafParents[leaf];
    uint32_t node = leaf;
    while (parent != kSvoInvalidParent && !(bin & kBinMark)) {
        node = parent;
        bin = g.nodeBin[parent];
        parent = svo_parent(g.nodes[parent]);
        isLeaf = false;
    }
    return node;
}

// AnisoSVOctreeGPU::NodeLevel / NodeVoxelSize (AnisoSVO.cuh:1276-1298)
__device__ __forceinline__ uint32_t svo_node_level(const GuideDev& g, uint32_t id, bool isLeaf) {
    if (isLeaf) return g.leafDepth;
    uint32_t lvl = 0;
    while (lvl + 1 < g.leafDepth && g.levelOffsets[lvl + 1] <= id) lvl++;
    return lvl;
}

}  // namespace mrb
