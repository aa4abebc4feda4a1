// Shared device definitions for the meturay_b200 wavefront path-tracing core.
//
// Arithmetic convention: every translation unit is compiled with
// -fmad=false, so a*b+c is two rounded operations exactly as written;
// fused multiply-adds appear only where __fmaf_rn is spelled out.  The
// per-ray math follows the operation order of the MRay reference
// (yalcinerbora/meturay) functions cited next to each routine.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

namespace mrb {

// ---------------------------------------------------------------------------
// HitKey layout (RayLib/HitStructs.h:154): 8 batch bits over 24 id bits.
// Batch ids of this core; NullBatch (0) sorts last under the descending
// partition order (RayLib/Types.h:10).
// ---------------------------------------------------------------------------
constexpr uint32_t kBatchNull = 0;
constexpr uint32_t kBatchLambert = 1;
constexpr uint32_t kBatchMetal = 2;
constexpr uint32_t kBatchRefract = 3;
constexpr uint32_t kBatchLight = 4;
constexpr uint32_t kBatchLambertC = 5;
constexpr uint32_t kBatchUnreal = 6;
constexpr uint32_t kBatchCount = 7;
constexpr uint32_t kIdBits = 24;
constexpr uint32_t kIdMask = 0xFFFFFFu;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr float kFltMax = 3.40282347e+38f;

// Ray types (RayAuxStruct.cuh RayType)
constexpr uint8_t kNeeRay = 0, kSpecPathRay = 1, kPathRay = 2, kCameraRay = 3;
constexpr uint32_t kTagCamera = 0x10000u;

// ---------------------------------------------------------------------------
// Device-resident layouts
// ---------------------------------------------------------------------------
// Traversal node: both child boxes live in the parent (64 B, 4 x 16 B loads).
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   d = (child0, child1, -, -): >= 0 inner node, < 0 leaf ~sortedTri
struct alignas(16) BvhNode {
    float4 a, b, c;
    int4 d;
};

struct RayAux {            // RayAuxPath (RayAuxStruct.cuh:27-40), 32 B
    float rf[3];           // radiance factor
    uint32_t sample;       // sample index
    uint32_t endpoint;     // light index for NEE rays
    uint16_t medium;
    uint8_t depth;
    uint8_t type;
    float prevPDF;
    uint32_t pad;
};

struct SceneDev {
    uint32_t vertexCount, triCount;
    const float* pos;            // 3 * vertexCount
    const float4* tbn;           // (w,x,y,z) per vertex
    const uint32_t* idx;         // 3 * triCount
    const uint32_t* triKey;      // per triangle HitKey
    const uint8_t* triCull;      // per triangle, 1 = cull back faces
    const float* lambertAlbedo;  // 3 per Lambert material
    const float* metalParams;    // eta3 k3 spec3 roughness
    const float* refractAlbedo;  // 3 per Refract material
    const uint32_t* refractMedium;
    const float* lambertCAlbedo; // 3 per LambertC material
    const float* unrealParams;   // albedo3 roughness metallic specular
    const float* lightRadiance;  // 3 per primitive light
    const uint32_t* lightPrim;
    uint32_t lightCount;
    const float* mediumIor;
    uint32_t baseMedium;
};

struct AccelDev {
    const BvhNode* nodes;  // inner nodes (n-1)
    const float4* tv0;     // sorted triangles: v0.xyz, w = original index bits
    const float4* te0;     // e0 = v1 - v0, w = HitKey bits
    const float4* te1;     // e1 = v2 - v0, w = cull flag
    int root;              // inner index, or ~0 for a single triangle
    uint32_t triCount;
};

struct CameraDev {         // GPUCameraPinhole frame (GPUCameraPinhole.cuh:135-162)
    float position[3];
    float bottomLeft[3];
    float right[3];
    float up[3];
    float planeSize[2];
    float nearFar[2];
};

struct PathOptions {
    uint32_t width, height, samples;   // samples: s -> s*s per pixel
    uint32_t maxDepth, rrStart, nee, mis;
    uint32_t seedLo, seedHi;
    const uint32_t* frame;             // device word: iteration index (RNG counter)
    uint32_t wfpg;                     // WFPG tracer: camera rays at depth 1, path chain kept
};

// ---------------------------------------------------------------------------
// Small vector / quaternion helpers (RayLib/Vector.hpp, Quaternion.hpp)
// ---------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};
struct Q4 {
    float w, x, y, z;
};
__device__ __forceinline__ V3 v3(float a, float b, float c) { return V3{a, b, c}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ bool nonzero(V3 a) { return a.x != 0.0f || a.y != 0.0f || a.z != 0.0f; }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 normalize(V3 v) {
    float inv = 1.0f / sqrtf(dot(v, v));
    return {v.x * inv, v.y * inv, v.z * inv};
}
__device__ __forceinline__ V3 vmax0(V3 v) { return {fmaxf(v.x, 0.0f), fmaxf(v.y, 0.0f), fmaxf(v.z, 0.0f)}; }
__device__ __forceinline__ V3 vsqrt(V3 v) { return {sqrtf(v.x), sqrtf(v.y), sqrtf(v.z)}; }
__device__ __forceinline__ V3 vdiv(V3 a, V3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
__device__ __forceinline__ V3 ld3(const float* p) { return {p[0], p[1], p[2]}; }
// Row-major 3x4 affine matrix m applied to a point (w = 1) and a direction
// (w = 0), each row summed left to right: Matrix4x4 * Vector4 of
// Ray::Transform (RayLib/Ray.hpp:459-465) without the constant fourth row.
__device__ __forceinline__ V3 xform_point(const float* m, V3 p) {
    return {((m[0] * p.x + m[1] * p.y) + m[2] * p.z) + m[3],
            ((m[4] * p.x + m[5] * p.y) + m[6] * p.z) + m[7],
            ((m[8] * p.x + m[9] * p.y) + m[10] * p.z) + m[11]};
}
__device__ __forceinline__ V3 xform_dir(const float* m, V3 d) {
    return {(m[0] * d.x + m[1] * d.y) + m[2] * d.z, (m[4] * d.x + m[5] * d.y) + m[6] * d.z,
            (m[8] * d.x + m[9] * d.y) + m[10] * d.z};
}

__device__ __forceinline__ Q4 qmul(Q4 a, Q4 b) {  // Quaternion.hpp:76-89
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
            a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
__device__ __forceinline__ Q4 qconj(Q4 q) { return {q.w, -q.x, -q.y, -q.z}; }
__device__ __forceinline__ float qdot(Q4 a, Q4 b) { return a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Q4 qnormalize(Q4 q) {
    float inv = 1.0f / sqrtf(qdot(q, q));
    return {q.w * inv, q.x * inv, q.y * inv, q.z * inv};
}
__device__ __forceinline__ V3 qrotate(Q4 q, V3 v) {  // Quaternion.hpp:229-238
    Q4 r = qmul(q, qmul(Q4{0.0f, v.x, v.y, v.z}, qconj(q)));
    return {r.x, r.y, r.z};
}
__device__ __forceinline__ V3 to_space(V3 v, Q4 q) { return qrotate(qconj(q), v); }
__device__ __forceinline__ V3 to_tangent(V3 v, Q4 q) { return qrotate(q, v); }
__device__ __forceinline__ Q4 q_from(float4 f) { return {f.x, f.y, f.z, f.w}; }

// ---------------------------------------------------------------------------
// Portable math.  sin/cos: Cody-Waite reduction by pi/2 (three-part split),
// Taylor polynomials on [-pi/4, pi/4].  acos: asin Taylor series on
// [0, 1/2] with the half-angle identity above.  Bit-identical to the host
// copy of the same steps, so FP32 paths do not diverge between the CPU
// check and the device.
// ---------------------------------------------------------------------------
constexpr float kPiF = 0x1.921fb6p+1f;
constexpr float kPio2F = 0x1.921fb6p+0f;
constexpr float kInvPiF = 0x1.45f306p-2f;

__device__ __forceinline__ float pm_sin_poly(float r) {
    float r2 = r * r;
    float p = -0x1.ae6456p-26f;
    p = p * r2 + 0x1.71de3ap-19f;
    p = p * r2 + -0x1.a01a02p-13f;
    p = p * r2 + 0x1.111112p-7f;
    p = p * r2 + -0x1.555556p-3f;
    return r + (r * r2) * p;
}
__device__ __forceinline__ float pm_cos_poly(float r) {
    float r2 = r * r;
    float p = 0x1.1eed8ep-29f;
    p = p * r2 + -0x1.27e4fcp-22f;
    p = p * r2 + 0x1.a01a02p-16f;
    p = p * r2 + -0x1.6c16c2p-10f;
    p = p * r2 + 0x1.555556p-5f;
    p = p * r2 + -0.5f;
    return 1.0f + r2 * p;
}
__device__ __forceinline__ void pm_sincos(float x, float& s, float& c) {
    float kf = rintf(x * 0x1.45f306p-1f);
    int k = static_cast<int>(kf);
    float r = x - kf * 0x1.92p+0f;
    r = r - kf * 0x1.fb4p-12f;
    r = r - kf * 0x1.4442d2p-24f;
    float sr = pm_sin_poly(r), cr = pm_cos_poly(r);
    switch (k & 3) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
}
__device__ __forceinline__ float pm_sin(float x) {
    float s, c;
    pm_sincos(x, s, c);
    return s;
}
__device__ __forceinline__ float pm_asin_poly(float z) {
    float z2 = z * z;
    float p = 0x1.df3bd4p-8f;
    p = p * z2 + 0x1.12ef3cp-7f;
    p = p * z2 + 0x1.3fde50p-7f;
    p = p * z2 + 0x1.7a8788p-7f;
    p = p * z2 + 0x1.c9999ap-7f;
    p = p * z2 + 0x1.1c4ec4p-6f;
    p = p * z2 + 0x1.6e8ba2p-6f;
    p = p * z2 + 0x1.f1c71cp-6f;
    p = p * z2 + 0x1.6db6dcp-5f;
    p = p * z2 + 0x1.333334p-4f;
    p = p * z2 + 0x1.555556p-3f;
    return z + (z * z2) * p;
}
__device__ __forceinline__ float pm_acos(float x) {
    float ax = fabsf(x);
    if (ax <= 0.5f) {
        float a = pm_asin_poly(ax);
        a = (x < 0.0f) ? -a : a;
        return kPio2F - a;
    }
    float z = sqrtf((1.0f - ax) * 0.5f);
    float a = 2.0f * pm_asin_poly(z);
    return (x > 0.0f) ? a : (kPiF - a);
}

// asin on [0, 1] from the same series (half-angle identity above 1/2)
__device__ __forceinline__ float pm_asin01(float z) {
    if (z <= 0.5f) return pm_asin_poly(z);
    return kPio2F - 2.0f * pm_asin_poly(sqrtf((1.0f - z) * 0.5f));
}
// atan2 from atan(a) = asin(a / sqrt(1 + a^2)) on a = min/max in [0, 1]
__device__ __forceinline__ float pm_atan2(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
    if (mx == 0.0f) return 0.0f;
    const float a = mn / mx;
    float r = pm_asin01(a / sqrtf(1.0f + a * a));
    if (ay > ax) r = kPio2F - r;
    if (x < 0.0f) r = kPiF - r;
    return (y < 0.0f) ? -r : r;
}

// exp(x): Cody-Waite reduction x = k ln2 + r with ln2 split into a 16-bit
// head (45426 / 2^16, so k * head is exact for |k| < 369) and the float
// nearest the remainder; e^r from its Taylor series through r^8 / 8!
// (|r| <= ln2 / 2, truncation below 2^-26); 2^k applied in two exact
// power-of-two steps so results down to the subnormal range round once.
__host__ __device__ __forceinline__ float pm_bits_float(int b) {
#ifdef __CUDA_ARCH__
    return __int_as_float(b);
#else
    float f;
    memcpy(&f, &b, 4);
    return f;
#endif
}
__host__ __device__ __forceinline__ float pm_exp(float x) {
    if (x != x) return x;
    if (x > 88.72283f) return pm_bits_float(0x7F800000);
    if (x < -103.97208f) return 0.0f;
    const float kf = rintf(x * 0x1.715476p+0f);
    const int k = static_cast<int>(kf);
    float r = x - kf * 0x1.62e4p-1f;
    r = r - kf * 0x1.7f7d1cp-20f;
    float p = 0x1.a01a02p-16f;
    p = p * r + 0x1.a01a02p-13f;
    p = p * r + 0x1.6c16c2p-10f;
    p = p * r + 0x1.111112p-7f;
    p = p * r + 0x1.555556p-5f;
    p = p * r + 0x1.555556p-3f;
    p = p * r + 0.5f;
    p = p * r + 1.0f;
    p = p * r + 1.0f;
    // k in [-150, 128]: 2^k = 2^k1 * 2^k2 with both factors normal
    const int k1 = k / 2, k2 = k - k1;
    p = p * pm_bits_float((k1 + 127) << 23);
    return p * pm_bits_float((k2 + 127) << 23);
}

// Quat::SLerp / Quat::BarySLerp (Quaternion.hpp:258-318)
__device__ __forceinline__ Q4 slerp(Q4 s, Q4 e, float t) {
    float cosT = qdot(s, e);
    float cosF = (cosT >= 0.0f) ? cosT : (-cosT);
    float s0, s1;
    if (cosF < (1.0f - 1.0e-5f)) {
        float angle = pm_acos(cosF);
        float sa = pm_sin(angle);
        s0 = pm_sin(angle * (1.0f - t)) / sa;
        s1 = pm_sin(angle * t) / sa;
    } else {
        s0 = (1.0f - t);
        s1 = t;
    }
    s1 = (cosT >= 0.0f) ? s1 : (-s1);
    return {s.w * s0 + e.w * s1, s.x * s0 + e.x * s1, s.y * s0 + e.y * s1, s.z * s0 + e.z * s1};
}
__device__ __forceinline__ Q4 bary_slerp(Q4 q0, Q4 q1, Q4 q2, float a, float b) {
    float c = (1.0f - a - b);
    if (fabsf(a + b) < 1.0e-5f) return q2;
    float ab = a / (a + b);
    Q4 qAB = slerp(q1, q0, ab);
    return slerp(qAB, q2, c);
}

// Ray::Nudge (RayLib/Ray.hpp:503-556), Ray Tracing Gems I ch. 6.
__device__ __forceinline__ float nudge1(float p, float d) {
    int ofi = static_cast<int>(256.0f * d);
    float pI = __int_as_float(__float_as_int(p) + ((p < 0.0f) ? -ofi : ofi));
    return (fabsf(p) < (1.0f / 32.0f)) ? (p + (1.0f / 65536.0f) * d) : pI;
}
__device__ __forceinline__ V3 nudge(V3 p, V3 d) { return {nudge1(p.x, d.x), nudge1(p.y, d.y), nudge1(p.z, d.z)}; }

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  Counter =
// {sample, frame, tag, block}, key = seed.  Uniform = top 24 bits * 2^-24.
// ---------------------------------------------------------------------------
struct Rand4 {
    float u[4];
};
__device__ __forceinline__ Rand4 philox_uniform4(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                 uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    Rand4 o;
    o.u[0] = static_cast<float>(c0 >> 8) * 0x1p-24f;
    o.u[1] = static_cast<float>(c1 >> 8) * 0x1p-24f;
    o.u[2] = static_cast<float>(c2 >> 8) * 0x1p-24f;
    o.u[3] = static_cast<float>(c3 >> 8) * 0x1p-24f;
    return o;
}

}  // namespace mrb

// Error reporting from host code (defined in runtime.cu)
namespace mrb {
void set_error(const char* fmt, ...);
}
#define MRB_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            ::mrb::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,             \
                             cudaGetErrorString(e_));                               \
            return -1;                                                              \
        }                                                                           \
    } while (0)
