// Shim that compiles MRay's own host-callable routines (and, through
// fragments cut at build time from the reference sources, its LBVH
// construction kernels run as host loops) into oracle/_ref/libmrayref.so.
//
// TEST INFRASTRUCTURE ONLY: it is used by tests/golden/make_golden.py to
// generate golden vectors from the reference itself.  Nothing here is part
// of the product, and no reference source is copied into this repository:
// the reference headers are #included from REF_ROOT and the LBVH fragments
// are extracted into oracle/_ref/ (git-ignored) by oracle/Makefile.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
using std::isinf;
using std::isnan;
using std::max;
using std::min;
using std::sqrt;

#include "RayLib/Types.h"
#include "RayLib/AABB.h"
#include "RayLib/Constants.h"
#include "RayLib/HemiDistribution.h"
#include "RayLib/MortonCode.h"
#include "RayLib/Quaternion.h"
#include "RayLib/Ray.h"
#include "RayLib/Triangle.h"
#include "RayLib/Vector.h"
#include "TracerCUDA/RNGenerator.h"
#include "TracerCUDA/TracerFunctions.cuh"

// ---- host stand-ins for the CUDA built-ins the LBVH kernels use --------
// Each simulated thread runs to completion before the next one starts, so
// plain loads/stores stand in for the atomics.
static uint3 blockIdx, threadIdx;
static dim3 blockDim, gridDim;
static inline int __clzll(long long x) { return x ? __builtin_clzll((unsigned long long)x) : 64; }
static inline unsigned int atomicExch(unsigned int* a, unsigned int v) {
    unsigned int o = *a;
    *a = v;
    return o;
}
static inline unsigned int atomicInc(unsigned int* a, unsigned int lim) {
    unsigned int o = *a;
    *a = (o >= lim) ? 0 : o + 1;
    return o;
}
static inline void __syncthreads() {}
#undef __shared__
#define __shared__ static

// LBVHNode (LinearBVH.cuh:21-43) and the kernels (LinearBVH.hpp:30-100,
// 168-247, 290-363), cut out of the reference by oracle/Makefile.
#include "lbvh_node.inc"
#include "lbvh_kernels.inc"

namespace {
struct FixedRng : public RNGeneratorGPUI {
    float v[8];
    int i = 0;
    float Uniform() override { return v[i++]; }
    float Uniform(float a, float b) override { return a + (b - a) * v[i++]; }
    Vector2f Uniform2D() override {
        float a = v[i++];
        float b = v[i++];
        return Vector2f(a, b);
    }
    float Normal() override { return 0.0f; }
    float Normal(float, float) override { return 0.0f; }
};
inline Vector3f V(const float* p) { return Vector3f(p[0], p[1], p[2]); }
inline void W(float* o, const Vector3f& v) { o[0] = v[0]; o[1] = v[1]; o[2] = v[2]; }
inline QuatF Q(const float* p) { return QuatF(p[0], p[1], p[2], p[3]); }
inline void WQ(float* o, const QuatF& q) { o[0] = q[0]; o[1] = q[1]; o[2] = q[2]; o[3] = q[3]; }

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
struct EmptyLeaf {};
}  // namespace

extern "C" {

uint64_t ref_morton3d(uint32_t x, uint32_t y, uint32_t z) {
    return MortonCode::Compose3D<uint64_t>(Vector3ui(x, y, z));
}

// Morton codes of AABB centroids.  The reference kernel (KCGenMortonCodes,
// LinearBVH.hpp:118-166) stages the extent with threads 0..6 copying 4-byte
// words of a 24-byte AABB (one word past its end), which cannot run on the
// host; its per-element body is evaluated here with the reference's own
// AABB3f::Centroid and MortonCode::Compose3D.
void ref_morton_codes(const float* aabbs, uint32_t n, const float* extent, float delta,
                      uint64_t* codes) {
    AABB3f ext(V(extent), V(extent + 3));
    for (uint32_t i = 0; i < n; i++) {
        AABB3f a(V(aabbs + 6 * i), V(aabbs + 6 * i + 3));
        Vector3f rel = a.Centroid() - ext.Min();
        uint32_t x = static_cast<uint32_t>(floor(rel[0] / delta));
        uint32_t y = static_cast<uint32_t>(floor(rel[1] / delta));
        uint32_t z = static_cast<uint32_t>(floor(rel[2] / delta));
        codes[i] = MortonCode::Compose3D<uint64_t>(Vector3ui(x, y, z));
    }
}

// KCConstructLBVHLeaf / KCConstructLBVHInter and BottomUpAABBLeaf/Inter, with
// the host driving the iteration the reference's CDP parent kernel runs.
int ref_lbvh(const uint64_t* codes, const uint32_t* sorted_idx, const float* leaf_aabbs,
             uint32_t n, uint32_t* left, uint32_t* right, uint32_t* parent, float* inner,
             uint32_t* root) {
    if (n < 2) return 2;
    std::vector<LBVHNode<uint32_t>> nodes(2 * n - 1);
    std::memset(nodes.data(), 0, sizeof(LBVHNode<uint32_t>) * nodes.size());
    std::vector<Vector2ui> ranges(n - 1);
    std::memset(ranges.data(), 0xFF, sizeof(Vector2ui) * (n - 1));
    std::vector<uint32_t> flags(n - 1, 0), leafData(n);
    for (uint32_t i = 0; i < n; i++) leafData[i] = sorted_idx[i];
    uint32_t counter = 0, rootIdx = 0;
    launch(n, [&]() {
        KCConstructLBVHLeaf<uint32_t>(rootIdx, nodes.data(), ranges.data(), leafData.data(),
                                      sorted_idx, codes, n);
    });
    int guard = 0;
    while (counter < (n - 1) && guard++ < 100000) {
        launch(n, [&]() {
            KCConstructLBVHInter<uint32_t>(counter, flags.data(), rootIdx, nodes.data(),
                                           ranges.data(), codes, n);
        });
    }
    std::vector<AABB3f> la(n);
    for (uint32_t i = 0; i < n; i++) la[i] = AABB3f(V(leaf_aabbs + 6 * i), V(leaf_aabbs + 6 * i + 3));
    std::memset(ranges.data(), 0xFF, sizeof(Vector2ui) * (n - 1));
    std::fill(flags.begin(), flags.end(), 0u);
    counter = 0;
    launch(n, [&]() { BottomUpAABBLeaf<uint32_t>(nodes.data(), ranges.data(), n); });
    guard = 0;
    while (counter < (n - 1) && guard++ < 100000) {
        launch(n, [&]() {
            BottomUpAABBInter<uint32_t>(counter, flags.data(), ranges.data(), nodes.data(),
                                        la.data(), sorted_idx, n);
        });
    }
    for (uint32_t j = 0; j < n - 1; j++) {
        left[j] = nodes[n + j].body.left;
        right[j] = nodes[n + j].body.right;
        W(inner + 6 * j, nodes[n + j].body.aabbMin);
        W(inner + 6 * j + 3, nodes[n + j].body.aabbMax);
    }
    for (uint32_t i = 0; i < 2 * n - 1; i++) parent[i] = nodes[i].parent;
    parent[rootIdx] = 0xFFFFFFFFu;
    *root = rootIdx;
    return 0;
}

int ref_intersect_tri(const float* ro, const float* rd, const float* p0, const float* p1,
                      const float* p2, int cull, float* t, float* bary3) {
    RayF r(V(rd), V(ro));
    Vector3f b;
    float tt;
    bool h = r.IntersectsTriangle(b, tt, V(p0), V(p1), V(p2), cull != 0);
    if (h) {
        *t = tt;
        W(bary3, b);
    }
    return h ? 1 : 0;
}
int ref_intersect_aabb(const float* ro, const float* rd, const float* mn, const float* mx,
                       float tmin, float tmax, float* tout) {
    RayF r(V(rd), V(ro));
    Vector2f to;
    bool h = r.IntersectsAABB(to, V(mn), V(mx), Vector2f(tmin, tmax));
    tout[0] = to[0];
    tout[1] = to[1];
    return h ? 1 : 0;
}
void ref_nudge(const float* pos, const float* dir, float* out) {
    RayF r(Vector3f(0, 0, 1), V(pos));
    W(out, r.Nudge(V(dir)).getPosition());
}
void ref_reflect(const float* d, const float* n, float* out) {
    RayF r(V(d), Vector3f(0.0f));
    W(out, r.Reflect(V(n)).getDirection());
}
int ref_refract(const float* d, const float* n, float from, float to, float* out) {
    RayF r(V(d), Vector3f(0.0f)), o;
    bool ok = r.Refract(o, V(n), from, to);
    W(out, o.getDirection());
    return ok ? 1 : 0;
}
void ref_hemi_cosine(const float* xi, float* dir, float* pdf) {
    W(dir, HemiDistribution::HemiCosineCDF(Vector2f(xi[0], xi[1]), *pdf));
}
void ref_bary_slerp(const float* q0, const float* q1, const float* q2, float a, float b,
                    float* out) {
    WQ(out, Quat::BarySLerp(Q(q0), Q(q1), Q(q2), a, b));
}
void ref_quat_rotate(const float* q, const float* v, float* out) { W(out, Q(q).ApplyRotation(V(v))); }
void ref_quat_mul(const float* a, const float* b, float* out) { WQ(out, Q(a) * Q(b)); }
void ref_space(const float* x, const float* y, const float* z, float* out) {
    QuatF q;
    TransformGen::Space(q, V(x), V(y), V(z));
    WQ(out, q);
}
void ref_calc_tangent(const float* p0, const float* p1, const float* p2, const float* uv0,
                      const float* uv1, const float* uv2, const float* n, float* out) {
    W(out, Triangle::CalculateTangent(V(p0), V(p1), V(p2), Vector2f(uv0[0], uv0[1]),
                                      Vector2f(uv1[0], uv1[1]), Vector2f(uv2[0], uv2[1]), V(n)));
}
void ref_orthogonal(const float* v, float* out) { W(out, OrthogonalVector(V(v))); }
float ref_dggx(float ndh, float alpha) { return TracerFunctions::DGGX(ndh, alpha); }
float ref_gsmith_corr(const float* wo, const float* wi, float alpha) {
    return TracerFunctions::GSmithCorralated(V(wo), V(wi), alpha);
}
float ref_gsmith_single(const float* v, float alpha) { return TracerFunctions::GSmithSingle(V(v), alpha); }
void ref_fresnel_conductor(float c, const float* eta, const float* k, float* out) {
    W(out, TracerFunctions::FresnelConductor(c, V(eta), V(k)));
}
float ref_fresnel_dielectric(float c, float a, float b) { return TracerFunctions::FresnelDielectric(c, a, b); }
void ref_vndf_sample(const float* v, float alpha, const float* xi, float* h, float* pdf) {
    FixedRng rng;
    rng.v[0] = xi[0];
    rng.v[1] = xi[1];
    W(h, TracerFunctions::VNDFGGXSmithSample(*pdf, V(v), alpha, rng));
}
float ref_vndf_pdf(const float* v, const float* h, float alpha) {
    return TracerFunctions::VNDFGGXSmithPDF(V(v), V(h), alpha);
}
float ref_power_heuristic(float n0, float p0, float n1, float p1) {
    return TracerFunctions::PowerHeuristic(n0, p0, n1, p1);
}

}  // extern "C"
