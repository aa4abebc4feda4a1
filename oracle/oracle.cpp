// CPU oracle for the meturay_b200 wavefront path-tracing path.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline / reference leg as the checker; never linked into
// or called by the product.
//
// Restates MRay (yalcinerbora/meturay) Source/TracerCUDA + Source/RayLib.
// Every function names the reference file:line it follows.  Build flags:
// -O2 -ffp-contract=off (no implicit FMA), so FP32 results follow the same
// operation order as the CUDA kernels built with -fmad=false.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <thread>
#include <vector>
#include <map>
#include <type_traits>

namespace {

// ------------------------------------------------------------------------
// Portable math.  sin/cos: Cody-Waite reduction by pi/2 split in three
// parts, then Taylor polynomials on [-pi/4, pi/4] (coefficients are the
// float-rounded 1/n! values).  acos: asin Taylor series on [0, 1/2] with the
// half-angle identity above 1/2.  The device copy uses the same steps.
// ------------------------------------------------------------------------
constexpr float kTwoOverPi = 0x1.45f306p-1f;
constexpr float kPio2Hi = 0x1.92p+0f;
constexpr float kPio2Mid = 0x1.fb4p-12f;
constexpr float kPio2Lo = 0x1.4442d2p-24f;
constexpr float kPiF = 0x1.921fb6p+1f;      // float(pi)  (Constants.h:99)
constexpr float kPio2F = 0x1.921fb6p+0f;
constexpr float kInvPiF = 0x1.45f306p-2f;   // float(1/pi) (Constants.h:101)

inline float sin_poly(float r) {
    float r2 = r * r;
    float p = -0x1.ae6456p-26f;
    p = p * r2 + 0x1.71de3ap-19f;
    p = p * r2 + -0x1.a01a02p-13f;
    p = p * r2 + 0x1.111112p-7f;
    p = p * r2 + -0x1.555556p-3f;
    return r + (r * r2) * p;
}
inline float cos_poly(float r) {
    float r2 = r * r;
    float p = 0x1.1eed8ep-29f;
    p = p * r2 + -0x1.27e4fcp-22f;
    p = p * r2 + 0x1.a01a02p-16f;
    p = p * r2 + -0x1.6c16c2p-10f;
    p = p * r2 + 0x1.555556p-5f;
    p = p * r2 + -0.5f;
    return 1.0f + r2 * p;
}
inline void pm_sincos(float x, float& s, float& c) {
    float kf = std::rint(x * kTwoOverPi);
    int k = static_cast<int>(kf);
    float r = x - kf * kPio2Hi;
    r = r - kf * kPio2Mid;
    r = r - kf * kPio2Lo;
    float sr = sin_poly(r), cr = cos_poly(r);
    switch (k & 3) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
}
inline float asin_poly(float z) {  // z in [0, 0.5]
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
inline float pm_acos(float x) {
    float ax = std::fabs(x);
    if (ax <= 0.5f) {
        float a = asin_poly(ax);
        a = (x < 0.0f) ? -a : a;
        return kPio2F - a;
    }
    float z = std::sqrt((1.0f - ax) * 0.5f);
    float a = 2.0f * asin_poly(z);
    return (x > 0.0f) ? a : (kPiF - a);
}

inline float pm_asin01(float z) {
    if (z <= 0.5f) return asin_poly(z);
    return kPio2F - 2.0f * asin_poly(std::sqrt((1.0f - z) * 0.5f));
}
inline float pm_atan2(float y, float x) {
    const float ax = std::fabs(x), ay = std::fabs(y);
    const float mx = std::fmax(ax, ay), mn = std::fmin(ax, ay);
    if (mx == 0.0f) return 0.0f;
    const float a = mn / mx;
    float r = pm_asin01(a / std::sqrt(1.0f + a * a));
    if (ay > ax) r = kPio2F - r;
    if (x < 0.0f) r = kPiF - r;
    return (y < 0.0f) ? -r : r;
}

// Math traits: FP32 uses the portable functions, FP64 the C library.
template <class T> struct M;
template <> struct M<float> {
    static float sqrt(float x) { return std::sqrt(x); }
    static void sincos(float x, float& s, float& c) { pm_sincos(x, s, c); }
    static float sin(float x) { float s, c; pm_sincos(x, s, c); return s; }
    static float acos(float x) { return pm_acos(x); }
    static constexpr float Pi = kPiF;
    static constexpr float InvPi = kInvPiF;
    static constexpr float SmallEps = 1.0e-7f;
    static constexpr float Eps = 1.0e-5f;
    static constexpr float LargeEps = 1.0e-4f;
    static constexpr float Max = 3.40282347e+38f;
};
template <> struct M<double> {
    static double sqrt(double x) { return std::sqrt(x); }
    static void sincos(double x, double& s, double& c) { s = std::sin(x); c = std::cos(x); }
    static double sin(double x) { return std::sin(x); }
    static double acos(double x) { return std::acos(x); }
    static constexpr double Pi = 3.1415926535897932384626433;
    static constexpr double InvPi = 1.0 / 3.1415926535897932384626433;
    static constexpr double SmallEps = 1.0e-7;
    static constexpr double Eps = 1.0e-5;
    static constexpr double LargeEps = 1.0e-4;
    static constexpr double Max = 3.40282347e+38;
};

// ------------------------------------------------------------------------
// Vectors and quaternions (RayLib/Vector.hpp, RayLib/Quaternion.hpp).
// ------------------------------------------------------------------------
template <class T> struct V3 {
    T x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline bool operator!=(V3<T> a, V3<T> b) { return a.x != b.x || a.y != b.y || a.z != b.z; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {  // Vector.hpp:867-873
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline V3<T> normalize(V3<T> v) {  // Vector.hpp:519-530
    T inv = T(1) / M<T>::sqrt(dot(v, v));
    return {v.x * inv, v.y * inv, v.z * inv};
}
template <class T> inline V3<T> vmax(V3<T> v, T s) { return {std::fmax(v.x, s), std::fmax(v.y, s), std::fmax(v.z, s)}; }
template <class T> inline V3<T> vsqrt(V3<T> v) { return {M<T>::sqrt(v.x), M<T>::sqrt(v.y), M<T>::sqrt(v.z)}; }

template <class T> struct Q4 { T w, x, y, z; };
template <class T> inline Q4<T> qmul(Q4<T> a, Q4<T> b) {  // Quaternion.hpp:76-89
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
            a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
template <class T> inline Q4<T> qconj(Q4<T> q) { return {q.w, -q.x, -q.y, -q.z}; }
template <class T> inline T qdot(Q4<T> a, Q4<T> b) { return a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline Q4<T> qnormalize(Q4<T> q) {
    T inv = T(1) / M<T>::sqrt(qdot(q, q));
    return {q.w * inv, q.x * inv, q.y * inv, q.z * inv};
}
template <class T> inline V3<T> qrotate(Q4<T> q, V3<T> v) {  // Quaternion.hpp:229-238
    Q4<T> qi = qconj(q);
    Q4<T> vq = {T(0), v.x, v.y, v.z};
    Q4<T> r = qmul(q, qmul(vq, qi));
    return {r.x, r.y, r.z};
}
template <class T> inline V3<T> to_space(V3<T> v, Q4<T> q) { return qrotate(qconj(q), v); }  // GPUSurface.h:45
template <class T> inline V3<T> to_tangent(V3<T> v, Q4<T> q) { return qrotate(q, v); }      // GPUSurface.h:38

template <class T> inline Q4<T> slerp(Q4<T> s, Q4<T> e, T t) {  // Quaternion.hpp:258-283
    T cosT = qdot(s, e);
    T cosF = (cosT >= 0) ? cosT : (-cosT);
    T s0, s1;
    if (cosF < (T(1) - M<T>::Eps)) {
        T angle = M<T>::acos(cosF);
        T sa = M<T>::sin(angle);
        s0 = M<T>::sin(angle * (T(1) - t)) / sa;
        s1 = M<T>::sin(angle * t) / sa;
    } else {
        s0 = (T(1) - t);
        s1 = t;
    }
    s1 = (cosT >= 0) ? s1 : (-s1);
    return {s.w * s0 + e.w * s1, s.x * s0 + e.x * s1, s.y * s0 + e.y * s1, s.z * s0 + e.z * s1};
}
template <class T> inline Q4<T> bary_slerp(Q4<T> q0, Q4<T> q1, Q4<T> q2, T a, T b) {  // Quaternion.hpp:285-318
    T c = (T(1) - a - b);
    if (std::fabs(a + b) < M<T>::Eps) return q2;
    T ab = a / (a + b);
    Q4<T> qAB = slerp(q1, q0, ab);
    return slerp(qAB, q2, c);
}

// Ray::Nudge (RayLib/Ray.hpp:503-556), RTG-I chapter 6.
inline V3<float> nudge(V3<float> p, V3<float> dir) {
    const float ORIGIN = 1.0f / 32.0f, FLOAT_SCALE = 1.0f / 65536.0f, INT_SCALE = 256.0f;
    float pc[3] = {p.x, p.y, p.z}, dc[3] = {dir.x, dir.y, dir.z}, out[3];
    for (int i = 0; i < 3; i++) {
        int32_t ofi = static_cast<int32_t>(INT_SCALE * dc[i]);
        int32_t pi;
        std::memcpy(&pi, &pc[i], 4);
        pi += (pc[i] < 0) ? -ofi : ofi;
        float pI;
        std::memcpy(&pI, &pi, 4);
        out[i] = (std::fabs(pc[i]) < ORIGIN) ? (pc[i] + FLOAT_SCALE * dc[i]) : pI;
    }
    return {out[0], out[1], out[2]};
}
inline V3<double> nudge(V3<double> p, V3<double> dir) {
    const double ORIGIN = 1.0 / 32.0, FLOAT_SCALE = 1.0 / 65536.0, INT_SCALE = 256.0;
    double pc[3] = {p.x, p.y, p.z}, dc[3] = {dir.x, dir.y, dir.z}, out[3];
    for (int i = 0; i < 3; i++) {
        int64_t ofi = static_cast<int64_t>(INT_SCALE * dc[i]);
        int64_t pi;
        std::memcpy(&pi, &pc[i], 8);
        pi += (pc[i] < 0) ? -ofi : ofi;
        double pI;
        std::memcpy(&pI, &pi, 8);
        out[i] = (std::fabs(pc[i]) < ORIGIN) ? (pc[i] + FLOAT_SCALE * dc[i]) : pI;
    }
    return {out[0], out[1], out[2]};
}

// ------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
// easy as 1, 2, 3", SC'11).  Counter = {sample, frame, tag, block}.
// ------------------------------------------------------------------------
inline void philox(const uint32_t c_in[4], const uint32_t k_in[2], uint32_t out[4]) {
    uint32_t c0 = c_in[0], c1 = c_in[1], c2 = c_in[2], c3 = c_in[3];
    uint32_t k0 = k_in[0], k1 = k_in[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = uint64_t(0xD2511F53u) * c0;
        uint64_t p1 = uint64_t(0xCD9E8D57u) * c2;
        uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
        uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}
constexpr uint32_t kTagCamera = 0x10000u;
struct Rng4 {
    float u[4];
};
inline Rng4 rng_block(uint32_t sample, uint32_t frame, uint32_t tag, uint32_t block,
                      uint32_t seed_lo, uint32_t seed_hi) {
    uint32_t c[4] = {sample, frame, tag, block}, k[2] = {seed_lo, seed_hi}, o[4];
    philox(c, k, o);
    Rng4 r;
    for (int i = 0; i < 4; i++) r.u[i] = static_cast<float>(o[i] >> 8) * 0x1p-24f;
    return r;
}

// ------------------------------------------------------------------------
// Morton codes (RayLib/MortonCode.h:45-56,150-158; LinearBVH.hpp:118-166,
// 398-414).
// ------------------------------------------------------------------------
inline uint64_t expand3d(uint32_t val) {
    uint64_t x = val;
    x &= 0x1fffff;
    x = (x | x << 32) & 0x001f00000000ffffull;
    x = (x | x << 16) & 0x001f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}
inline uint64_t morton3d(uint32_t x, uint32_t y, uint32_t z) {
    return (expand3d(x) << 0) | (expand3d(y) << 1) | (expand3d(z) << 2);
}
inline float morton_delta(const float ext[6]) {  // LinearBVH.hpp:398-414
    const double res = 1.0f / static_cast<double>(1 << 21);
    double dx = static_cast<double>(ext[3] - ext[0]) * res;
    double dy = static_cast<double>(ext[4] - ext[1]) * res;
    double dz = static_cast<double>(ext[5] - ext[2]) * res;
    return static_cast<float>(std::max({dx, dy, dz}));
}

template <class K>
void radix_sort(K* keys, uint32_t* vals, uint32_t n, int begin, int end, bool desc) {
    std::vector<K> k2(n);
    std::vector<uint32_t> v2(n);
    K* ka = keys; K* kb = k2.data();
    uint32_t* va = vals; uint32_t* vb = v2.data();
    int passes = 0;
    for (int bit = begin; bit < end; bit += 8) {
        int nb = std::min(8, end - bit);
        uint32_t mask = (1u << nb) - 1u;
        uint32_t cnt[257] = {0};
        for (uint32_t i = 0; i < n; i++) {
            uint32_t d = uint32_t(ka[i] >> bit) & mask;
            if (desc) d = mask - d;
            cnt[d + 1]++;
        }
        for (int d = 0; d < 256; d++) cnt[d + 1] += cnt[d];
        for (uint32_t i = 0; i < n; i++) {
            uint32_t d = uint32_t(ka[i] >> bit) & mask;
            if (desc) d = mask - d;
            uint32_t p = cnt[d]++;
            kb[p] = ka[i];
            vb[p] = va[i];
        }
        std::swap(ka, kb);
        std::swap(va, vb);
        passes++;
    }
    if (passes & 1) {
        std::memcpy(keys, ka, sizeof(K) * n);
        std::memcpy(vals, va, sizeof(uint32_t) * n);
    }
}

// Delta between adjacent sorted codes (LinearBVH.hpp:30-39), extended with
// the index-augmented tie break for equal codes (Karras 2012, sec. 4): the
// reference rejects duplicate codes, this keeps unique-code trees identical.
inline uint32_t lbvh_delta(const uint64_t* c, uint32_t i) {
    uint64_t d = c[i] ^ c[i + 1];
    if (d != 0) return uint32_t(__builtin_clzll(d));
    uint32_t di = i ^ (i + 1);
    return 64u + uint32_t(__builtin_clz(di));
}

// ------------------------------------------------------------------------
// Scene access helpers
// ------------------------------------------------------------------------
constexpr uint32_t kBatchNull = 0, kBatchLambert = 1, kBatchMetal = 2, kBatchRefract = 3,
                   kBatchLight = 4, kBatchLambertC = 5, kBatchUnreal = 6;
constexpr uint32_t kInvalid = 0xFFFFFFFFu;

template <class T> inline V3<T> vpos(const oracle_scene* s, uint32_t v) {
    return {T(s->pos[3 * v + 0]), T(s->pos[3 * v + 1]), T(s->pos[3 * v + 2])};
}
template <class T> inline Q4<T> vtbn(const oracle_scene* s, uint32_t v) {
    const float* q = s->tbn + 4 * v;
    return {T(q[0]), T(q[1]), T(q[2]), T(q[3])};
}

// ------------------------------------------------------------------------
// Ray/triangle (RayLib/Ray.hpp:143-184) and ray/box tests.
// ------------------------------------------------------------------------
template <class T>
inline bool intersect_tri(V3<T> o, V3<T> d, V3<T> t0, V3<T> e0, V3<T> e1, bool cull,
                          T& t, T& b0, T& b1, T* vout = nullptr) {
    V3<T> p = cross(d, e1);
    T det = dot(e0, p);
    if ((cull && (det < M<T>::SmallEps)) || (std::fabs(det) < M<T>::SmallEps)) return false;
    T invDet = T(1) / det;
    V3<T> tv = o - t0;
    T u = dot(tv, p) * invDet;
    if (u < 0 || u > 1) return false;
    V3<T> q = cross(tv, e0);
    T v = dot(d, q) * invDet;
    if ((v < 0) || (v + u) > 1) return false;
    t = dot(e1, q) * invDet;
    if (t <= M<T>::SmallEps) return false;
    // bary reordered to (c, a, b): hit struct keeps (1-u-v, u)
    b0 = T(1) - u - v;
    b1 = u;
    if (vout) *vout = v;
    return true;
}

// Slab test with precomputed o*invD; fmaf keeps FP32 bit-identical to the
// device kernel.  Returns entry distance via tn.
inline bool box_hit(const float lo[3], const float hi[3], const float inv[3],
                    const float ooi[3], float tmin, float tmax, float& tn) {
    float tl[3], th[3];
    for (int i = 0; i < 3; i++) {
        float a = std::fmaf(lo[i], inv[i], -ooi[i]);
        float b = std::fmaf(hi[i], inv[i], -ooi[i]);
        tl[i] = std::fmin(a, b);
        th[i] = std::fmax(a, b);
    }
    tn = std::fmax(std::fmax(tl[0], tl[1]), std::fmax(tl[2], tmin));
    float tf = std::fmin(std::fmin(th[0], th[1]), std::fmin(th[2], tmax));
    return tn <= tf;
}
inline bool box_hit(const float lo[3], const float hi[3], const double inv[3],
                    const double ooi[3], double tmin, double tmax, double& tn) {
    double tl[3], th[3];
    for (int i = 0; i < 3; i++) {
        double a = std::fma(double(lo[i]), inv[i], -ooi[i]);
        double b = std::fma(double(hi[i]), inv[i], -ooi[i]);
        tl[i] = std::fmin(a, b);
        th[i] = std::fmax(a, b);
    }
    tn = std::fmax(std::fmax(tl[0], tl[1]), std::fmax(tl[2], tmin));
    double tf = std::fmin(std::fmin(th[0], th[1]), std::fmin(th[2], tmax));
    return tn <= tf;
}
inline float safe_dir(float d) { return (std::fabs(d) > 1e-20f) ? d : std::copysign(1e-20f, d); }
inline double safe_dir(double d) { return (std::fabs(d) > 1e-20) ? d : std::copysign(1e-20, d); }

}  // namespace

// ------------------------------------------------------------------------
// LBVH container
// ------------------------------------------------------------------------
struct oracle_bvh {
    uint32_t n = 0;
    uint32_t root = 0;
    std::vector<uint64_t> codes;
    std::vector<uint32_t> sorted_idx;
    std::vector<float> leaf_aabbs;   // by original triangle index
    std::vector<uint32_t> left, right, parent;
    std::vector<float> inner;        // (n-1)*6
    std::vector<float> e0, e1, v0;   // per original triangle (precomputed edges)
};

namespace {

template <class T> struct Hit {
    uint32_t key = 0;
    uint32_t prim = kInvalid;
    T t = 0;
    T b0 = 0, b1 = 0;
};

template <class T>
inline void tri_test(const oracle_scene* s, const oracle_bvh* b, uint32_t tri, V3<T> o, V3<T> d,
                     T tmin, T& tmax, Hit<T>& h) {
    V3<T> p0 = {T(b->v0[3 * tri]), T(b->v0[3 * tri + 1]), T(b->v0[3 * tri + 2])};
    V3<T> e0 = {T(b->e0[3 * tri]), T(b->e0[3 * tri + 1]), T(b->e0[3 * tri + 2])};
    V3<T> e1 = {T(b->e1[3 * tri]), T(b->e1[3 * tri + 1]), T(b->e1[3 * tri + 2])};
    bool cull = s->tri_cull ? (s->tri_cull[tri] != 0) : false;
    T t, b0, b1;
    if (intersect_tri(o, d, p0, e0, e1, cull, t, b0, b1)) {
        // AcceptHit (GPUAcceleratorCommonKC.cuh:35-78): t in [tMin, tMax)
        if (t >= tmin && t < tmax) {
            tmax = t;
            h.t = t;
            h.b0 = b0;
            h.b1 = b1;
            h.prim = tri;
            h.key = s->tri_key[tri];
        }
    }
}

// Closest hit over the LBVH: both child boxes are tested at each inner node
// and the nearer one is entered first (ties go to the left child); the
// farther one is pushed.  The device kernel walks the same tree the same way.
// Traversal work counters (inner nodes entered, triangles tested), summed
// over all threads; read with oracle_trace_counters.
std::atomic<uint64_t> g_nodes{0}, g_tris{0};

template <class T>
Hit<T> trace_one(const oracle_scene* s, const oracle_bvh* b, V3<T> o, V3<T> d, T tmin, T tmax) {
    Hit<T> h;
    uint64_t nodes = 0, tris = 0;
    struct Flush {
        uint64_t& n; uint64_t& t;
        ~Flush() { g_nodes.fetch_add(n, std::memory_order_relaxed); g_tris.fetch_add(t, std::memory_order_relaxed); }
    } flush{nodes, tris};
    const uint32_t n = b->n;
    if (n == 0) return h;
    if (n == 1) {
        tri_test(s, b, b->sorted_idx[0], o, d, tmin, tmax, h);
        return h;
    }
    T inv[3] = {T(1) / safe_dir(d.x), T(1) / safe_dir(d.y), T(1) / safe_dir(d.z)};
    T ooi[3] = {o.x * inv[0], o.y * inv[1], o.z * inv[2]};
    uint32_t stack[128];
    int sp = 0;
    uint32_t node = b->root;  // global node index (>= n: inner)
    for (;;) {
        if (node >= n) {
            nodes++;
            uint32_t j = node - n;
            uint32_t c[2] = {b->left[j], b->right[j]};
            bool hit[2];
            T tn[2];
            for (int k = 0; k < 2; k++) {
                const float* box = (c[k] < n) ? &b->leaf_aabbs[6 * b->sorted_idx[c[k]]]
                                              : &b->inner[6 * (c[k] - n)];
                hit[k] = box_hit(box, box + 3, inv, ooi, tmin, tmax, tn[k]);
            }
            if (hit[0] && hit[1]) {
                bool swap = tn[1] < tn[0];
                stack[sp++] = swap ? c[0] : c[1];
                node = swap ? c[1] : c[0];
                continue;
            } else if (hit[0]) {
                node = c[0];
                continue;
            } else if (hit[1]) {
                node = c[1];
                continue;
            }
        } else {
            tris++;
            tri_test(s, b, b->sorted_idx[node], o, d, tmin, tmax, h);
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return h;
}

template <class T>
Hit<T> trace_linear_one(const oracle_scene* s, const oracle_bvh* b, V3<T> o, V3<T> d, T tmin,
                        T tmax) {
    Hit<T> h;
    for (uint32_t i = 0; i < s->tri_count; i++) tri_test(s, b, i, o, d, tmin, tmax, h);
    return h;
}

template <class F>
void parallel_for(uint32_t n, uint32_t threads, F f) {
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    threads = std::min<uint32_t>(threads, std::max(1u, n));
    if (threads <= 1) {
        f(0u, n);
        return;
    }
    std::vector<std::thread> th;
    std::atomic<uint32_t> next{0};
    const uint32_t chunk = 256;
    for (uint32_t t = 0; t < threads; t++) {
        th.emplace_back([&]() {
            for (;;) {
                uint32_t b = next.fetch_add(chunk);
                if (b >= n) break;
                f(b, std::min(n, b + chunk));
            }
        });
    }
    for (auto& t : th) t.join();
}

// ------------------------------------------------------------------------
// Path tracer (PathTracerKC.cuh:335-649, material KC files,
// GPULightSamplerUniform.cuh:95-135, GPULightPrimitive.cuh:139-170,
// GPUPrimitiveTriangle.h:65-115,624-700, GenerationKernels.cuh:26-108,
// GPUCameraPinhole.cuh:209-243).
// ------------------------------------------------------------------------
enum RayType : uint8_t { NEE_RAY = 0, SPECULAR_PATH_RAY = 1, PATH_RAY = 2, CAMERA_RAY = 3 };

template <class T> struct Aux {
    V3<T> rf;
    uint32_t sample;
    uint32_t endpoint;
    uint32_t medium;
    uint32_t depth;
    RayType type;
    T prevPDF;
};
template <class T> struct PRay {
    V3<T> o, d;
    T tmin, tmax;
    Aux<T> aux;
};
template <class T> struct Surface {
    V3<T> pos;
    Q4<T> w2t;
    V3<T> geo;
    bool back;
};

template <class T>
Surface<T> gen_surface(const oracle_scene* s, uint32_t prim, T ha, T hb, V3<T> rayDir) {
    bool twoSided = s->tri_cull ? (s->tri_cull[prim] == 0) : true;
    T a = ha, b = hb;
    T c = T(1) - a - b;
    uint32_t i0 = s->idx[3 * prim], i1 = s->idx[3 * prim + 1], i2 = s->idx[3 * prim + 2];
    Q4<T> tbn = bary_slerp(vtbn<T>(s, i0), vtbn<T>(s, i1), vtbn<T>(s, i2), a, b);
    tbn = qnormalize(tbn);
    V3<T> p0 = vpos<T>(s, i0), p1 = vpos<T>(s, i1), p2 = vpos<T>(s, i2);
    Surface<T> sf;
    sf.pos = (p0 * a + p1 * b) + p2 * c;
    V3<T> g = normalize(cross(p1 - p0, p2 - p0));
    g = normalize(g);
    sf.w2t = tbn;
    sf.back = twoSided && (dot(g, rayDir) > T(0));
    if (sf.back) {
        g = -g;
        sf.w2t = qmul(Q4<T>{T(0), T(1), T(0), T(0)}, sf.w2t);
    }
    sf.geo = g;
    return sf;
}

template <class T> struct Ctx {
    const oracle_scene* s;
    const oracle_bvh* b;
    const oracle_options* o;
    T* out;  // sample radiance
};

template <class T> inline void accumulate(Ctx<T>& c, uint32_t sample, V3<T> v) {
    c.out[3 * sample + 0] += v.x;
    c.out[3 * sample + 1] += v.y;
    c.out[3 * sample + 2] += v.z;
}

// BxDF sample result
template <class T> struct BSample {
    V3<T> dir, pos;
    V3<T> refl;
    T pdf;
    uint32_t medium;
};

template <class T>
inline V3<T> hemi_cosine(T xi0, T xi1, T& pdf) {  // HemiDistribution.h:10-30
    T coeff = T(2) * M<T>::Pi * xi1;
    T sn, cs;
    M<T>::sincos(coeff, sn, cs);
    V3<T> d;
    d.x = M<T>::sqrt(xi0) * cs;
    d.y = M<T>::sqrt(xi0) * sn;
    d.z = M<T>::sqrt(std::fmax(T(0), (T(1) - d.x * d.x - d.y * d.y)));
    pdf = d.z * M<T>::InvPi;
    return d;
}

// TracerFunctions.cuh:8-30
template <class T> inline T fresnel_dielectric(T cosIn, T iorIn, T iorOut) {
    T sinIn = M<T>::sqrt(std::fmax(T(0), T(1) - cosIn * cosIn));
    T sinOut = iorIn / iorOut * sinIn;
    if (sinOut >= T(1)) return T(1);
    T cosOut = M<T>::sqrt(std::fmax(T(0), T(1) - sinOut * sinOut));
    T par = ((iorOut * cosIn - iorIn * cosOut) / (iorOut * cosIn + iorIn * cosOut));
    par = par * par;
    T perp = ((iorIn * cosIn - iorOut * cosOut) / (iorIn * cosIn + iorOut * cosOut));
    perp = perp * perp;
    return (par + perp) * T(0.5);
}
// TracerFunctions.cuh:33-75 (per component)
template <class T> inline V3<T> fresnel_conductor(T cosIn, V3<T> eta, V3<T> k) {
    T cosInSqr = cosIn * cosIn;
    T sinInSqr = std::fmax(T(0), T(1) - cosInSqr);
    T sinInSqr2 = sinInSqr * sinInSqr;
    T sinInSqr4 = sinInSqr2 * sinInSqr2;
    V3<T> etaSqr = eta * eta;
    V3<T> kSqr = k * k;
    V3<T> diff = etaSqr - kSqr - V3<T>(sinInSqr, sinInSqr, sinInSqr);
    V3<T> a2b2 = diff * diff;
    a2b2 = a2b2 + T(4) * etaSqr * kSqr;
    a2b2 = vsqrt(vmax(a2b2, T(0)));
    V3<T> a = T(0.5) * (a2b2 + diff);
    a = vsqrt(vmax(a, T(0)));
    V3<T> perpT1 = a2b2 + V3<T>(cosInSqr, cosInSqr, cosInSqr);
    V3<T> perpT2 = a * (T(2) * cosIn);
    V3<T> perp = V3<T>((perpT1.x - perpT2.x) / (perpT1.x + perpT2.x),
                       (perpT1.y - perpT2.y) / (perpT1.y + perpT2.y),
                       (perpT1.z - perpT2.z) / (perpT1.z + perpT2.z));
    V3<T> parT1 = a2b2 * cosInSqr + V3<T>(sinInSqr4, sinInSqr4, sinInSqr4);
    V3<T> parT2 = perpT2 * sinInSqr2;
    V3<T> num = perp * (parT1 - parT2);
    V3<T> den = parT1 + parT2;
    V3<T> par = V3<T>(num.x / den.x, num.y / den.y, num.z / den.z);
    return (par + perp) * T(0.5);
}
template <class T> inline T dggx(T NdH, T alpha) {  // TracerFunctions.cuh:77-86
    T a2 = alpha * alpha;
    T den = NdH * NdH * (a2 - T(1)) + T(1);
    den = den * den;
    den *= M<T>::Pi;
    return a2 / den;
}
template <class T> inline T lambda_smith(V3<T> v, T alpha) {  // :88-97
    V3<T> s = v * v;
    T a2 = alpha * alpha;
    T inner = a2 * (s.x + s.y) / s.z;
    T l = M<T>::sqrt(T(1) + inner) - T(1);
    return l * T(0.5);
}
template <class T> inline T g_smith_single(V3<T> v, T alpha) { return T(1) / (T(1) + lambda_smith(v, alpha)); }
template <class T> inline T g_smith_corr(V3<T> o, V3<T> i, T alpha) {
    return T(1) / (lambda_smith(o, alpha) + lambda_smith(i, alpha) + T(1));
}
template <class T> inline T vndf_pdf(V3<T> V, V3<T> H, T alpha) {  // :181-190
    T VdH = std::fmax(T(0), dot(H, V));
    T NdH = std::fmax(T(0), H.z);
    T NdV = std::fmax(T(0), V.z);
    T D = dggx(NdH, alpha);
    T G = g_smith_single(V, alpha);
    return (NdV == T(0)) ? T(0) : (VdH * D * G / NdV);
}
template <class T> inline V3<T> vndf_sample(T& pdf, V3<T> V, T alpha, T xi0, T xi1) {  // :192-251
    T a = alpha;
    V3<T> VH = normalize(V3<T>(a * V.x, a * V.y, V.z));
    T lensq = VH.x * VH.x + VH.y * VH.y;
    V3<T> T1 = (lensq > 0) ? V3<T>(-VH.y, VH.x, T(0)) / M<T>::sqrt(lensq) : V3<T>(1, 0, 0);
    V3<T> T2 = cross(VH, T1);
    T r = M<T>::sqrt(xi0);
    T phi = T(2) * M<T>::Pi * xi1;
    T sn, cs;
    M<T>::sincos(phi, sn, cs);
    T t1 = r * cs;
    T t2 = r * sn;
    T s = T(0.5) * (T(1) + VH.z);
    t2 = (T(1) - s) * M<T>::sqrt(T(1) - t1 * t1) + s * t2;
    T val = T(1) - t1 * t1 - t2 * t2;
    V3<T> NH = t1 * T1 + t2 * T2 + M<T>::sqrt(std::fmax(T(0), val)) * VH;
    V3<T> NM = V3<T>(a * NH.x, a * NH.y, std::fmax(T(0), NH.z));
    T len2 = dot(NM, NM);
    if (len2 < M<T>::Eps) NM = V3<T>(0, 0, 1);
    else NM = NM * (T(1) / M<T>::sqrt(len2));
    pdf = vndf_pdf(V, NM, alpha);
    return NM;
}

template <class T> struct MetalP {
    V3<T> eta, k, spec;
    T rough;
};
template <class T> inline MetalP<T> metal_params(const float* p) {
    return {V3<T>(p[0], p[1], p[2]), V3<T>(p[3], p[4], p[5]), V3<T>(p[6], p[7], p[8]), T(p[9])};
}

// MetalGlassMaterialsKC.cuh:26-146
template <class T>
BSample<T> metal_sample(const MetalP<T>& m, V3<T> wi, const Surface<T>& sf, T xi0, T xi1,
                        uint32_t medium) {
    T alpha = m.rough * m.rough;
    V3<T> V = to_tangent(wi, sf.w2t);
    BSample<T> out;
    T pdf;
    V3<T> H = vndf_sample(pdf, V, alpha, xi0, xi1);
    T VdH = std::fmax(T(0), dot(V, H));
    V3<T> L = T(2) * VdH * H - V;
    pdf = (VdH == T(0)) ? T(0) : pdf / (T(4) * VdH);
    T LdH = std::fmax(T(0), dot(L, H));
    T NdH = std::fmax(T(0), H.z);
    T NdV = std::fmax(T(0), V.z);
    V3<T> F = fresnel_conductor(VdH, m.eta, m.k);
    F = F * m.spec;
    T D = dggx(NdH, alpha);
    T G = g_smith_corr(V, L, alpha);
    G = (LdH == T(0)) ? T(0) : G;
    G = (VdH == T(0)) ? T(0) : G;
    V3<T> st = D * F * G * T(0.25) / NdV;
    st = (NdV == T(0)) ? V3<T>() : st;
    if (std::isinf(D) || std::isnan(D)) {
        if (m.rough == T(0)) L = T(2) * V.z * V3<T>(0, 0, 1) - V;
        st = G * F;
        T gs = g_smith_single(V, alpha);
        if (gs != T(0)) st = st / gs;
        else st = V3<T>();
        pdf = T(1);
    }
    out.dir = to_space(L, sf.w2t);
    out.pos = nudge(sf.pos, sf.geo);
    out.refl = st;
    out.pdf = pdf;
    out.medium = medium;
    return out;
}
// MetalGlassMaterialsKC.cuh:174-214
template <class T>
V3<T> metal_eval(const MetalP<T>& m, V3<T> wo, V3<T> wi, const Surface<T>& sf) {
    T alpha = m.rough * m.rough;
    V3<T> L = to_tangent(wo, sf.w2t);
    V3<T> V = to_tangent(wi, sf.w2t);
    V3<T> H = normalize(L + V);
    T LdH = std::fmax(T(0), dot(L, H));
    T VdH = std::fmax(T(0), dot(V, H));
    T NdH = std::fmax(T(0), H.z);
    T NdV = std::fmax(T(0), V.z);
    T D = dggx(NdH, alpha);
    D = (std::isnan(D) || std::isinf(D)) ? T(0) : D;
    T G = g_smith_corr(V, L, alpha);
    G = (LdH == T(0)) ? T(0) : G;
    G = (VdH == T(0)) ? T(0) : G;
    V3<T> F = fresnel_conductor(VdH, m.eta, m.k);
    F = F * m.spec;
    V3<T> st = D * F * G * T(0.25) / NdV;
    return (NdV == T(0)) ? V3<T>() : st;
}
// LambertMaterialKC.cuh:14-103
template <class T>
BSample<T> lambert_sample(V3<T> albedo, const Surface<T>& sf, T xi0, T xi1, uint32_t medium) {
    BSample<T> out;
    T pdf;
    V3<T> d = hemi_cosine(xi0, xi1, pdf);
    d = normalize(d);
    T nDotL = std::fmax(d.z, T(0));
    out.dir = to_space(d, sf.w2t);
    out.pos = nudge(sf.pos, sf.geo);
    out.refl = nDotL * albedo * M<T>::InvPi;
    out.pdf = pdf;
    out.medium = medium;
    return out;
}
template <class T> V3<T> lambert_eval(V3<T> albedo, V3<T> wo, const Surface<T>& sf) {
    V3<T> n = to_space(V3<T>(0, 0, 1), sf.w2t);
    T nDotL = std::fmax(dot(n, wo), T(0));
    return nDotL * albedo * M<T>::InvPi;
}
// SimpleMaterialsKC.cuh:172-286 and Ray::Reflect/Refract (Ray.hpp:302-356)
template <class T>
BSample<T> refract_sample(V3<T> albedo, uint32_t matMedium, const oracle_scene* s, V3<T> wi,
                          const Surface<T>& sf, uint32_t curMedium, T xi) {
    BSample<T> out;
    T iIOR = T(s->medium_ior[matMedium]);
    T dIOR = T(s->medium_ior[s->base_medium]);
    V3<T> n = to_space(V3<T>(0, 0, 1), sf.w2t);
    bool entering = !sf.back;
    T from = T(s->medium_ior[curMedium]);
    T to = entering ? iIOR : dIOR;
    T f = fresnel_dielectric(std::fabs(dot(wi, n)), from, to);
    if (xi < f) {
        out.dir = T(2) * dot(wi, n) * n - wi;
        out.pos = nudge(sf.pos, sf.geo);
        out.pdf = f;
        out.medium = curMedium;
        out.refl = f * albedo;
        return out;
    }
    out.medium = entering ? matMedium : s->base_medium;
    out.pdf = T(1) - f;
    T ratio = from / to;
    T cosIn = dot(n, wi);
    T sinInSqr = std::fmax(T(0), T(1) - cosIn * cosIn);
    T sinOutSqr = ratio * ratio * sinInSqr;
    T cosOut = M<T>::sqrt(std::fmax(T(0), T(1) - sinOutSqr));
    if (sinOutSqr >= T(1)) {
        out.pdf = T(0);
        out.refl = V3<T>();
        out.dir = wi;
        out.pos = sf.pos;
        return out;
    }
    out.dir = ratio * (-wi) + (ratio * cosIn - cosOut) * n;
    out.pos = nudge(sf.pos, -sf.geo);
    out.refl = albedo * T(1) * (T(1) - f);
    return out;
}

// Quat::RotationBetweenZAxis (Quaternion.hpp:333-358)
template <class T> inline Q4<T> rotation_between_z(V3<T> b) {
    V3<T> zc(-b.y, b.x, T(0));
    const T zd = b.z;
    const T sn = M<T>::sqrt((T(1) - zd) * T(0.5));
    const T cs = M<T>::sqrt((zd + T(1)) * T(0.5));
    zc = normalize(zc);
    if (std::fabs(zd + T(1)) < M<T>::LargeEps) return Q4<T>{T(0), T(0), T(1), T(0)};
    if (std::fabs(zd - T(1)) < M<T>::LargeEps) return Q4<T>{T(1), T(0), T(0), T(0)};
    return Q4<T>{cs, zc.x * sn, zc.y * sn, zc.z * sn};
}
// LambertConstFuncs (SimpleMaterialsKC.cuh:16-103), HemiUniformCDF
// (HemiDistribution.h:34-51)
template <class T>
BSample<T> lambertc_sample(V3<T> albedo, const Surface<T>& sf, T xi0, T xi1, uint32_t medium) {
    BSample<T> out;
    const V3<T> n = to_space(V3<T>(0, 0, 1), sf.w2t);
    const T c0 = M<T>::sqrt(std::fmax(T(0), T(1) - xi0 * xi0));
    const T c1 = T(2) * M<T>::Pi * xi1;
    T sn, cs;
    M<T>::sincos(c1, sn, cs);
    V3<T> d(c0 * cs, c0 * sn, xi0);
    out.pdf = M<T>::InvPi * T(0.5f);
    d = normalize(d);
    d = qrotate(rotation_between_z(n), d);
    const T nDotL = std::fabs(dot(n, d));
    out.dir = d;
    out.pos = nudge(sf.pos, sf.geo);
    out.refl = nDotL * albedo * M<T>::InvPi;
    out.medium = medium;
    return out;
}
template <class T> V3<T> lambertc_eval(V3<T> albedo, V3<T> wo, const Surface<T>& sf) {
    const V3<T> n = to_space(V3<T>(0, 0, 1), sf.w2t);
    return std::fmax(dot(n, wo), T(0)) * albedo * M<T>::InvPi;
}
template <class T> T lambert_pdf(V3<T> wo, const Surface<T>& sf) {
    const V3<T> n = to_space(V3<T>(0, 0, 1), sf.w2t);
    return std::fmax(dot(wo, n), T(0)) * M<T>::InvPi;
}
// MetalMatFuncs::Pdf (MetalGlassMaterialsKC.cuh:148-172)
template <class T> T metal_pdf(const MetalP<T>& m, V3<T> wo, V3<T> wi, const Surface<T>& sf) {
    const T alpha = m.rough * m.rough;
    const V3<T> L = to_tangent(wo, sf.w2t), V = to_tangent(wi, sf.w2t);
    const V3<T> H = normalize(L + V);
    const T NdH = std::fmax(T(0), H.z), VdH = std::fmax(T(0), dot(V, H));
    T p = vndf_pdf(V, H, alpha);
    const T D = dggx(NdH, alpha);
    p = (std::isnan(D) || std::isinf(D)) ? T(0) : p;
    return (VdH == T(0)) ? T(0) : p / (T(4) * VdH);
}
// UnrealDeviceFuncs (UnrealMaterialKC.cuh:19-359)
template <class T> struct UnrealP {
    V3<T> albedo;
    T rough, metallic, specular;
};
template <class T> inline UnrealP<T> unreal_params(const float* p) {
    return {V3<T>(p[0], p[1], p[2]), T(p[3]), T(p[4]), T(p[5])};
}
template <class T> inline T luminance(V3<T> c) {  // ColorConversion.h:15-21
    return T(0.2120f) * c.x + T(0.7150f) * c.y + T(0.0722f) * c.z;
}
template <class T> inline T unreal_mis_ratio(T metallic, T specular, T lum) {
    T diffuse = T(2) * M<T>::Pi * lum;
    diffuse *= (T(1) - metallic);
    const T specRatio = (T(1) - metallic) * specular + metallic * lum;
    const T total = specRatio + diffuse;
    return diffuse / total;
}
template <class T> inline V3<T> unreal_f0(V3<T> albedo, T metallic, T specular) {
    specular *= T(0.08f);
    return V3<T>(specular, specular, specular) * (T(1) - metallic) + albedo * metallic;
}
template <class T> inline V3<T> f_schlick(T VdH, V3<T> f0) {  // TracerFunctions.cuh:160-179
    const T pt = T(1) - VdH;
    T p5 = pt * pt;
    p5 *= p5;
    p5 *= pt;
    V3<T> r = (V3<T>(1, 1, 1) - f0) * p5;
    return r + f0;
}
template <class T>
BSample<T> unreal_sample(const UnrealP<T>& m, V3<T> wi, const Surface<T>& sf, T xiSel, T xi0,
                         T xi1, uint32_t medium) {
    BSample<T> out;
    const T alpha = m.rough * m.rough;
    const V3<T> V = to_tangent(wi, sf.w2t);
    T misRatio = unreal_mis_ratio(m.metallic, m.specular, luminance(m.albedo));
    const bool diffuse = xiSel < misRatio;
    T VdH, pdfSel, pdfOther;
    V3<T> H, L;
    if (diffuse) {
        L = hemi_cosine(xi0, xi1, pdfSel);
        H = normalize(V + L);
        VdH = std::fmax(T(0), dot(V, H));
        pdfOther = vndf_pdf(V, H, alpha);
        pdfOther = (VdH == T(0)) ? T(0) : pdfOther / (T(4) * VdH);
    } else {
        H = vndf_sample(pdfSel, V, alpha, xi0, xi1);
        VdH = std::fmax(T(0), dot(V, H));
        L = T(2) * VdH * H - V;
        pdfOther = std::fmax(T(0), L.z) * M<T>::InvPi;
        pdfSel = (VdH == T(0)) ? T(0) : pdfSel / (T(4) * VdH);
        misRatio = T(1) - misRatio;
    }
    T& pdfSpec = diffuse ? pdfOther : pdfSel;
    pdfSpec = (VdH == T(0)) ? T(0) : pdfSpec;
    const T LdH = std::fmax(T(0), dot(L, H)), NdH = std::fmax(T(0), H.z),
            NdV = std::fmax(T(0), V.z);
    const T D = dggx(NdH, alpha);
    T G = g_smith_corr(V, L, alpha);
    G = (LdH == T(0)) ? T(0) : G;
    G = (VdH == T(0)) ? T(0) : G;
    const V3<T> F = f_schlick(VdH, unreal_f0(m.albedo, m.metallic, m.specular));
    V3<T> spec = D * F * G * T(0.25) / NdV;
    spec = (NdV == T(0)) ? V3<T>() : spec;
    if (std::isinf(D) || std::isnan(D)) {
        spec = G * F / g_smith_single(V, alpha);
        pdfSpec = diffuse ? T(0) : T(1);
    }
    const T NdL = std::fmax(T(0), L.z);
    const V3<T> diffAlbedo = (T(1) - m.metallic) * m.albedo;
    const V3<T> diffTerm = NdL * diffAlbedo * M<T>::InvPi;
    const T w0 = misRatio * pdfSel, w1 = (T(1) - misRatio) * pdfOther;
    const T misWeight = w0 / (w0 + w1);
    out.pdf = (pdfSel == T(0)) ? T(0) : (misRatio * pdfSel / misWeight);
    out.dir = to_space(L, sf.w2t);
    out.pos = nudge(sf.pos, sf.geo);
    out.refl = diffTerm + spec;
    out.medium = medium;
    return out;
}
template <class T>
V3<T> unreal_eval(const UnrealP<T>& m, V3<T> wo, V3<T> wi, const Surface<T>& sf) {
    const T alpha = m.rough * m.rough;
    const V3<T> L = to_tangent(wo, sf.w2t), V = to_tangent(wi, sf.w2t);
    const V3<T> H = normalize(L + V);
    const T LdH = std::fmax(T(0), dot(L, H)), VdH = std::fmax(T(0), dot(V, H));
    const T NdH = std::fmax(T(0), H.z), NdV = std::fmax(T(0), V.z);
    T D = dggx(NdH, alpha);
    D = (std::isnan(D) || std::isinf(D)) ? T(0) : D;
    T G = g_smith_corr(V, L, alpha);
    G = (LdH == T(0)) ? T(0) : G;
    G = (VdH == T(0)) ? T(0) : G;
    const V3<T> F = f_schlick(VdH, unreal_f0(m.albedo, m.metallic, m.specular));
    V3<T> spec = D * F * G * T(0.25) / NdV;
    spec = (NdV == T(0)) ? V3<T>() : spec;
    const T NdL = std::fmax(T(0), L.z);
    const V3<T> diffTerm = NdL * ((T(1) - m.metallic) * m.albedo) * M<T>::InvPi;
    return diffTerm + spec;
}
template <class T> T unreal_pdf(const UnrealP<T>& m, V3<T> wo, V3<T> wi, const Surface<T>& sf) {
    const T alpha = m.rough * m.rough;
    const V3<T> L = to_tangent(wo, sf.w2t), V = to_tangent(wi, sf.w2t);
    const V3<T> H = normalize(L + V);
    const T NdH = std::fmax(T(0), H.z), VdH = std::fmax(T(0), dot(V, H));
    T ps = vndf_pdf(V, H, alpha);
    const T D = dggx(NdH, alpha);
    ps = (std::isnan(D) || std::isinf(D)) ? T(0) : ps;
    ps = (VdH == T(0)) ? T(0) : ps / (T(4) * VdH);
    const T pd = std::fmax(T(0), L.z) * M<T>::InvPi;
    const T r = unreal_mis_ratio(m.metallic, m.specular, luminance(m.albedo));
    return r * pd + (T(1) - r) * ps;
}
template <class T> inline T power_heuristic(T p0, T p1) {  // TracerFunctions.cuh:300-308
    const T w0 = T(1) * p0, w1 = T(1) * p1;
    return (w0 * w0) / (w0 * w0 + w1 * w1);
}


// ========================================================================
// Wavefront path guiding (WFPGTracer.cu, WFPGTracerKC.cuh, AnisoSVO.cu/.cuh,
// ProductSampler.cuh, BlockTextureFilter.cuh, PathNode.cuh), FP32,
// processed depth by depth over every path of the frame.  The bin counts
// and the fixed-point radiance sums are order independent, the per-bin and
// per-ray random numbers are keyed by bin / path, so the octree state and
// every guided direction are reproducible exactly.
// ========================================================================
constexpr uint32_t kSvoInvalidParent = 0xFFFFFFFu;
constexpr uint32_t kBinMark = 0x80000000u;
constexpr uint32_t kBinLeaf = 0x80000000u;
constexpr uint32_t kBinInvalid = 0xFFFFFFFFu;
constexpr uint16_t kHalfMax = 0x7BFFu;
constexpr double kFixScale = 16777216.0;
constexpr uint32_t kTagGuide = 0x20000u;
constexpr uint32_t kTagGuideBin = 0x30000u;
constexpr uint32_t kGuideValid = 1u << 17;
constexpr uint32_t kGuideBxdf = 1u << 16;

inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitsf(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t f2u_sat(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967040.0f) return 0xFFFFFFFFu;
    return static_cast<uint32_t>(x);
}
inline int32_t f2i_sat(float x) {
    if (x != x) return 0;
    if (x >= 2147483520.0f) return 0x7FFFFFFF;
    if (x <= -2147483648.0f) return static_cast<int32_t>(0x80000000u);
    return static_cast<int32_t>(x);
}
// IEEE binary32 -> binary16, round to nearest even
inline uint16_t f2h(float f) {
    const uint32_t x = fbits(f);
    const uint32_t sign = (x >> 16) & 0x8000u;
    const uint32_t ax = x & 0x7FFFFFFFu;
    if (ax > 0x7F800000u) return uint16_t(sign | 0x7E00u);
    if (ax >= 0x47800000u) return uint16_t(sign | 0x7C00u);
    if (ax < 0x38800000u) {
        const uint32_t e = ax >> 23;
        if (e == 0) return uint16_t(sign);
        const uint32_t m = (ax & 0x7FFFFFu) | 0x800000u;
        const uint32_t sh = 126u - e;
        if (sh > 24u) return uint16_t(sign);
        uint32_t q = m >> sh;
        const uint32_t rem = m & ((1u << sh) - 1u), halfway = 1u << (sh - 1u);
        if (rem > halfway || (rem == halfway && (q & 1u))) q++;
        return uint16_t(sign | q);
    }
    uint32_t h = (((ax >> 23) - 112u) << 10) | ((ax & 0x7FFFFFu) >> 13);
    const uint32_t rem = ax & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
    return uint16_t(sign | h);
}
inline float h2f(uint16_t h) {
    const uint32_t sign = (uint32_t(h) & 0x8000u) << 16;
    const uint32_t e = (h >> 10) & 0x1Fu, m = h & 0x3FFu;
    if (e == 0) {
        if (m == 0) return bitsf(sign);
        const float v = static_cast<float>(m) * 0x1p-24f;
        return sign ? -v : v;
    }
    if (e == 31) return bitsf(sign | 0x7F800000u | (m << 13));
    return bitsf(sign | ((e + 112u) << 23) | (m << 13));
}
inline float next_up(float x) {
    if (x != x || x == bitsf(0x7F800000u)) return x;
    if (x == 0.0f) return bitsf(1u);
    const uint32_t b = fbits(x);
    return bitsf(x > 0.0f ? b + 1u : b - 1u);
}
// "lowbias32" integer hash (C. Wellons, hash-prospector)
inline uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}
using F3 = V3<float>;
using FQ = Q4<float>;

// RayLib/CoordinateConversion.h:112-233
constexpr float kTwoOvrPiF = 0x1.45f306p-1f;
constexpr float kPiOvr4F = 0x1.921fb6p-1f;
inline void dir_to_octa(F3 d, float& s, float& t) {
    if (d.x == 0.0f && d.y == 0.0f) { s = 0.0f; t = 0.0f; return; }
    const float xAbs = std::fabs(d.x), yAbs = std::fabs(d.y);
    const float phiPrime = pm_atan2(yAbs, xAbs);
    const float radius = std::sqrt(1.0f - std::fabs(d.z));
    float v = radius * kTwoOvrPiF * phiPrime;
    float u = radius - v;
    if (d.z < 0.0f) {
        const float up = 1.0f - v, vp = 1.0f - u;
        u = up;
        v = vp;
    }
    u *= std::signbit(d.x) ? -1.0f : 1.0f;
    v *= std::signbit(d.y) ? -1.0f : 1.0f;
    s = (u + 1.0f) * 0.5f;
    t = (v + 1.0f) * 0.5f;
}
inline F3 octa_to_dir(float s, float t) {
    const float u = s * 2.0f - 1.0f, v = t * 2.0f - 1.0f;
    const float ua = std::fabs(u), va = std::fabs(v);
    const float d = 1.0f - (ua + va);
    const float radius = 1.0f - std::fabs(d);
    float phiPrime = 0.0f;
    if (radius != 0.0f) phiPrime = ((va - ua) / radius + 1.0f) * kPiOvr4F;
    float sp, cp;
    pm_sincos(phiPrime, sp, cp);
    const float cosPhi = (std::signbit(u) ? -1.0f : 1.0f) * cp;
    const float sinPhi = (std::signbit(v) ? -1.0f : 1.0f) * sp;
    const float z = (std::signbit(d) ? -1.0f : 1.0f) * (1.0f - radius * radius);
    const float xyFactor = radius * std::sqrt(2.0f - radius * radius);
    return F3(cosPhi * xyFactor, sinPhi * xyFactor, z);
}
inline F3 octa_to_dir_yup(float s, float t) {
    const F3 r = octa_to_dir(s, t);
    return F3(r.y, r.z, r.x);
}
inline void dir_yup_to_octa(F3 d, float& s, float& t) { dir_to_octa(F3(d.z, d.x, d.y), s, t); }
inline void octa_wrap(float& s, float& t) {
    float a = s, b = t;
    if (s < 0.0f) a = -2.0f - s;
    if (t < 0.0f) b = -2.0f - t;
    const float ia = std::trunc(a), ib = std::trunc(b);
    float fa = std::fabs(a - ia), fb = std::fabs(b - ib);
    const int32_t ii = f2i_sat(ia), ij = f2i_sat(ib);
    if ((ii & 1) ^ (ij & 1)) {
        fa = 1.0f - fa;
        fb = 1.0f - fb;
    }
    s = fa;
    t = fb;
}
inline void octa_wrap_int(int32_t& x, int32_t& y, int32_t dimX, int32_t dimY) {
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
// Utility::SphericalToCartesianUnit of the 2 x 16-bit voxel normal
inline F3 unpack_normal16(uint32_t pn) {
    const float az = static_cast<float>(pn & 0xFFFFu) / 65535.0f * (kPiF * 2.0f) - kPiF;
    const float in = static_cast<float>(pn >> 16) / 65535.0f * kPiF;
    float sa, ca, si, ci;
    pm_sincos(az, sa, ca);
    pm_sincos(in, si, ci);
    return normalize(F3(ca * si, sa * si, ci));
}
// VoxelPayload::ReadNormalAndSpecular / WriteNormalAndSpecular
inline F3 read_normal_spec(uint32_t packed, float& stdDev, float& spec) {
    const float kx = (1.0f / 511.0f) * 2.0f;
    float nx = static_cast<float>(packed & 511u) * kx;
    float ny = static_cast<float>((packed >> 9) & 511u) * kx;
    nx -= 1.0f;
    ny -= 1.0f;
    const float nz = std::sqrt(std::fmax(0.0f, 1.0f - nx * nx - ny * ny));
    F3 n = normalize(F3(nx, ny, nz));
    if ((packed >> 31) & 1u) n.z *= -1.0f;
    const float len = static_cast<float>((packed >> 18) & 127u) * (1.0f / 127.0f);
    spec = static_cast<float>((packed >> 25) & 63u) * (1.0f / 6.0f);
    stdDev = (1.0f - len) / len;
    return n;
}
inline uint32_t write_normal_spec(F3 n, float spec) {
    const float length = std::sqrt(dot(n, n));
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
    const uint32_t sz = std::signbit(n.z) ? 1u : 0u;
    return (px & 511u) | ((py & 511u) << 9) | ((pl & 127u) << 18) | ((ps & 63u) << 25) | (sz << 31);
}
inline uint64_t to_fixed(float x) {
    return (x > 0.0f) ? static_cast<uint64_t>(std::nearbyint(static_cast<double>(x) * kFixScale)) : 0ull;
}
inline float lum3(F3 c) { return 0.2120f * c.x + 0.7150f * c.y + 0.0722f * c.z; }

inline uint32_t node_child_index(uint64_t n) { return uint32_t(n & 0x7FFFFFFull); }
inline uint32_t node_parent(uint64_t n) { return uint32_t((n >> 27) & 0xFFFFFFFull); }
inline uint32_t node_mask(uint64_t n) { return uint32_t((n >> 55) & 0xFFull); }
inline bool node_children_leaf(uint64_t n) { return (n >> 63) != 0; }
inline uint32_t node_child_offset(uint64_t n, uint32_t c) {
    return uint32_t(__builtin_popcount(((1u << c) - 1u) & node_mask(n)));
}

struct Chain {
    uint32_t levels, paths;
    std::vector<float> pos;      // levels * paths * 3
    std::vector<float> rf;       // levels * paths * 3
    std::vector<uint8_t> valid;  // levels * paths
    std::vector<float> nee, path;
    // shadow-ray event of the NEE / path ray of each slot for the vertex
    // that launched it: 1 its light contribution was taken, 2 (NEE only)
    // it was stopped by a surface
    std::vector<uint8_t> eventNee, eventPath;
    Chain(uint32_t L, uint32_t P)
        : levels(L), paths(P), pos(size_t(L) * P * 3, 0.0f), rf(size_t(L) * P * 3, 0.0f),
          valid(size_t(L) * P, 0), nee(size_t(L) * P * 3, 0.0f), path(size_t(L) * P * 3, 0.0f),
          eventNee(size_t(L) * P, 0), eventPath(size_t(L) * P, 0) {}
    size_t at(uint32_t d, uint32_t p) const { return size_t(d) * paths + p; }
};


// PathTracerPathWork (PathTracerKC.cuh:428-649); with a chain and guide
// words it is WFPGTracerPathWork (WFPGTracerKC.cuh:212-519), FP32 only.
template <class T>
void path_work(Ctx<T>& c, const PRay<T>& r, uint32_t prim, T ha, T hb, uint32_t batch,
               uint32_t id, bool gen, std::vector<PRay<T>>& next,
               const uint32_t* guide = nullptr, Chain* chain = nullptr) {
    const oracle_scene* s = c.s;
    const Aux<T>& aux = r.aux;
    if (aux.type == NEE_RAY) return;
    if (!gen && !chain) return;  // outputs of the last iteration are never traced
    Surface<T> sf = gen_surface(s, prim, ha, hb, r.d);
    V3<T> wi = -normalize(r.d);
    V3<T> rf = aux.rf;  // vacuum / sigmaT == 0 transmittance is exactly 1
    bool specular;
    if (batch == kBatchLambert || batch == kBatchLambertC) specular = false;
    else if (batch == kBatchMetal) specular = (T(1) - T(s->metal_params[10 * id + 9])) >= T(0.99f);
    else if (batch == kBatchUnreal) specular = (T(1) - T(s->unreal_params[6 * id + 3])) >= T(0.99f);
    else specular = true;
    if constexpr (std::is_same_v<T, float>) {
        if (chain) {
            // WFPGPathNode of this vertex; the rays it launches start empty
            const size_t at = chain->at(aux.depth, aux.sample);
            chain->pos[3 * at] = sf.pos.x;
            chain->pos[3 * at + 1] = sf.pos.y;
            chain->pos[3 * at + 2] = sf.pos.z;
            chain->rf[3 * at] = rf.x;
            chain->rf[3 * at + 1] = rf.y;
            chain->rf[3 * at + 2] = rf.z;
            chain->valid[at] = 1;
            if (aux.depth + 1 < chain->levels) {
                const size_t nx = chain->at(aux.depth + 1, aux.sample);
                for (int k = 0; k < 3; k++) chain->nee[3 * nx + k] = chain->path[3 * nx + k] = 0.0f;
                chain->eventNee[nx] = chain->eventPath[nx] = 0;
            }
        }
    }
    if (!gen) return;
    uint32_t sampleIdx = aux.sample;
    Rng4 ra = rng_block(sampleIdx, c.o->frame, aux.depth, 0, c.o->seed_lo, c.o->seed_hi);
    Rng4 rb = rng_block(sampleIdx, c.o->frame, aux.depth, 1, c.o->seed_lo, c.o->seed_hi);

    // ---- NEE (PathTracerKC.cuh:505-583) ----
    if (c.o->nee && !specular && s->light_count > 0) {
        uint32_t lc = s->light_count;
        float r1 = ra.u[0] * static_cast<float>(lc);
        uint32_t li = static_cast<uint32_t>(r1);
        if (li == lc) li--;
        uint32_t lp = s->light_prim[li];
        // PrimSamplePos (GPUPrimitiveTriangle.h:65-115)
        T sx = M<T>::sqrt(T(ra.u[1]));
        T r2 = T(ra.u[2]);
        T la = T(1) - sx;
        T lb = (T(1) - r2) * sx;
        T lcw = sx * r2;
        uint32_t i0 = s->idx[3 * lp], i1 = s->idx[3 * lp + 1], i2 = s->idx[3 * lp + 2];
        V3<T> p0 = vpos<T>(s, i0), p1 = vpos<T>(s, i1), p2 = vpos<T>(s, i2);
        T area = M<T>::sqrt(dot(cross(p1 - p0, p2 - p0), cross(p1 - p0, p2 - p0))) * T(0.5);
        T lpdf = T(1) / area;
        Q4<T> q = bary_slerp(qnormalize(vtbn<T>(s, i0)), qnormalize(vtbn<T>(s, i1)),
                             qnormalize(vtbn<T>(s, i2)), la, lb);
        V3<T> ln = to_space(V3<T>(0, 0, 1), q);
        V3<T> lpos = (p0 * la + p1 * lb) + p2 * lcw;
        ln = normalize(ln);
        V3<T> ldir = lpos - sf.pos;
        T d2 = dot(ldir, ldir);
        T dist = M<T>::sqrt(d2);
        ldir = ldir * (T(1) / dist);
        T nDotL = std::fabs(dot(ln, -ldir));
        lpdf *= d2 / nDotL;
        lpdf *= (T(1) / static_cast<T>(lc));
        V3<T> refl;
        T pdfBxdf = T(0);
        const bool mis = c.o->mis != 0;
        if (batch == kBatchLambert) {
            const float* al = s->lambert_albedo + 3 * id;
            refl = lambert_eval(V3<T>(al[0], al[1], al[2]), ldir, sf);
            if (mis) pdfBxdf = lambert_pdf(ldir, sf);
        } else if (batch == kBatchLambertC) {
            const float* al = s->lambertc_albedo + 3 * id;
            refl = lambertc_eval(V3<T>(al[0], al[1], al[2]), ldir, sf);
            if (mis) pdfBxdf = lambert_pdf(ldir, sf);
        } else if (batch == kBatchUnreal) {
            const UnrealP<T> up = unreal_params<T>(s->unreal_params + 6 * id);
            refl = unreal_eval(up, ldir, wi, sf);
            if (mis) pdfBxdf = unreal_pdf(up, ldir, wi, sf);
        } else {
            const MetalP<T> mp = metal_params<T>(s->metal_params + 10 * id);
            refl = metal_eval(mp, ldir, wi, sf);
            if (mis) pdfBxdf = metal_pdf(mp, ldir, wi, sf);
        }
        T pdfNee = lpdf;
        if (mis) {
            pdfNee /= power_heuristic(lpdf, pdfBxdf);
            if (std::isnan(pdfNee)) pdfNee = T(0);
        }
        V3<T> nrf = rf * refl;
        nrf = (pdfNee == T(0)) ? V3<T>() : (nrf / pdfNee);
        if (nrf != V3<T>()) {
            PRay<T> o;
            o.o = nudge(sf.pos, sf.geo);
            o.d = ldir;
            o.tmin = T(0);
            o.tmax = M<T>::Max;
            o.aux = aux;
            o.aux.rf = nrf;
            o.aux.endpoint = li;
            o.aux.type = NEE_RAY;
            o.aux.prevPDF = std::numeric_limits<T>::quiet_NaN();
            next.push_back(o);
        }
    }
    // ---- BxDF sample (PathTracerKC.cuh:585-648), or the guided direction
    BSample<T> bs;
    bool guided = false;
    if constexpr (std::is_same_v<T, float>) {
        if (guide && !specular) {
            const float gp = h2f(uint16_t(guide[1] & 0xFFFFu));
            if ((guide[1] & kGuideValid) && gp == gp) {
                const F3 dir = octa_to_dir_yup(h2f(uint16_t(guide[0] & 0xFFFFu)), h2f(uint16_t(guide[0] >> 16)));
                bs.dir = dir;
                bs.pdf = gp;
                bs.pos = nudge(sf.pos, sf.geo);
                bs.medium = aux.medium;
                if (batch == kBatchLambert) {
                    const float* al = s->lambert_albedo + 3 * id;
                    bs.refl = lambert_eval(F3(al[0], al[1], al[2]), dir, sf);
                } else if (batch == kBatchLambertC) {
                    const float* al = s->lambertc_albedo + 3 * id;
                    bs.refl = lambertc_eval(F3(al[0], al[1], al[2]), dir, sf);
                } else if (batch == kBatchUnreal) {
                    bs.refl = unreal_eval(unreal_params<float>(s->unreal_params + 6 * id), dir, wi, sf);
                } else {
                    bs.refl = metal_eval(metal_params<float>(s->metal_params + 10 * id), dir, wi, sf);
                }
                guided = true;
            }
        }
    }
    if (guided) {
    } else if (batch == kBatchLambert) {
        const float* al = s->lambert_albedo + 3 * id;
        bs = lambert_sample(V3<T>(al[0], al[1], al[2]), sf, T(rb.u[0]), T(rb.u[1]), aux.medium);
    } else if (batch == kBatchLambertC) {
        const float* al = s->lambertc_albedo + 3 * id;
        bs = lambertc_sample(V3<T>(al[0], al[1], al[2]), sf, T(rb.u[0]), T(rb.u[1]), aux.medium);
    } else if (batch == kBatchUnreal) {
        bs = unreal_sample(unreal_params<T>(s->unreal_params + 6 * id), wi, sf, T(rb.u[2]),
                           T(rb.u[0]), T(rb.u[1]), aux.medium);
    } else if (batch == kBatchMetal) {
        bs = metal_sample(metal_params<T>(s->metal_params + 10 * id), wi, sf, T(rb.u[0]),
                          T(rb.u[1]), aux.medium);
    } else {
        const float* al = s->refract_albedo + 3 * id;
        bs = refract_sample(V3<T>(al[0], al[1], al[2]), s->refract_medium[id], s, wi, sf,
                            aux.medium, T(rb.u[0]));
    }
    V3<T> prf = rf * bs.refl;
    prf = (bs.pdf == T(0)) ? V3<T>() : (prf / bs.pdf);
    T avg = dot(prf, V3<T>(T(0.333f), T(0.333f), T(0.333f)));
    bool term = false;
    if (!specular && aux.depth > c.o->rr_start) {
        // TracerFunctions.cuh:320-331
        T prob = std::fmin(std::fmax(avg, T(0.005f)), T(1));
        if (T(ra.u[3]) >= prob) term = true;
        else prf = prf * (T(1) / prob);
    }
    if ((!term || specular) && prf != V3<T>()) {
        PRay<T> o;
        o.o = bs.pos;
        o.d = bs.dir;
        o.tmin = T(0);
        o.tmax = M<T>::Max;
        o.aux = aux;
        o.aux.medium = bs.medium;
        o.aux.rf = prf;
        o.aux.type = specular ? SPECULAR_PATH_RAY : PATH_RAY;
        o.aux.prevPDF = bs.pdf;
        o.aux.depth = aux.depth + 1;
        next.push_back(o);
    }
}

// PathTracerKC.cuh:335-426
template <class T>
void boundary_work(Ctx<T>& c, const PRay<T>& r, uint32_t lightIdx, uint32_t prim, T ha, T hb,
                   T hitT, Chain* chain = nullptr) {
    const Aux<T>& aux = r.aux;
    const oracle_scene* s = c.s;
    const bool pathAsMis = c.o->mis && aux.type == PATH_RAY;
    T misWeight = T(1);
    if (pathAsMis) {
        const Surface<T> sf = gen_surface(s, prim, ha, hb, r.d);
        const V3<T> dir = normalize(r.d);
        T pdfM = T(0), pdfC = T(0);
        if (lightIdx < s->light_count) {
            pdfM = T(1) / static_cast<T>(s->light_count);
            uint32_t i0 = s->idx[3 * prim], i1 = s->idx[3 * prim + 1], i2 = s->idx[3 * prim + 2];
            V3<T> p0 = vpos<T>(s, i0), p1 = vpos<T>(s, i1), p2 = vpos<T>(s, i2);
            V3<T> cr = cross(p1 - p0, p2 - p0);
            T area = M<T>::sqrt(dot(cr, cr)) * T(0.5);
            V3<T> ln = to_space(V3<T>(0, 0, 1), sf.w2t);
            T nDotL = std::fabs(dot(ln, -dir));
            pdfC = (T(1) / area) * hitT * hitT / nDotL;
        }
        misWeight = power_heuristic(aux.prevPDF, pdfC * pdfM);
    }
    bool camera = aux.type == CAMERA_RAY;
    bool specPath = aux.type == SPECULAR_PATH_RAY;
    bool neeOn = c.o->nee && aux.type == NEE_RAY;
    bool pathNeeOff = (!c.o->nee) && (aux.type == PATH_RAY || aux.type == SPECULAR_PATH_RAY);
    bool correct = neeOn && (aux.endpoint == lightIdx);
    if (pathNeeOff || pathAsMis || correct || camera || specPath) {
        const float* e = c.s->light_radiance + 3 * lightIdx;
        V3<T> total = V3<T>(T(e[0]), T(e[1]), T(e[2])) * aux.rf;
        total = total * misWeight;
        accumulate(c, aux.sample, total);
        if constexpr (std::is_same_v<T, float>) {
            // WFPGTracerBoundaryWork: AccumRadianceDownChain input
            if (chain && !camera) {
                const size_t at = chain->at(aux.depth, aux.sample);
                float* dst = (aux.type == NEE_RAY) ? &chain->nee[3 * at] : &chain->path[3 * at];
                dst[0] = total.x;
                dst[1] = total.y;
                dst[2] = total.z;
                // DepositNEEHitMiss(prev vertex, hit) (WFPGTracerKC.cuh:192-194)
                ((aux.type == NEE_RAY) ? chain->eventNee : chain->eventPath)[at] = 1;
            }
        }
    }
}

template <class T>
uint64_t render(const oracle_scene* s, const oracle_bvh* b, const oracle_camera* cam,
                const oracle_options* opt, T* out) {
    const uint32_t sp = opt->samples;
    const uint32_t SW = opt->width * sp, SH = opt->height * sp;
    uint32_t rowB = opt->row_begin, rowE = opt->row_end;
    if (rowE == 0 || rowE > SH) rowE = SH;
    if (rowB > rowE) rowB = rowE;
    const uint32_t rowStep = opt->row_step ? opt->row_step : 1;
    const uint32_t rowCount = (rowE - rowB + rowStep - 1) / rowStep;
    const uint32_t count = rowCount * SW;
    std::atomic<uint64_t> rays{0};
    const float* P = cam->position;
    parallel_for(count, opt->threads, [&](uint32_t b0, uint32_t b1) {
        Ctx<T> c{s, b, opt, out};
        uint64_t local = 0;
        std::vector<PRay<T>> cur, next;
        for (uint32_t k = b0; k < b1; k++) {
            uint32_t sid = (rowB + (k / SW) * rowStep) * SW + k % SW;
            out[3 * sid] = out[3 * sid + 1] = out[3 * sid + 2] = T(0);
            // Camera ray (GPUCameraPinhole.cuh:209-243; GenerationKernels.cuh:48-75)
            uint32_t sx = sid % SW, sy = sid / SW;
            Rng4 rc = rng_block(sid, opt->frame, kTagCamera, 0, opt->seed_lo, opt->seed_hi);
            float dx = cam->plane_size[0] / static_cast<float>(SW);
            float dy = cam->plane_size[1] / static_cast<float>(SH);
            float sdx = static_cast<float>(sx) * dx;
            float sdy = static_cast<float>(sy) * dy;
            sdx += rc.u[0] * dx;
            sdy += rc.u[1] * dy;
            V3<float> sp3;
            for (int i = 0; i < 3; i++) {
                float v = cam->bottom_left[i] + ((sdx * cam->right[i]) + (sdy * cam->up[i]));
                if (i == 0) sp3.x = v; else if (i == 1) sp3.y = v; else sp3.z = v;
            }
            V3<float> dirf = normalize(sp3 - V3<float>(P[0], P[1], P[2]));
            PRay<T> r;
            r.o = V3<T>(T(P[0]), T(P[1]), T(P[2]));
            r.d = V3<T>(T(dirf.x), T(dirf.y), T(dirf.z));
            r.tmin = T(cam->near_far[0]);
            r.tmax = T(cam->near_far[1]);
            r.aux = Aux<T>{V3<T>(1, 1, 1), sid, kInvalid, s->base_medium, 0, CAMERA_RAY,
                           std::numeric_limits<T>::quiet_NaN()};
            cur.clear();
            cur.push_back(r);
            for (uint32_t it = 0; it < opt->max_depth && !cur.empty(); it++) {
                next.clear();
                bool gen = (it + 1) < opt->max_depth;
                for (const PRay<T>& ray : cur) {
                    local++;
                    Hit<T> h = trace_one<T>(s, b, ray.o, ray.d, ray.tmin, ray.tmax);
                    if (h.prim == kInvalid) continue;
                    uint32_t batch = h.key >> 24, id = h.key & 0xFFFFFFu;
                    if (batch == kBatchNull) continue;
                    if (batch == kBatchLight) boundary_work(c, ray, id, h.prim, h.b0, h.b1, h.t);
                    else path_work(c, ray, h.prim, h.b0, h.b1, batch, id, gen, next);
                }
                std::swap(cur, next);
            }
        }
        rays.fetch_add(local);
    });
    return rays.load();
}


// ------------------------------------------------------------------------
// Sparse voxel octree: TriFunctions::Voxelize (GPUPrimitiveTriangle.h:
// 385-620) and AnisoSVOctreeCPU::Constrcut (AnisoSVO.cu:657-1188) with its
// level kernels KCMarkMortonChanges / KCMarkChild / KCExtractChildrenCounts
// / KCSetChildrenPtrs / KCSetParentOf(Leaf)Children (AnisoSVO.cu:58-222),
// restated in the reference's own order (the device build derives the same
// canonical layout from prefix ranks instead).
// ------------------------------------------------------------------------
struct SvoP {
    float lo[3], hi[3];
    uint32_t res, depth;
    float leaf;
};
inline SvoP svo_params_of(const float ext[6], uint32_t res) {
    SvoP P{};
    float span[3] = {ext[3] - ext[0], ext[4] - ext[1], ext[5] - ext[2]};
    int md = 0;  // Vector::Max: first index of the largest component
    if (span[1] > span[md]) md = 1;
    if (span[2] > span[md]) md = 2;
    const float world = span[md];
    const float pad = world / static_cast<float>(res);
    for (int c = 0; c < 3; c++) {
        P.lo[c] = ext[c] - pad;
        P.hi[c] = ext[c] + (pad + world);
    }
    P.res = res;
    uint32_t d = 0;
    while ((1u << (d + 1)) <= res) d++;
    P.depth = d;
    P.leaf = (world + 2.0f * pad) / static_cast<float>(res);
    return P;
}

// returns the voxel count; writes codes/normals when out != nullptr
uint32_t voxelize_tri(const SvoP& P, V3<float> p0, V3<float> p1, V3<float> p2,
                      std::vector<uint64_t>* codes, std::vector<uint32_t>* normals) {
    using F3 = V3<float>;
    const F3 pos[3] = {p0, p1, p2};
    const F3 n = normalize(cross(p1 - p0, p2 - p0));
    const float an[3] = {std::fabs(n.x), std::fabs(n.y), std::fabs(n.z)};
    int dom = 0;
    float mx = an[0];
    if (an[1] > mx) { mx = an[1]; dom = 1; }
    if (an[2] > mx) { mx = an[2]; dom = 2; }
    const float nd = dom == 0 ? n.x : (dom == 1 ? n.y : n.z);
    const bool neg = std::signbit(nd);
    const float domSign = neg ? -1.0f : 1.0f;
    // Utility::CartesianToSphericalUnit (CoordinateConversion.h:97-108)
    const float az = pm_atan2(n.y, n.x);
    const float incl = pm_acos(std::fmin(std::fmax(n.z, -1.0f), 1.0f));
    const float s0 = (az + kPiF) * kInvPiF * 0.5f;
    const float s1 = incl * kInvPiF;
    int u = static_cast<int>(s0 * 65535.0f), v = static_cast<int>(s1 * 65535.0f);
    u = std::min(std::max(u, 0), 65535);
    v = std::min(std::max(v, 0), 65535);
    const uint32_t packed = uint32_t(u) | (uint32_t(v) << 16);
    // Quaternion(angle, axis) (Quaternion.hpp:15-24).  The half angle is
    // float(pi)/4 or float(pi)/2; their sin and cos are taken correctly
    // rounded (the values the C library returns for these two arguments),
    // not from the portable polynomials, which are an ulp off at pi/4.
    Q4<float> rot{1.0f, 0.0f, 0.0f, 0.0f};
    if (dom != 2 || neg) {
        const bool halfPi = (dom == 2);
        const float sn = halfPi ? 1.0f : 0x1.6a09e6p-1f;
        const float cs = halfPi ? -0x1.777a5cp-25f : 0x1.6a09e6p-1f;
        F3 axis = (dom == 0) ? F3(-domSign * 0.0f, -domSign * 1.0f, -domSign * 0.0f)
                 : (dom == 1) ? F3(domSign * 1.0f, domSign * 0.0f, domSign * 0.0f)
                              : F3(0.0f, 1.0f, 0.0f);
        rot = Q4<float>{cs, axis.x * sn, axis.y * sn, axis.z * sn};
    }
    // TransformGen::Ortogonal (Matrix.hpp:1021-1039), column-major product
    const float l = P.lo[0], r = P.hi[0], t = P.hi[1], b = P.lo[1], nn = P.lo[2], f = P.hi[2];
    const float xt = -((r + l) / (r - l)), yt = -((t + b) / (t - b)), zt = -((f + nn) / (f - nn));
    const float xs = 2.0f / (r - l), ys = 2.0f / (t - b), zs = 2.0f / (f - nn);
    float q2[3][2];
    float amn[2] = {M<float>::Max, M<float>::Max}, amx[2] = {-M<float>::Max, -M<float>::Max};
    for (int i = 0; i < 3; i++) {
        F3 pt(xs * pos[i].x + xt, ys * pos[i].y + yt, zs * pos[i].z + zt);
        pt = qrotate(rot, pt);
        q2[i][0] = pt.x;
        q2[i][1] = pt.y;
        for (int c = 0; c < 2; c++) {
            amn[c] = std::fmin(amn[c], q2[i][c]);
            amx[c] = std::fmax(amx[c], q2[i][c]);
        }
    }
    const float res = static_cast<float>(P.res);
    const int ri = static_cast<int>(P.res);
    auto clampi = [&](int x) { return std::min(std::max(x, 0), ri); };
    const int x0 = clampi(static_cast<int>(std::floor((0.5f + 0.5f * amn[0]) * res)));
    const int x1 = clampi(static_cast<int>(std::ceil((0.5f + 0.5f * amx[0]) * res)));
    const int y0 = clampi(static_cast<int>(std::floor((0.5f + 0.5f * amn[1]) * res)));
    const int y1 = clampi(static_cast<int>(std::ceil((0.5f + 0.5f * amx[1]) * res)));
    const float half = 1.0f / res;
    const float deltaPix = 2.0f * half;
    F3 pl[3];
    for (int i = 0; i < 3; i++) {
        const float* a = q2[i];
        const float* c = q2[(i + 1) % 3];
        pl[i] = cross(F3(c[0] - a[0], c[1] - a[1], 0.0f), F3(a[0], a[1], 1.0f));
        pl[i].z -= half * std::fabs(pl[i].x) + half * std::fabs(pl[i].y);
    }
    const F3 pc[3] = {cross(pl[0], pl[2]), cross(pl[0], pl[1]), cross(pl[1], pl[2])};
    float c2[3][2];
    for (int i = 0; i < 3; i++) {
        c2[i][0] = pc[i].x / pc[i].z;
        c2[i][1] = pc[i].y / pc[i].z;
    }
    const float ec0[2] = {c2[1][0] - c2[0][0], c2[1][1] - c2[0][1]};
    const float ec1[2] = {c2[2][0] - c2[0][0], c2[2][1] - c2[0][1]};
    const float denomC = 1.0f / (ec0[0] * ec1[1] - ec1[0] * ec0[1]);
    const float e0[2] = {q2[1][0] - q2[0][0], q2[1][1] - q2[0][1]};
    const float e1[2] = {q2[2][0] - q2[0][0], q2[2][1] - q2[0][1]};
    const float denom = 1.0f / (e0[0] * e1[1] - e1[0] * e0[1]);
    uint32_t w = 0;
    for (int y = y0; y < y1; y++)
        for (int x = x0; x < x1; x++) {
            const float px = (static_cast<float>(x) + 0.5f) * deltaPix - 1.0f;
            const float py = (static_cast<float>(y) + 0.5f) * deltaPix - 1.0f;
            const float ec2[2] = {px - c2[0][0], py - c2[0][1]};
            const float bb = (ec2[0] * ec1[1] - ec1[0] * ec2[1]) * denomC;
            const float cc = (ec0[0] * ec2[1] - ec2[0] * ec0[1]) * denomC;
            const float aa = 1.0f - bb - cc;
            if (!(bb >= 0.0f && bb <= 1.0f && cc >= 0.0f && cc <= 1.0f && aa >= 0.0f && aa <= 1.0f))
                continue;
            if (codes) {
                const float e2[2] = {px - q2[0][0], py - q2[0][1]};
                const float ab = (e2[0] * e1[1] - e1[0] * e2[1]) * denom;
                const float ac = (e0[0] * e2[1] - e2[0] * e0[1]) * denom;
                const float aA = 1.0f - ab - ac;
                const F3 vp = (p0 * aA + p1 * ab) + p2 * ac;
                const float vpc[3] = {vp.x, vp.y, vp.z};
                uint32_t vi[3];
                for (int k = 0; k < 3; k++) {
                    float fi = (vpc[k] - P.lo[k]) / (P.hi[k] - P.lo[k]);
                    fi *= res;
                    // the device conversion saturates below zero; ClampSelf(0, res-1)
                    uint32_t q = fi > 0.0f ? static_cast<uint32_t>(fi) : 0u;
                    vi[k] = std::min(q, P.res - 1);
                }
                codes->push_back(morton3d(vi[0], vi[1], vi[2]));
                normals->push_back(packed);
            }
            w++;
        }
    return w;
}

}  // namespace

struct oracle_svo {
    SvoP P{};
    std::vector<uint32_t> triVoxelCounts;
    std::vector<uint64_t> leafCodes;
    std::vector<uint32_t> levelOffsets;
    std::vector<uint64_t> nodes;
    std::vector<uint32_t> leafParents;
    std::vector<uint32_t> leafLight;
    uint32_t voxelCount = 0;
    // voxel records behind each leaf, in sorted order (payload input)
    std::vector<uint32_t> runStart, runVoxel, voxNormal, voxLightKey;
    // radiance-cache payload (VoxelPayload, AnisoSVO.cuh:22-114)
    std::vector<uint32_t> leafNormSpec, nodeNormSpec, leafAvg, nodeAvg, leafBin, nodeBin, leafCnt;
    std::vector<uint64_t> leafIrr;
    // shadow-ray counters (hits, misses per leaf) and binary16 node guiding
    // factors (dShadowRayHitLeaf / dShadowRayMissLeaf / dGuidingFactorNode)
    std::vector<uint32_t> leafShadow;
    std::vector<uint16_t> nodeFactor;
};

namespace {
// __brevll on the host
inline uint64_t brev64(uint64_t x) {
    x = ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
    x = ((x >> 2) & 0x3333333333333333ull) | ((x & 0x3333333333333333ull) << 2);
    x = ((x >> 4) & 0x0F0F0F0F0F0F0F0Full) | ((x & 0x0F0F0F0F0F0F0F0Full) << 4);
    x = ((x >> 8) & 0x00FF00FF00FF00FFull) | ((x & 0x00FF00FF00FF00FFull) << 8);
    x = ((x >> 16) & 0x0000FFFF0000FFFFull) | ((x & 0x0000FFFF0000FFFFull) << 16);
    return (x >> 32) | (x << 32);
}
// AnisoSVOctreeGPU packing (AnisoSVO.cuh:125-151)
inline uint32_t svo_child_mask(uint64_t n) { return uint32_t(n >> 55) & 0xFFu; }
inline uint32_t svo_children_index(uint64_t n) { return uint32_t(n) & 0x7FFFFFFu; }
inline uint32_t svo_child_offset(uint64_t n, uint32_t childId) {
    return uint32_t(__builtin_popcount(svo_child_mask(n) & ((1u << childId) - 1u)));
}
inline void svo_set_children_index(uint64_t& n, uint32_t c) {
    n = (n & ~uint64_t(0x7FFFFFFu)) | (uint64_t(c) & 0x7FFFFFFu);
}
inline void svo_set_parent(uint64_t& n, uint32_t p) {
    n = (n & ~(uint64_t(0xFFFFFFFu) << 27)) | ((uint64_t(p) & 0xFFFFFFFu) << 27);
}
}  // namespace

extern "C" oracle_svo* oracle_svo_build(const float* pos, const uint32_t* idx, const uint32_t* key,
                                        uint32_t T, const float* extent, uint32_t res,
                                        int* status) {
    oracle_svo* o = new oracle_svo();
    o->P = svo_params_of(extent, res);
    const SvoP& P = o->P;
    std::vector<uint64_t> codes;
    std::vector<uint32_t> normals, lights;
    o->triVoxelCounts.resize(T);
    for (uint32_t t = 0; t < T; t++) {
        V3<float> a(pos[3 * idx[3 * t]], pos[3 * idx[3 * t] + 1], pos[3 * idx[3 * t] + 2]);
        V3<float> b(pos[3 * idx[3 * t + 1]], pos[3 * idx[3 * t + 1] + 1], pos[3 * idx[3 * t + 1] + 2]);
        V3<float> c(pos[3 * idx[3 * t + 2]], pos[3 * idx[3 * t + 2] + 1], pos[3 * idx[3 * t + 2] + 2]);
        const size_t before = codes.size();
        o->triVoxelCounts[t] = voxelize_tri(P, a, b, c, &codes, &normals);
        const uint32_t lk = ((key[t] >> 24) == kBatchLight) ? key[t] : 0u;
        lights.resize(codes.size(), 0u);
        for (size_t i = before; i < codes.size(); i++) lights[i] = lk;
    }
    const uint32_t total = uint32_t(codes.size());
    o->voxelCount = total;
    // cub::DeviceRadixSort::SortPairs on bits [0, 3*depth + 1), then RLE
    std::vector<uint32_t> order(total);
    for (uint32_t i = 0; i < total; i++) order[i] = i;
    std::vector<uint64_t> sorted = codes;
    radix_sort<uint64_t>(sorted.data(), order.data(), total, 0, int(3 * P.depth + 1), false);
    for (uint32_t i = 0; i < total; i++)
        if (i == 0 || sorted[i] != sorted[i - 1]) {
            o->leafCodes.push_back(sorted[i]);
            o->leafLight.push_back(0u);
        }
    {  // first light voxel of each run
        size_t u = 0;
        for (uint32_t i = 0; i < total; i++) {
            if (i > 0 && sorted[i] != sorted[i - 1]) u++;
            if (!o->leafLight[u]) o->leafLight[u] = lights[order[i]];
        }
    }
    const uint32_t U = uint32_t(o->leafCodes.size());
    const uint32_t D = P.depth;
    o->runVoxel = order;
    o->voxNormal = normals;
    o->voxLightKey = lights;
    for (uint32_t i = 0; i < total; i++)
        if (i == 0 || sorted[i] != sorted[i - 1]) o->runStart.push_back(i);
    o->runStart.push_back(total);
    // level node counts: KCMarkMortonChanges + reduce, per level
    std::vector<uint32_t> levelCounts(D + 1, 0);
    levelCounts[0] = 1;
    for (uint32_t L = 1; L <= D; L++) {
        uint32_t changes = 0;
        const uint32_t msbStart = 64 - D * 3;
        for (uint32_t j = 0; j + 1 < U; j++) {
            uint64_t a = brev64(o->leafCodes[j]) >> msbStart;
            uint64_t b = brev64(o->leafCodes[j + 1]) >> msbStart;
            a &= (1ull << (L * 3)) - 1;
            b &= (1ull << (L * 3)) - 1;
            changes += (a != b) ? 1u : 0u;
        }
        levelCounts[L] = changes + 1;
    }
    o->levelOffsets.assign(D + 2, 0);
    for (uint32_t L = 0; L <= D; L++) o->levelOffsets[L + 1] = o->levelOffsets[L] + levelCounts[L];
    const uint32_t N = o->levelOffsets[D];
    o->nodes.assign(N, 0x007FFFFFFFFFFFFFull);
    o->leafParents.assign(U, 0xFFFFFFFFu);
    for (uint32_t L = 0; L < D; L++) {
        // KCMarkChild: walk from the root, then set the child bit
        for (uint32_t j = 0; j < U; j++) {
            const uint64_t code = o->leafCodes[j];
            uint32_t shift = (D - 1) * 3;
            uint32_t cur = 0;
            for (uint32_t i = 0; i < L; i++) {
                const uint64_t nd = o->nodes[cur];
                const uint32_t cid = uint32_t(code >> shift) & 7u;
                cur = svo_children_index(nd) + svo_child_offset(nd, cid);
                shift -= 3;
            }
            const uint32_t cid = uint32_t(code >> shift) & 7u;
            o->nodes[cur] |= (uint64_t(1u << cid) << 55);
        }
        // KCExtractChildrenCounts + ExclusiveSum + KCSetChildrenPtrs
        const bool last = (L == D - 1);
        const uint32_t nextOffset = last ? 0 : o->levelOffsets[L + 1];
        uint32_t run = 0;
        for (uint32_t k = 0; k < levelCounts[L]; k++) {
            uint64_t& nd = o->nodes[o->levelOffsets[L] + k];
            const uint32_t cnt = uint32_t(__builtin_popcount(svo_child_mask(nd)));
            svo_set_children_index(nd, nextOffset + run);
            if (last) nd |= (1ull << 63);
            run += cnt;
        }
        if (run != levelCounts[L + 1]) {
            if (status) *status = 2;
            return o;
        }
        // KCSetParentOfChildren / KCSetParentOfLeafChildren
        for (uint32_t k = 0; k < levelCounts[L]; k++) {
            const uint32_t g = o->levelOffsets[L] + k;
            const uint64_t nd = o->nodes[g];
            const uint32_t cnt = uint32_t(__builtin_popcount(svo_child_mask(nd)));
            const uint32_t ci = svo_children_index(nd);
            for (uint32_t i = 0; i < cnt; i++) {
                if (last) o->leafParents[ci + i] = g;
                else svo_set_parent(o->nodes[ci + i], g);
            }
        }
    }
    if (status) *status = 0;
    return o;
}

extern "C" void oracle_svo_destroy(oracle_svo* o) { delete o; }

extern "C" void oracle_svo_sizes(const oracle_svo* o, uint32_t* s) {
    s[0] = o->voxelCount;
    s[1] = uint32_t(o->leafCodes.size());
    s[2] = uint32_t(o->nodes.size());
    s[3] = o->P.depth;
    s[4] = uint32_t(o->levelOffsets.size());
    s[5] = uint32_t(o->triVoxelCounts.size());
}

extern "C" void oracle_svo_get(const oracle_svo* o, uint64_t* nodes, uint32_t* leafParents,
                               uint64_t* leafCodes, uint32_t* leafLights, uint32_t* levelOffsets,
                               uint32_t* triVoxelCounts, float* params) {
    auto cp = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(nodes, o->nodes);
    cp(leafParents, o->leafParents);
    cp(leafCodes, o->leafCodes);
    cp(leafLights, o->leafLight);
    cp(levelOffsets, o->levelOffsets);
    cp(triVoxelCounts, o->triVoxelCounts);
    if (params) {
        for (int c = 0; c < 3; c++) {
            params[c] = o->P.lo[c];
            params[3 + c] = o->P.hi[c];
        }
        params[6] = o->P.leaf;
    }
}

namespace {

struct Tree {
    const oracle_svo* o;
    float level_voxel_size(uint32_t level) const {
        return o->P.leaf * static_cast<float>(1u << (o->P.depth - level));
    }
    // AnisoSVOctreeGPU::Descend (AnisoSVO.cuh:1128-1155)
    bool descend(uint32_t& index, uint64_t code, uint32_t depth) const {
        uint32_t shift = (o->P.depth - 1) * 3;
        uint32_t cur = 0;
        for (uint32_t i = 0; i < depth; i++) {
            const uint64_t node = o->nodes[cur];
            const uint32_t childId = uint32_t(code >> shift) & 7u;
            if (!((node_mask(node) >> childId) & 1u)) return false;
            cur = node_child_index(node) + node_child_offset(node, childId);
            shift -= 3;
        }
        index = cur;
        return true;
    }
    // AnisoSVOctreeGPU::NearestNodeIndex (AnisoSVO.cuh:1171-1242)
    bool nearest(uint32_t& index, F3 p, uint32_t depth) const {
        index = kInvalid;
        const SvoP& P = o->P;
        if (!(p.x >= P.lo[0] && p.x <= P.hi[0] && p.y >= P.lo[1] && p.y <= P.hi[1] &&
              p.z >= P.lo[2] && p.z <= P.hi[2]))
            return false;
        const float vs = level_voxel_size(depth);
        const float li[3] = {(p.x - P.lo[0]) / vs, (p.y - P.lo[1]) / vs, (p.z - P.lo[2]) / vs};
        float fr[3], fl[3];
        uint32_t inc[3];
        for (int c = 0; c < 3; c++) {
            const float ip = std::trunc(li[c]);
            fr[c] = li[c] - ip;
            fl[c] = std::floor(li[c]);
            inc[c] = (fr[c] < 0.5f) ? 0xFFFFFFFFu : 1u;
            fr[c] = 0.5f - std::fabs(fr[c] - 0.5f);
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
            const uint64_t code = morton3d(dense[0] + sh[0] * inc[0], dense[1] + sh[1] * inc[1],
                                           dense[2] + sh[2] * inc[2]);
            if (descend(index, code, depth)) return true;
        }
        return false;
    }
    float read_radiance(F3 coneDir, uint32_t id, bool isLeaf) const {
        if (id == kInvalid) return 0.0f;
        float sd, sp;
        const F3 n = read_normal_spec(isLeaf ? o->leafNormSpec[id] : o->nodeNormSpec[id], sd, sp);
        const bool towards = dot(n, -coneDir) >= 0.0f;
        const uint32_t w = isLeaf ? o->leafAvg[id] : o->nodeAvg[id];
        return h2f(uint16_t(towards ? (w & 0xFFFFu) : (w >> 16)));
    }
    // AnisoSVOctreeGPU::ConeTraceRay (AnisoSVO.cuh:767-1000), bounded loop
    float cone_trace(F3 pos, F3 dir, float tMin, float aperture, uint32_t maxQueryLevelOffset,
                     bool& isLeaf, uint32_t& leafId) const {
        const SvoP& P = o->P;
        const float EPS = 1.0e-5f;
        leafId = kInvalid;
        isLeaf = false;
        if (std::fabs(dir.x) < EPS) dir.x = std::copysign(EPS, dir.x);
        if (std::fabs(dir.y) < EPS) dir.y = std::copysign(EPS, dir.y);
        if (std::fabs(dir.z) < EPS) dir.z = std::copysign(EPS, dir.z);
        const F3 sc(1.0f / (P.hi[0] - P.lo[0]), 1.0f / (P.hi[1] - P.lo[1]), 1.0f / (P.hi[2] - P.lo[2]));
        F3 d = dir * sc;
        F3 p = (pos + F3(-P.lo[0], -P.lo[1], -P.lo[2])) * sc;
        if (!(d.x == d.x && d.y == d.y && d.z == d.z && p.x == p.x && p.y == p.y && p.z == p.z))
            return tMin;
        p.x = (d.x < 0.0f) ? (1.0f - p.x) : p.x;
        p.y = (d.y < 0.0f) ? (1.0f - p.y) : p.y;
        p.z = (d.z < 0.0f) ? (1.0f - p.z) : p.z;
        uint32_t mirror = 0;
        if (d.x < 0.0f) mirror |= 1u;
        if (d.y < 0.0f) mirror |= 2u;
        if (d.z < 0.0f) mirror |= 4u;
        const F3 dc(1.0f / std::fabs(d.x), 1.0f / std::fabs(d.y), 1.0f / std::fabs(d.z));
        const F3 pb = p * dc;
        {
            const F3 t0 = -pb;
            const float tSvo = std::fmax(std::fmax(t0.x, t0.y), t0.z);
            if (!(t0.x < tMin && t0.y < tMin && t0.z < tMin)) tMin = next_up(tSvo);
        }
        auto neg_exp2i = [](uint32_t q) { return (q == 0) ? 1.0f : bitsf((127u - q) << 23); };
        uint64_t stack = 0;
        uint32_t depthBits = 0, nodeId = 0;
        F3 corner(0.0f, 0.0f, 0.0f);
        bool emptyNode = false;
        for (uint32_t step = 0; nodeId != kSvoInvalidParent; step++) {
            if (step == (1u << 16)) {
                leafId = kInvalid;
                isLeaf = false;
                break;
            }
            const float childSpan = neg_exp2i(depthBits + 1), curSpan = neg_exp2i(depthBits);
            const F3 center = corner + F3(childSpan, childSpan, childSpan);
            const F3 topRight = corner + F3(curSpan, curSpan, curSpan);
            const F3 tm = topRight * dc - pb;
            const float tMax = std::fmin(std::fmin(tm.x, tm.y), tm.z);
            if (emptyNode) {
                tMin = next_up(tMax);
                const uint32_t b = uint32_t(stack & 7u);
                corner = corner - F3((b & 1u) ? curSpan : 0.0f, (b & 2u) ? curSpan : 0.0f,
                                     (b & 4u) ? curSpan : 0.0f);
                stack >>= 3;
                depthBits -= 1;
                emptyNode = false;
                continue;
            }
            const uint64_t node = o->nodes[nodeId];
            if (tMax < tMin) {
                const uint32_t b = uint32_t(stack & 7u);
                corner = corner - F3((b & 1u) ? curSpan : 0.0f, (b & 2u) ? curSpan : 0.0f,
                                     (b & 4u) ? curSpan : 0.0f);
                stack >>= 3;
                depthBits -= 1;
                nodeId = node_parent(node);
                emptyNode = false;
            } else {
                const F3 tc = center * dc - pb;
                uint32_t childId = 0;
                if (tc.x < tMin) childId |= 1u;
                if (tc.y < tMin) childId |= 2u;
                if (tc.z < tMin) childId |= 4u;
                const uint32_t mir = childId ^ mirror;
                const bool has = (node_mask(node) >> mir) & 1u;
                if (has) {
                    nodeId = node_child_index(node) + node_child_offset(node, mir);
                    const uint32_t level = depthBits + 1;
                    const float area = tMin * tMin * aperture;
                    const float diam2 = 4.0f * (area * kInvPiF);
                    const float vs = level_voxel_size(level);
                    bool term = diam2 > vs * vs;
                    const bool childLeaf = node_children_leaf(node);
                    term |= (P.depth - level) <= maxQueryLevelOffset;
                    if (childLeaf || term) {
                        isLeaf = childLeaf;
                        leafId = nodeId;
                        break;
                    }
                }
                emptyNode = !has;
                corner = corner + F3((childId & 1u) ? childSpan : 0.0f, (childId & 2u) ? childSpan : 0.0f,
                                     (childId & 4u) ? childSpan : 0.0f);
                stack = (stack << 3) | childId;
                depthBits += 1;
            }
        }
        return tMin;
    }
    uint32_t marked_bin(uint32_t leaf, bool& isLeaf) const {
        isLeaf = true;
        uint32_t bin = o->leafBin[leaf];
        uint32_t parent = o->leafParents[leaf];
        uint32_t node = leaf;
        while (parent != kSvoInvalidParent && !(bin & kBinMark)) {
            node = parent;
            bin = o->nodeBin[parent];
            parent = node_parent(o->nodes[parent]);
            isLeaf = false;
        }
        return node;
    }
};

// Ray binning of one wavefront (WFPGTracer.cu:488-628): KCInitializeSVOBins
// (WFPGTracerKC.cuh:965-1018; the leaf of each hit, neighbours searched),
// leaf ray counts (sort + RLE + KCWriteLeafRayAmounts), KCCollapseRayCountsLeaf
// / KCCollapseRayCounts bottom-up to minLevel (AnisoSVO.cu:265-350,
// 1485-1528) and KCCheckReducedSVOBins (WFPGTracerKC.cuh:1045-1066).  hit(i, p)
// gives ray i's hit position or false for a ray the binning skips.  binKey[i]:
// kBinInvalid, leaf | kBinLeaf, or the node index of the marked bin.
template <class HitPos>
void bin_rays(oracle_svo* svo, uint32_t n, uint32_t minLevel, uint32_t binRayCount, HitPos hit,
              uint32_t* binKey) {
    Tree tree{svo};
    const uint32_t D = svo->P.depth;
    std::fill(svo->leafBin.begin(), svo->leafBin.end(), 0u);
    std::fill(svo->nodeBin.begin(), svo->nodeBin.end(), 0u);
    for (uint32_t i = 0; i < n; i++) {
        binKey[i] = kBinInvalid;
        F3 p;
        if (!hit(i, p)) continue;
        uint32_t leaf;
        if (tree.nearest(leaf, p, D)) {
            binKey[i] = leaf | kBinLeaf;
            svo->leafBin[leaf] += 1u;
        }
    }
    for (size_t l = 0; l < svo->leafBin.size(); l++) {
        if (D == minLevel) { svo->leafBin[l] |= kBinMark; continue; }
        const uint32_t cnt = svo->leafBin[l] & ~kBinMark;
        if (cnt == 0) continue;
        if (cnt < binRayCount) svo->nodeBin[svo->leafParents[l]] += cnt;
        else svo->leafBin[l] |= kBinMark;
    }
    for (int L = int(D) - 1; L >= int(minLevel); L--) {
        for (uint32_t k = svo->levelOffsets[L]; k < svo->levelOffsets[L + 1]; k++) {
            if (uint32_t(L) == minLevel) { svo->nodeBin[k] |= kBinMark; continue; }
            const uint32_t cnt = svo->nodeBin[k] & ~kBinMark;
            if (cnt < binRayCount) svo->nodeBin[node_parent(svo->nodes[k])] += cnt;
            else svo->nodeBin[k] |= kBinMark;
        }
    }
    for (uint32_t i = 0; i < n; i++) {
        if (binKey[i] == kBinInvalid) continue;
        bool isLeaf;
        const uint32_t node = tree.marked_bin(binKey[i] & ~kBinLeaf, isLeaf);
        if (!isLeaf) binKey[i] = node;
    }
}

// AnisoSVOctreeGPU::DepositRadiance (AnisoSVO.cuh:1080-1098) with
// VoxelPayload::WriteLeafRadiance (:490-537): the leaf of the vertex (with the
// neighbour search), the side its normal puts wo on, one sample of the
// luminance there (2^-24 fixed point).  False when no leaf is found.
// With hits / misses it is also DepositNEEHitMiss (AnisoSVO.cuh:1101-1115)
// at the same leaf.
bool deposit_leaf(oracle_svo* svo, const Tree& tree, F3 pos, F3 wo, float luminance,
                  uint32_t hits = 0, uint32_t misses = 0) {
    uint32_t leaf;
    if (!tree.nearest(leaf, pos, svo->P.depth)) return false;
    svo->leafShadow[2 * leaf] += hits;
    svo->leafShadow[2 * leaf + 1] += misses;
    float sd, spc;
    const F3 n = read_normal_spec(svo->leafNormSpec[leaf], sd, spc);
    const float NdL = dot(n, wo);
    int side;
    if (NdL >= 0.0f) side = 0;
    else if (NdL < 0.0f) side = 1;
    else return true;
    svo->leafIrr[2 * leaf + side] += to_fixed(luminance);
    svo->leafCnt[2 * leaf + side] += 1u;
    return true;
}

// KCReduceVoxelPayload (AnisoSVOKC.cuh:8-320), one voxel at a time with
// sequential sums, then KCAverageNormals bottom-up (AnisoSVO.cu:428-528)
void payload_init(oracle_svo* o, const float* lightRad, uint32_t omit) {
    const uint32_t U = uint32_t(o->leafCodes.size()), N = uint32_t(o->nodes.size());
    const uint32_t D = o->P.depth;
    o->leafNormSpec.assign(U, 0);
    o->leafIrr.assign(2 * size_t(U), 0);
    o->leafCnt.assign(2 * size_t(U), 0);
    o->leafAvg.assign(U, 0);
    o->nodeAvg.assign(N, 0);
    o->nodeNormSpec.assign(N, 0);
    o->leafBin.assign(U, 0);
    o->nodeBin.assign(N, 0);
    o->leafShadow.assign(2 * size_t(U), 0);
    o->nodeFactor.assign(N, 0x7FFFu);
    for (uint32_t j = 0; j < U; j++) {
        const uint32_t b = o->runStart[j], e = o->runStart[j + 1], dup = e - b;
        const F3 n0 = unpack_normal16(o->voxNormal[o->runVoxel[b]]);
        F3 m0 = n0, m1 = -n0;
        uint32_t c0 = 0, c1 = 0;
        for (int it = 0; it < 4; it++) {
            m0 = normalize(m0);
            m1 = normalize(m1);
            F3 a0(0.0f, 0.0f, 0.0f), a1(0.0f, 0.0f, 0.0f);
            uint32_t k0 = 0, k1 = 0;
            for (uint32_t i = b; i < e; i++) {
                const F3 n = unpack_normal16(o->voxNormal[o->runVoxel[i]]);
                if (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f) continue;
                const float d0 = 1.0f - dot(m0, n), d1 = 1.0f - dot(m1, n);
                if (d0 >= d1) { a0 = a0 + n; k0++; } else { a1 = a1 + n; k1++; }
            }
            m0 = a0;
            m1 = a1;
            c0 = k0;
            c1 = k1;
        }
        F3 mean = (c0 >= c1) ? m0 * (1.0f / static_cast<float>(c0)) : m1 * (1.0f / static_cast<float>(c1));
        float lum = 0.0f;
        const uint32_t passes = (dup + 63u) / 64u;
        for (uint32_t pass = 0; pass < passes; pass++) {
            mean = normalize(mean);
            const uint32_t pe = std::min(e, b + (pass + 1) * 64u);
            for (uint32_t i = b + pass * 64u; i < pe; i++) {
                const uint32_t key = o->voxLightKey[o->runVoxel[i]];
                if (!key) continue;
                const float* r = lightRad + 3 * (key & 0xFFFFFFu);
                lum = lum + (0.2120f * r[0] + 0.7150f * r[1] + 0.0722f * r[2]);
            }
        }
        if (lum != 0.0f) {
            lum /= static_cast<float>(dup);
            lum *= 10000.0f;
            if (omit) lum = 0.0f;
            o->leafIrr[2 * j] = o->leafIrr[2 * j + 1] = to_fixed(lum);
            o->leafCnt[2 * j] = o->leafCnt[2 * j + 1] = 10000u;
        }
        o->leafNormSpec[j] = write_normal_spec(mean, 0.0f);
    }
    for (int L = int(D) - 1; L >= 0; L--) {
        const bool childLeaf = (L == int(D) - 1);
        for (uint32_t k = o->levelOffsets[L]; k < o->levelOffsets[L + 1]; k++) {
            const uint64_t node = o->nodes[k];
            const uint32_t cnt = uint32_t(__builtin_popcount(node_mask(node)));
            const uint32_t ci = node_child_index(node);
            F3 nb[8];
            float avgSpec = 0.0f;
            for (uint32_t i = 0; i < cnt; i++) {
                float sd, sp;
                const F3 n = read_normal_spec(childLeaf ? o->leafNormSpec[ci + i] : o->nodeNormSpec[ci + i],
                                              sd, sp);
                const float len = 1.0f / (1.0f + sd);
                nb[i] = n * len;
                avgSpec += sp;
            }
            avgSpec *= 1.0f / static_cast<float>(cnt);
            F3 mean[2][2];
            uint32_t counts[2][2] = {{0, 0}, {0, 0}};
            mean[0][0] = nb[0];
            mean[0][1] = -nb[0];
            mean[1][0] = mean[1][1] = F3(0.0f, 0.0f, 0.0f);
            for (int pass = 0; pass < 4; pass++) {
                const int rd = pass % 2, wr = rd ? 0 : 1;
                for (uint32_t i = 0; i < cnt; i++) {
                    const F3 n = nb[i];
                    if (n.x == 0.0f && n.y == 0.0f && n.z == 0.0f) continue;
                    const float d0 = 1.0f - dot(mean[rd][0], n), d1 = 1.0f - dot(mean[rd][1], n);
                    const int up = (d0 >= d1) ? 0 : 1;
                    mean[wr][up] = mean[wr][up] + n;
                    counts[wr][up] += 1;
                }
                mean[rd][0] = mean[rd][1] = F3(0.0f, 0.0f, 0.0f);
                counts[rd][0] = counts[rd][1] = 0;
            }
            const int idx = (counts[0][0] >= counts[0][1]) ? 0 : 1;
            const F3 m = mean[0][idx] * (1.0f / static_cast<float>(counts[0][idx]));
            o->nodeNormSpec[k] = write_normal_spec(m, avgSpec);
        }
    }
}

// NormalizeAndFilterRadiance (AnisoSVO.cu:352-428,1415-1484)
void normalize_filter(oracle_svo* o) {
    const uint32_t U = uint32_t(o->leafCodes.size());
    const uint32_t D = o->P.depth;
    for (uint32_t l = 0; l < U; l++) {
        uint32_t w = 0;
        for (int s = 0; s < 2; s++) {
            const uint32_t c = o->leafCnt[2 * l + s];
            float avg = 0.0f;
            if (c) avg = static_cast<float>(static_cast<double>(o->leafIrr[2 * l + s]) / kFixScale /
                                            static_cast<double>(c));
            avg = std::fmin(avg, 65504.0f);
            w |= uint32_t(f2h(avg)) << (16 * s);
        }
        o->leafAvg[l] = w;
    }
    for (int L = int(D) - 1; L >= 0; L--) {
        const bool childLeaf = (L == int(D) - 1);
        for (uint32_t k = o->levelOffsets[L]; k < o->levelOffsets[L + 1]; k++) {
            const uint64_t node = o->nodes[k];
            const uint32_t cnt = uint32_t(__builtin_popcount(node_mask(node))), ci = node_child_index(node);
            float sd, sp;
            const F3 n = read_normal_spec(o->nodeNormSpec[k], sd, sp);
            float sum[2] = {0.0f, 0.0f};
            uint32_t valid[2] = {0, 0};
            // guiding factor (AnisoSVO.cu:586-613): mean of the children's
            // factors that are not NaN; a leaf's is misses / (hits + misses)
            // (VoxelPayload::ReadGuidingFactor, AnisoSVO.cuh:477-488)
            float factorSum = 0.0f;
            uint32_t factorValid = 0;
            for (uint32_t i = 0; i < cnt; i++) {
                const uint32_t c = ci + i;
                const float factor =
                    childLeaf ? static_cast<float>(o->leafShadow[2 * c + 1]) /
                                    (static_cast<float>(o->leafShadow[2 * c]) +
                                     static_cast<float>(o->leafShadow[2 * c + 1]))
                              : h2f(o->nodeFactor[c]);
                if (!std::isnan(factor)) {
                    factorValid++;
                    factorSum += factor;
                }
                const uint32_t irr = childLeaf ? o->leafAvg[c] : o->nodeAvg[c];
                const F3 cn = read_normal_spec(childLeaf ? o->leafNormSpec[c] : o->nodeNormSpec[c], sd, sp);
                const bool swap = dot(cn, n) < 0.0f;
                for (int j = 0; j < 2; j++) {
                    const int rdx = swap ? ((j + 1) % 2) : j;
                    const uint16_t h = uint16_t(irr >> (16 * rdx));
                    if (h != kHalfMax) {
                        valid[j]++;
                        sum[j] += h2f(h);
                    }
                }
            }
            uint32_t w = 0;
            for (int j = 0; j < 2; j++) {
                const uint16_t h = valid[j] ? f2h(std::fmin(sum[j] / static_cast<float>(valid[j]), 65504.0f))
                                            : kHalfMax;
                w |= uint32_t(h) << (16 * j);
            }
            o->nodeAvg[k] = w;
            // no child with data: 0 / 0, the binary16 NaN 0x7FFF
            o->nodeFactor[k] = factorValid ? f2h(factorSum / static_cast<float>(factorValid)) : 0x7FFFu;
        }
    }
    for (uint32_t L = 1; L <= D; L++) {
        const bool leaf = (L == D);
        const uint32_t b = leaf ? 0u : o->levelOffsets[L];
        const uint32_t e = leaf ? U : o->levelOffsets[L + 1];
        for (uint32_t k = b; k < e; k++) {
            const uint32_t parent = leaf ? o->leafParents[k] : node_parent(o->nodes[k]);
            uint32_t& w = leaf ? o->leafAvg[k] : o->nodeAvg[k];
            const uint32_t pw = o->nodeAvg[parent];
            uint32_t lo = w & 0xFFFFu, hi = w >> 16;
            if (lo == kHalfMax) lo = pw & 0xFFFFu;
            if (hi == kHalfMax) hi = pw >> 16;
            w = lo | (hi << 16);
        }
    }
}

// ---- BxDF dispatch by batch -------------------------------------------
bool mat_specular(const oracle_scene* s, uint32_t batch, uint32_t id) {
    if (batch == kBatchLambert || batch == kBatchLambertC) return false;
    if (batch == kBatchMetal) return (1.0f - s->metal_params[10 * id + 9]) >= 0.99f;
    if (batch == kBatchUnreal) return (1.0f - s->unreal_params[6 * id + 3]) >= 0.99f;
    return true;
}
F3 mat_eval(const oracle_scene* s, uint32_t batch, uint32_t id, F3 wo, F3 wi, const Surface<float>& sf) {
    if (batch == kBatchLambert) {
        const float* a = s->lambert_albedo + 3 * id;
        return lambert_eval(F3(a[0], a[1], a[2]), wo, sf);
    }
    if (batch == kBatchLambertC) {
        const float* a = s->lambertc_albedo + 3 * id;
        return lambertc_eval(F3(a[0], a[1], a[2]), wo, sf);
    }
    if (batch == kBatchUnreal) return unreal_eval(unreal_params<float>(s->unreal_params + 6 * id), wo, wi, sf);
    if (batch == kBatchMetal) return metal_eval(metal_params<float>(s->metal_params + 10 * id), wo, wi, sf);
    return F3(0.0f, 0.0f, 0.0f);
}
float mat_pdf(const oracle_scene* s, uint32_t batch, uint32_t id, F3 wo, F3 wi, const Surface<float>& sf) {
    if (batch == kBatchLambert || batch == kBatchLambertC) return lambert_pdf(wo, sf);
    if (batch == kBatchUnreal) return unreal_pdf(unreal_params<float>(s->unreal_params + 6 * id), wo, wi, sf);
    if (batch == kBatchMetal) return metal_pdf(metal_params<float>(s->metal_params + 10 * id), wo, wi, sf);
    return 0.0f;
}
BSample<float> mat_sample(const oracle_scene* s, uint32_t batch, uint32_t id, F3 wi,
                          const Surface<float>& sf, uint32_t medium, float u0, float u1, float u2) {
    if (batch == kBatchLambert) {
        const float* a = s->lambert_albedo + 3 * id;
        return lambert_sample(F3(a[0], a[1], a[2]), sf, u0, u1, medium);
    }
    if (batch == kBatchLambertC) {
        const float* a = s->lambertc_albedo + 3 * id;
        return lambertc_sample(F3(a[0], a[1], a[2]), sf, u0, u1, medium);
    }
    if (batch == kBatchUnreal)
        return unreal_sample(unreal_params<float>(s->unreal_params + 6 * id), wi, sf, u2, u0, u1, medium);
    if (batch == kBatchMetal)
        return metal_sample(metal_params<float>(s->metal_params + 10 * id), wi, sf, u0, u1, medium);
    const float* a = s->refract_albedo + 3 * id;
    return refract_sample(F3(a[0], a[1], a[2]), s->refract_medium[id], s, wi, sf, medium, u0);
}

// BxDFProjFunc of KCGenAndSampleDistributionProduct
F3 bxdf_proj(int cx, int cy, F3 nrm) {
    const float rc = 1.0f / 8.0f;
    const float s = (static_cast<float>(cx) + 0.5f) * rc, t = (static_cast<float>(cy) + 0.5f) * rc;
    F3 dir = octa_to_dir_yup(s, t);
    const F3 right = normalize(cross(dir, nrm));
    float angle = 4.0f * kPiF / 64.0f;
    angle *= 0.5f;
    float sn, cs;
    pm_sincos(angle, sn, cs);
    const FQ q{cs, right.x * sn, right.y * sn, right.z * sn};
    return qrotate(q, dir);
}
// inclusive Kogge-Stone scan over 8 lanes (as the warp computes it)
void scan8(const float in[8], float out[8]) {
    float x[8];
    for (int i = 0; i < 8; i++) x[i] = in[i];
    for (int off = 1; off < 8; off <<= 1) {
        float y[8];
        for (int i = 0; i < 8; i++) y[i] = x[i];
        for (int i = 0; i < 8; i++)
            if (i >= off) x[i] = y[i - off] + y[i];
    }
    for (int i = 0; i < 8; i++) out[i] = x[i];
}

// ProductSampler's constructor (ProductSampler.cuh:160-215): the mean and
// the maximum of each of the 8x8 product cells' DPP x DPP texels.  The mean
// adds the texels as the sampler's cub warp reduction does: the cell's
// texels in row-major order, in chunks of at most 32 (a logical warp of
// min(32, max(2, DPP^2)) lanes, lanes past DPP^2 holding 0), each chunk
// summed as a pairwise tree (lane pairs at distance 1, 2, 4, ...), the chunk
// sums added in order to 0.
template <int X>
void product_cells(const float* field, float small[64], float normc[64]) {
    constexpr int DPP = X / 8, N = DPP * DPP;
    constexpr int W = N >= 32 ? 32 : (N < 2 ? 2 : N);
    constexpr int IT = N >= 32 ? N / 32 : 1;
    for (int c = 0; c < 64; c++) {
        const int cx = c & 7, cy = c >> 3;
        float total = 0.0f, mx = 0.0f;
        for (int it = 0; it < IT; it++) {
            float v[W];
            for (int l = 0; l < W; l++) {
                const int li = l + it * 32;
                v[l] = (li < N) ? field[(cy * DPP + li / DPP) * X + cx * DPP + li % DPP] : 0.0f;
                mx = std::fmax(mx, v[l]);
            }
            for (int off = 1; off < W; off <<= 1)
                for (int l = 0; l + off < W; l += 2 * off) v[l] = v[l] + v[l + off];
            total += v[0];
        }
        small[c] = total / static_cast<float>(N);
        normc[c] = mx;
    }
}

// GeneratePDFAndCDF (ProductSampler.cuh:217-368): rows of the product of
// the cell means and the BxDF's gray values (floored at VeryLargeEpsilon),
// row and marginal CDFs by 8-wide inclusive scans.
struct ProductCdf {
    float pdfX[64], cdfX[64], pdfY[8], cdfY[8];
};

void product_build(const float gray[64], const float small[64], ProductCdf& P) {
    float rowTot[8];
    for (int row = 0; row < 8; row++) {
        float prod[8], incl[8];
        for (int cx = 0; cx < 8; cx++)
            prod[cx] = std::fmax(1.0e-3f, gray[row * 8 + cx] * small[row * 8 + cx]);
        scan8(prod, incl);
        const float rowTotal = incl[7];
        const float rcp = 1.0f / rowTotal;
        for (int cx = 0; cx < 8; cx++) {
            P.cdfX[row * 8 + cx] = incl[cx] * rcp;
            P.pdfX[row * 8 + cx] = prod[cx] * 8.0f * rcp;
        }
        rowTot[row] = rowTotal;
    }
    float incl[8];
    scan8(rowTot, incl);
    const float rcp = 1.0f / incl[7];
    for (int l = 0; l < 8; l++) {
        P.cdfY[l] = incl[l] * rcp;
        P.pdfY[l] = rowTot[l] * (8.0f * rcp);
    }
}

// ProductSampler::Pdf (ProductSampler.cuh:508-540), indices clamped to the
// map (the reference reads past it for uv = 1).
template <int X>
float product_pdf(const float* field, const float small[64], const ProductCdf& P, float u,
                  float v) {
    constexpr int DPP = X / 8;
    const float dppF = static_cast<float>(DPP);
    const float ex = u * 8.0f, ey = v * 8.0f;
    const float ox = std::floor(ex), oy = std::floor(ey);
    const float ix = (ex - ox) * dppF, iy = (ey - oy) * dppF;
    const int ocx = std::min(std::max(f2i_sat(ox), 0), 7), ocy = std::min(std::max(f2i_sat(oy), 0), 7);
    int gx = ocx * DPP + f2i_sat(std::floor(ix)), gy = ocy * DPP + f2i_sat(std::floor(iy));
    gx = std::min(std::max(gx, 0), X - 1);
    gy = std::min(std::max(gy, 0), X - 1);
    const int cell = ocy * 8 + ocx;
    const float inner = field[gy * X + gx] / small[cell];
    return P.pdfX[cell] * P.pdfY[ocy] * inner;
}

// ProductSampler::Sample (ProductSampler.cuh:370-470): the row and the
// column by CDF search (first entry not below the draw, clamped to the last
// cell), then rejection sampling inside the cell: in each of 24 rounds
// every lane draws (u, v, acceptance) and the lowest accepting lane wins;
// if none does, lane 0's last draw is taken with an inner pdf of 1.
// draw(round, lane, u, v, a) supplies the numbers.  Returns the map
// coordinates and the product pdf (before the sphere's 1/(4 pi)).
template <int X, class Draw>
void product_sample(const float* field, const float small[64], const float normc[64],
                    const ProductCdf& P, float xi0, float xi1, Draw&& draw, float& ss, float& tt,
                    float& pdfS, int* rowOut = nullptr, int* colOut = nullptr) {
    constexpr int DPP = X / 8;
    const float dppF = static_cast<float>(DPP);
    int rowId = 8;
    for (int l = 0; l < 8; l++)
        if (!(xi0 > P.cdfY[l])) {
            rowId = l;
            break;
        }
    rowId = std::min(rowId, 7);
    int colId = 8;
    for (int l = 0; l < 8; l++)
        if (!(xi1 > P.cdfX[rowId * 8 + l])) {
            colId = l;
            break;
        }
    colId = std::min(colId, 7);
    if (rowOut) *rowOut = rowId;
    if (colOut) *colOut = colId;
    const int cell = rowId * 8 + colId;
    float u = 0.0f, v = 0.0f, tex = 0.0f, u0 = 0.0f, v0 = 0.0f, tex0 = 0.0f;
    bool lucky = false;
    for (int round = 0; round < 24 && !lucky; round++) {
        for (uint32_t lane = 0; lane < 32; lane++) {
            float du, dv, da;
            draw(round, lane, du, dv, da);
            const int ix = f2i_sat(du * dppF), iy = f2i_sat(dv * dppF);
            const float tx = field[(rowId * DPP + iy) * X + colId * DPP + ix];
            if (lane == 0) {
                u0 = du;
                v0 = dv;
                tex0 = tx;
            }
            if (da <= tx / normc[cell]) {
                u = du;
                v = dv;
                tex = tx;
                lucky = true;
                break;
            }
        }
    }
    if (!lucky) {
        u = u0;
        v = v0;
        tex = tex0;
    }
    const float pdfInner = lucky ? tex / small[cell] : 1.0f;
    pdfS = P.pdfY[rowId] * P.pdfX[cell] * pdfInner;
    const float rcpX = 1.0f / static_cast<float>(X);
    ss = (static_cast<float>(colId) * dppF + u * dppF) * rcpX;
    tt = (static_cast<float>(rowId) * dppF + v * dppF) * rcpX;
}

// One-sample MIS of the drawn direction (SampleMIS, ProductSampler.cuh:
// 640-650): pdfSampled * ratio / BalanceHeuristic.
inline float mis_pdf(float pdfSampled, float ratio, float pdfOther) {
    const float w0 = ratio * pdfSampled, w1 = (1.0f - ratio) * pdfOther;
    const float pdf = pdfSampled * ratio / (w0 / (w0 + w1));
    return (pdfSampled == 0.0f) ? 0.0f : pdf;
}

}  // namespace

extern "C" void oracle_svo_payload_init(oracle_svo* o, const float* light_rad, uint32_t omit) {
    payload_init(o, light_rad, omit);
    normalize_filter(o);
}

extern "C" int64_t oracle_voxelize(const float* pos, const uint32_t* idx, uint32_t T,
                                   const float* extent, uint32_t res, uint64_t* counts,
                                   uint64_t* codes, uint32_t* normals, uint64_t capacity) {
    const SvoP P = svo_params_of(extent, res);
    std::vector<uint64_t> c;
    std::vector<uint32_t> nr;
    for (uint32_t t = 0; t < T; t++) {
        V3<float> a(pos[3 * idx[3 * t]], pos[3 * idx[3 * t] + 1], pos[3 * idx[3 * t] + 2]);
        V3<float> b(pos[3 * idx[3 * t + 1]], pos[3 * idx[3 * t + 1] + 1], pos[3 * idx[3 * t + 1] + 2]);
        V3<float> d(pos[3 * idx[3 * t + 2]], pos[3 * idx[3 * t + 2] + 1], pos[3 * idx[3 * t + 2] + 2]);
        counts[t] = voxelize_tri(P, a, b, d, codes ? &c : nullptr, codes ? &nr : nullptr);
    }
    uint64_t total = 0;
    for (uint32_t t = 0; t < T; t++) total += counts[t];
    if (!codes) return int64_t(total);
    if (total > capacity) return -1;
    std::copy(c.begin(), c.end(), codes);
    std::copy(nr.begin(), nr.end(), normals);
    return int64_t(total);
}

extern "C" void oracle_svo_bin_rays(oracle_svo* o, const float* org, const float* dir,
                                    const float* t, const uint8_t* valid, uint32_t n,
                                    uint32_t minLevel, uint32_t binRayCount, uint32_t* binOut) {
    bin_rays(o, n, std::min(minLevel, o->P.depth), binRayCount,
             [&](uint32_t i, F3& p) {
                 if (!valid[i]) return false;
                 p = F3(org[3 * i] + t[i] * dir[3 * i], org[3 * i + 1] + t[i] * dir[3 * i + 1],
                        org[3 * i + 2] + t[i] * dir[3 * i + 2]);
                 return true;
             },
             binOut);
}

extern "C" void oracle_svo_set_radiance(oracle_svo* o, const uint64_t* leafIrr,
                                        const uint32_t* leafCnt) {
    std::copy(leafIrr, leafIrr + o->leafIrr.size(), o->leafIrr.begin());
    std::copy(leafCnt, leafCnt + o->leafCnt.size(), o->leafCnt.begin());
}

extern "C" void oracle_svo_normalize(oracle_svo* o) { normalize_filter(o); }

// DepositNEEHitMiss of n vertices over zeroed counters: is_hit[i] picks the
// hit or the miss counter of the vertex's leaf.
extern "C" void oracle_svo_deposit_nee(oracle_svo* o, const float* pos, const uint8_t* isHit,
                                       uint32_t n) {
    std::fill(o->leafShadow.begin(), o->leafShadow.end(), 0u);
    Tree tree{o};
    for (uint32_t i = 0; i < n; i++) {
        uint32_t leaf;
        if (!tree.nearest(leaf, F3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), o->P.depth)) continue;
        o->leafShadow[2 * leaf + (isHit[i] ? 0 : 1)] += 1u;
    }
}

// Shadow-ray counters (2 per leaf: hits, misses) in; NULL leaves them.
extern "C" void oracle_svo_set_shadow(oracle_svo* o, const uint32_t* leafShadow) {
    if (leafShadow) std::copy(leafShadow, leafShadow + o->leafShadow.size(), o->leafShadow.begin());
}

// Shadow-ray counters and binary16 node guiding factors out; NULL skips.
extern "C" void oracle_svo_guiding_get(const oracle_svo* o, uint32_t* leafShadow,
                                       uint16_t* nodeFactor) {
    if (leafShadow) std::memcpy(leafShadow, o->leafShadow.data(), o->leafShadow.size() * 4);
    if (nodeFactor) std::memcpy(nodeFactor, o->nodeFactor.data(), o->nodeFactor.size() * 2);
}

extern "C" void oracle_svo_deposit(oracle_svo* o, const float* pos, const float* wo,
                                   const float* lum, uint32_t n) {
    std::fill(o->leafIrr.begin(), o->leafIrr.end(), 0ull);
    std::fill(o->leafCnt.begin(), o->leafCnt.end(), 0u);
    Tree tree{o};
    for (uint32_t i = 0; i < n; i++)
        deposit_leaf(o, tree, F3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]),
                     F3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), lum[i]);
}

extern "C" void oracle_svo_cone_trace(const oracle_svo* o, const float* org, const float* dir,
                                      const float* tmin, const float* aperture,
                                      uint32_t maxQueryOffset, uint32_t n, float* tOut,
                                      uint32_t* idOut, uint8_t* leafOut, float* radOut) {
    Tree tree{o};
    for (uint32_t i = 0; i < n; i++) {
        bool isLeaf = false;
        uint32_t id = kInvalid;
        const F3 d(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        tOut[i] = tree.cone_trace(F3(org[3 * i], org[3 * i + 1], org[3 * i + 2]), d, tmin[i],
                                  aperture[i], maxQueryOffset, isLeaf, id);
        idOut[i] = id;
        leafOut[i] = isLeaf ? 1 : 0;
        radOut[i] = tree.read_radiance(d, id, isLeaf);
    }
}

extern "C" void oracle_svo_payload_get(const oracle_svo* o, uint32_t* leafNormSpec,
                                       uint32_t* nodeNormSpec, uint64_t* leafIrr, uint32_t* leafCnt,
                                       uint32_t* leafAvg, uint32_t* nodeAvg) {
    auto cp = [](auto* dst, const auto& v) {
        if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    cp(leafNormSpec, o->leafNormSpec);
    cp(nodeNormSpec, o->nodeNormSpec);
    cp(leafIrr, o->leafIrr);
    cp(leafCnt, o->leafCnt);
    cp(leafAvg, o->leafAvg);
    cp(nodeAvg, o->nodeAvg);
}

namespace {

struct WRay {
    PRay<float> r;
    uint32_t g0 = 0, g1 = 0x7E00u;  // guide words of this step (invalid by default)
    bool guided = false;
    // hit record
    uint32_t key = 0, prim = kInvalid;
    float t = 0.0f, b0 = 0.0f, b1 = 0.0f;
};

// The non-product sampler of one bin (KCGenAndSampleDistribution,
// WFPGTracerKC.cuh:1356-1559): a 2D piecewise-constant distribution over
// the filtered X x X field, one ray at a time.  Row prefix sums run left to
// right, the marginal over rows bottom to top, both in float; a sample
// takes the first row whose prefix exceeds xi0 * total, then the first cell
// of that row whose prefix exceeds xi1 * rowTotal, with the offset inside
// the cell from the remainder.  Density over the unit square: f * X^2 /
// total; over the sphere (equal-area map): that / (4 pi).
template <int X>
void guide_bin_pwc(const oracle_scene* s, const oracle_options* opt,
                   const oracle_wfpg_options* w, uint32_t depthTag, const std::vector<float>& field,
                   const std::vector<uint32_t>& rays, std::vector<WRay>& wave) {
    const uint32_t frame = opt->frame;
    std::vector<float> rowPre(X * X);
    float marg[X];
    for (int y = 0; y < X; y++) {
        float acc = 0.0f;
        for (int x = 0; x < X; x++) {
            acc += field[y * X + x];
            rowPre[y * X + x] = acc;
        }
    }
    {
        float acc = 0.0f;
        for (int y = 0; y < X; y++) {
            acc += rowPre[y * X + X - 1];
            marg[y] = acc;
        }
    }
    const float total = marg[X - 1];
    const float scale = static_cast<float>(X * X) / total;
    const float kInv4Pi = 0.25f * kInvPiF;
    const float below1 = 0x1.fffffep-1f;
    auto pdf_at = [&](float u, float v) {
        int ix = f2i_sat(std::floor(u * static_cast<float>(X)));
        int iy = f2i_sat(std::floor(v * static_cast<float>(X)));
        ix = std::min(std::max(ix, 0), X - 1);
        iy = std::min(std::max(iy, 0), X - 1);
        return field[iy * X + ix] * scale * kInv4Pi;
    };
    for (uint32_t i : rays) {
        WRay& wr = wave[i];
        const uint32_t batch = wr.key >> 24, id = wr.key & 0xFFFFFFu;
        const bool isLight = batch == kBatchLight;
        const bool spec = !isLight && mat_specular(s, batch, id);
        const Surface<float> sf = gen_surface(s, wr.prim, wr.b0, wr.b1, wr.r.d);
        const F3 wi = -wr.r.d;
        const uint32_t smp = wr.r.aux.sample;
        const Rng4 r0 = rng_block(smp, frame, kTagGuide | depthTag, 0u, opt->seed_lo, opt->seed_hi);
        const bool purePG = w->pure_pg != 0;
        float ss = 0.0f, tt = 0.0f, pdf = 1.0f;
        bool bxdfSel = true;
        if (!purePG && (isLight || spec)) {
        } else if (!purePG && r0.u[0] >= w->mis_ratio) {
            const Rng4 r1 = rng_block(smp, frame, kTagGuide | depthTag, 1u, opt->seed_lo, opt->seed_hi);
            const BSample<float> bs = mat_sample(s, batch, id, wi, sf, wr.r.aux.medium, r1.u[0], r1.u[1], r1.u[2]);
            dir_yup_to_octa(bs.dir, ss, tt);
            const float pdfSampled = bs.pdf;
            const float pdfOther = pdf_at(ss, tt);
            const float ratio = 1.0f - w->mis_ratio;
            const float w0 = ratio * pdfSampled, w1 = (1.0f - ratio) * pdfOther;
            pdf = pdfSampled * ratio / (w0 / (w0 + w1));
            pdf = (pdfSampled == 0.0f) ? 0.0f : pdf;
            bxdfSel = true;
        } else {
            const float tY = r0.u[1] * total;
            int y = X - 1;
            for (int k = 0; k < X; k++)
                if (marg[k] > tY) { y = k; break; }
            const float rowTot = rowPre[y * X + X - 1];
            const float prevY = (y > 0) ? marg[y - 1] : 0.0f;
            const float dv = std::min(std::max((tY - prevY) / rowTot, 0.0f), below1);
            const float tX = r0.u[2] * rowTot;
            int x = X - 1;
            for (int k = 0; k < X; k++)
                if (rowPre[y * X + k] > tX) { x = k; break; }
            const float prevX = (x > 0) ? rowPre[y * X + x - 1] : 0.0f;
            const float du = std::min(std::max((tX - prevX) / field[y * X + x], 0.0f), below1);
            const float rcpX = 1.0f / static_cast<float>(X);
            ss = (static_cast<float>(x) + du) * rcpX;
            tt = (static_cast<float>(y) + dv) * rcpX;
            const float pdfSampled = field[y * X + x] * scale * kInv4Pi;
            if (purePG) {
                pdf = pdfSampled;
            } else {
                const F3 wo = octa_to_dir_yup(ss, tt);
                const float pdfOther = mat_pdf(s, batch, id, wo, wi, sf);
                const float ratio = w->mis_ratio;
                const float w0 = ratio * pdfSampled, w1 = (1.0f - ratio) * pdfOther;
                pdf = pdfSampled * ratio / (w0 / (w0 + w1));
                pdf = (pdfSampled == 0.0f) ? 0.0f : pdf;
            }
            bxdfSel = false;
        }
        if (pdf != pdf || ss != ss || tt != tt) {
            ss = 0.5f;
            tt = 0.5f;
            pdf = 1.0f;
        }
        wr.g0 = uint32_t(f2h(ss)) | (uint32_t(f2h(tt)) << 16);
        wr.g1 = uint32_t(f2h(pdf)) | (bxdfSel ? kGuideBxdf : 0u) | kGuideValid;
    }
}

// One bin of KCGenAndSampleDistributionProduct, X x X field
template <int X>
void guide_bin(const oracle_scene* s, const Tree& tree, const oracle_options* opt,
               const oracle_wfpg_options* w, uint32_t depthTag, uint32_t key,
               const std::vector<uint32_t>& rays, std::vector<WRay>& wave) {
    constexpr int DPP = X / 8;
    const float dppF = static_cast<float>(DPP);
    const uint32_t frame = opt->frame;
    const float aperture = (4.0f * kPiF) / (static_cast<float>(X) * static_cast<float>(X));
    const uint32_t mix = hash32(frame ^ hash32(depthTag ^ 0xA511E9B3u ^ opt->seed_lo));
    uint64_t best = ~0ull;
    uint32_t rep = 0;
    for (uint32_t i : rays) {
        const uint32_t smp = wave[i].r.aux.sample;
        const uint64_t k = (uint64_t(hash32(smp ^ mix)) << 32) | smp;
        if (k < best) {
            best = k;
            rep = i;
        }
    }
    const WRay& rr = wave[rep];
    const Surface<float> sf0 = gen_surface(s, rr.prim, rr.b0, rr.b1, rr.r.d);
    F3 org = nudge(sf0.pos, sf0.geo);
    org = org + sf0.geo * (tree.o->P.leaf * 0.01f);
    float tMin = tree.o->P.leaf * 0.15f;
    tMin += 1.0e-5f;
    const Rng4 rj = rng_block(key, frame, kTagGuideBin | depthTag, 0u, opt->seed_lo, opt->seed_hi);
    std::vector<float> field(X * X), tmp(X * X);
    for (int p = 0; p < X * X; p++) {
        const int x = p % X, y = p / X;
        float ss = (static_cast<float>(x) + rj.u[0]) / static_cast<float>(X);
        float tt = (static_cast<float>(y) + rj.u[1]) / static_cast<float>(X);
        octa_wrap(ss, tt);
        const F3 dir = octa_to_dir_yup(ss, tt);
        bool isLeaf;
        uint32_t id;
        tree.cone_trace(org, dir, tMin, aperture, 0u, isLeaf, id);
        float r = tree.read_radiance(dir, id, isLeaf);
        if (r == 0.0f) r = 1.0e-4f;
        field[p] = r;
    }
    for (int p = 0; p < X * X; p++) {
        const int x = p % X, y = p / X;
        float acc = 0.0f;
        for (int j = -5; j <= 5; j++) {
            int nx = x + j, ny = y;
            if (nx >= X || nx < 0) octa_wrap_int(nx, ny, X, X);
            acc += field[ny * X + nx] * w->filter[j + 5];
        }
        tmp[p] = acc;
    }
    for (int p = 0; p < X * X; p++) {
        const int x = p % X, y = p / X;
        float acc = 0.0f;
        for (int j = -5; j <= 5; j++) {
            int nx = x, ny = y + j;
            if (ny >= X || ny < 0) octa_wrap_int(nx, ny, X, X);
            acc += tmp[ny * X + nx] * w->filter[j + 5];
        }
        field[p] = acc;
    }
    if (!w->product) {
        guide_bin_pwc<X>(s, opt, w, depthTag, field, rays, wave);
        return;
    }
    float small[64], normc[64];
    product_cells<X>(field.data(), small, normc);
    const float kInv4Pi = 0.25f * kInvPiF;
    for (uint32_t i : rays) {
        WRay& wr = wave[i];
        const uint32_t batch = wr.key >> 24, id = wr.key & 0xFFFFFFu;
        const bool isLight = batch == kBatchLight;
        const bool spec = !isLight && mat_specular(s, batch, id);
        const Surface<float> sf = gen_surface(s, wr.prim, wr.b0, wr.b1, wr.r.d);
        const F3 wi = -wr.r.d;
        const F3 nrm = to_space(F3(0.0f, 0.0f, 1.0f), sf.w2t);
        float gray[64];
        for (int c = 0; c < 64; c++) {
            gray[c] = 1.0f;
            if (!isLight && !spec) gray[c] = lum3(mat_eval(s, batch, id, bxdf_proj(c & 7, c >> 3, nrm), wi, sf));
        }
        ProductCdf P;
        product_build(gray, small, P);
        const uint32_t smp = wr.r.aux.sample;
        const Rng4 r0 = rng_block(smp, frame, kTagGuide | depthTag, 0u, opt->seed_lo, opt->seed_hi);
        const bool purePG = w->pure_pg != 0;
        float ss = 0.0f, tt = 0.0f, pdf = 1.0f;
        bool bxdfSel = true;
        if (!purePG && (isLight || spec)) {
        } else if (!purePG && r0.u[0] >= w->mis_ratio) {
            const Rng4 r1 = rng_block(smp, frame, kTagGuide | depthTag, 1u, opt->seed_lo, opt->seed_hi);
            const BSample<float> bs = mat_sample(s, batch, id, wi, sf, wr.r.aux.medium, r1.u[0], r1.u[1], r1.u[2]);
            dir_yup_to_octa(bs.dir, ss, tt);
            const float pdfOther = product_pdf<X>(field.data(), small, P, ss, tt) * kInv4Pi;
            pdf = mis_pdf(bs.pdf, 1.0f - w->mis_ratio, pdfOther);
            bxdfSel = true;
        } else {
            auto draw = [&](int round, uint32_t lane, float& du, float& dv, float& da) {
                const Rng4 rl = rng_block(smp, frame, kTagGuide | depthTag, 2u + uint32_t(round) * 32u + lane,
                                          opt->seed_lo, opt->seed_hi);
                du = rl.u[0];
                dv = rl.u[1];
                da = rl.u[2];
            };
            float pdfS;
            product_sample<X>(field.data(), small, normc, P, r0.u[1], r0.u[2], draw, ss, tt, pdfS);
            if (purePG) {
                pdf = pdfS * kInv4Pi;
            } else {
                const F3 wo = octa_to_dir_yup(ss, tt);
                pdf = mis_pdf(pdfS * kInv4Pi, w->mis_ratio, mat_pdf(s, batch, id, wo, wi, sf));
            }
            bxdfSel = false;
        }
        if (pdf != pdf || ss != ss || tt != tt) {
            ss = 0.5f;
            tt = 0.5f;
            pdf = 1.0f;
        }
        wr.g0 = uint32_t(f2h(ss)) | (uint32_t(f2h(tt)) << 16);
        wr.g1 = uint32_t(f2h(pdf)) | (bxdfSel ? kGuideBxdf : 0u) | kGuideValid;
    }
}

}  // namespace

// The product sampler on table inputs (test infrastructure: the pin of the
// restatement against the reference's own ProductSampler run by
// oracle/psamp/psamp_harness.cu).  Per bin a 64x64 field; per ray a table
// surface (kPinSurface floats: RGB per product cell, a BxDF sample's uv and
// pdf, Pdf(wo) = a + b wo.x + c wo.y) and 32 lanes x streamLen uniforms,
// consumed as SampleMIS and Sample draw them (ProductSampler.cuh:370-470,
// 556-660): lane 0 draws the MIS choice, then (guide branch) the row; the
// leader lane of the chosen row within its group of four rows (lane
// 8 * (row % 4)) draws the column; then every lane draws (u, v) and the
// acceptance per rejection round.
namespace {
constexpr int kPinSurface = 198;
}

extern "C" void oracle_product_pin(const float* fields, uint32_t bins, uint32_t raysPerBin,
                                   const float* surfaces, const float* streams,
                                   uint32_t streamLen, float misRatio, float mult, float* uv,
                                   float* pdfOut, uint32_t* selOut, float* smallOut,
                                   float* normOut) {
    constexpr int X = 64;
    for (uint32_t b = 0; b < bins; b++) {
        const float* field = fields + size_t(b) * X * X;
        float small[64], normc[64];
        product_cells<X>(field, small, normc);
        for (int c = 0; c < 64; c++) {
            smallOut[b * 64 + c] = small[c];
            normOut[b * 64 + c] = normc[c];
        }
        for (uint32_t r = 0; r < raysPerBin; r++) {
            const uint32_t ray = b * raysPerBin + r;
            const float* t = surfaces + size_t(ray) * kPinSurface;
            const float* st = streams + size_t(ray) * 32 * streamLen;
            uint32_t next[32] = {};
            auto take = [&](uint32_t lane) {
                const uint32_t k = next[lane]++;
                return k < streamLen ? st[size_t(lane) * streamLen + k] : 0.5f;
            };
            float gray[64];
            for (int c = 0; c < 64; c++) gray[c] = lum3(F3(t[3 * c], t[3 * c + 1], t[3 * c + 2]));
            ProductCdf P;
            product_build(gray, small, P);
            float ss = 0.0f, tt = 0.0f, pdf = 0.0f;
            bool sel;
            const float xi = take(0);
            if (xi >= misRatio) {
                ss = t[192];
                tt = t[193];
                const float pdfOther = product_pdf<X>(field, small, P, ss, tt) * mult;
                pdf = mis_pdf(t[194], 1.0f - misRatio, pdfOther);
                sel = true;
            } else {
                const float xi0 = take(0);
                int row = 8;
                for (int l = 0; l < 8; l++)
                    if (!(xi0 > P.cdfY[l])) {
                        row = l;
                        break;
                    }
                row = std::min(row, 7);
                const float xi1 = take(uint32_t(8 * (row % 4)));
                auto draw = [&](int, uint32_t lane, float& du, float& dv, float& da) {
                    du = take(lane);
                    dv = take(lane);
                    da = take(lane);
                };
                float pdfS;
                product_sample<X>(field, small, normc, P, xi0, xi1, draw, ss, tt, pdfS);
                const float pdfOther = t[195] + t[196] * ss + t[197] * tt;
                pdf = mis_pdf(pdfS * mult, misRatio, pdfOther);
                sel = false;
            }
            uv[2 * size_t(ray)] = ss;
            uv[2 * size_t(ray) + 1] = tt;
            pdfOut[ray] = pdf;
            selOut[ray] = sel ? 1u : 0u;
        }
    }
}

extern "C" uint64_t oracle_render_wfpg(const oracle_scene* s, const oracle_bvh* b,
                                       const oracle_camera* cam, const oracle_options* opt,
                                       const oracle_wfpg_options* w, oracle_svo* svo, float* out,
                                       uint32_t* dumpGuide, uint32_t* dumpBin) {
    const uint32_t sp = opt->samples;
    const uint32_t SW = opt->width * sp, SH = opt->height * sp;
    const uint32_t P = SW * SH;
    const uint32_t levels = opt->max_depth + 1;
    Chain chain(levels, P);
    Tree tree{svo};
    const uint32_t D = svo->P.depth;
    const uint32_t minLevel = std::min(w->min_bin_level, D);
    Ctx<float> c{s, b, opt, out};
    for (uint32_t i = 0; i < 3 * P; i++) out[i] = 0.0f;
    std::vector<WRay> cur, next;
    cur.reserve(P);
    const float* Pc = cam->position;
    for (uint32_t sid = 0; sid < P; sid++) {
        // camera ray as in render(); WFPG numbers it depth 1 (RayAuxInitWFPG)
        const uint32_t sx = sid % SW, sy = sid / SW;
        const Rng4 rc = rng_block(sid, opt->frame, kTagCamera, 0, opt->seed_lo, opt->seed_hi);
        float dx = cam->plane_size[0] / static_cast<float>(SW);
        float dy = cam->plane_size[1] / static_cast<float>(SH);
        float sdx = static_cast<float>(sx) * dx;
        float sdy = static_cast<float>(sy) * dy;
        sdx += rc.u[0] * dx;
        sdy += rc.u[1] * dy;
        float v[3];
        for (int i = 0; i < 3; i++) v[i] = cam->bottom_left[i] + ((sdx * cam->right[i]) + (sdy * cam->up[i]));
        const F3 dirf = normalize(F3(v[0], v[1], v[2]) - F3(Pc[0], Pc[1], Pc[2]));
        WRay wr;
        wr.r.o = F3(Pc[0], Pc[1], Pc[2]);
        wr.r.d = dirf;
        wr.r.tmin = cam->near_far[0];
        wr.r.tmax = cam->near_far[1];
        wr.r.aux = Aux<float>{F3(1, 1, 1), sid, kInvalid, s->base_medium, 1, CAMERA_RAY,
                              std::numeric_limits<float>::quiet_NaN()};
        cur.push_back(wr);
        const size_t at = chain.at(0, sid);
        chain.pos[3 * at] = Pc[0];
        chain.pos[3 * at + 1] = Pc[1];
        chain.pos[3 * at + 2] = Pc[2];
        chain.rf[3 * at] = chain.rf[3 * at + 1] = chain.rf[3 * at + 2] = 1.0f;
        chain.valid[at] = 1;
    }
    uint64_t rays = 0;
    for (uint32_t it = 0; it < opt->max_depth && !cur.empty(); it++) {
        parallel_for(uint32_t(cur.size()), opt->threads, [&](uint32_t b0, uint32_t b1) {
            for (uint32_t i = b0; i < b1; i++) {
                WRay& wr = cur[i];
                const Hit<float> h = trace_one<float>(s, b, wr.r.o, wr.r.d, wr.r.tmin, wr.r.tmax);
                wr.prim = h.prim;
                wr.key = (h.prim == kInvalid) ? 0u : h.key;
                wr.t = h.t;
                wr.b0 = h.b0;
                wr.b1 = h.b1;
                wr.guided = false;
                wr.g0 = 0u;
                wr.g1 = 0x7E00u;
            }
        });
        rays += cur.size();
        const bool guideNow = !w->skip_pg && it < w->guide_bounce;
        if (guideNow) {
            std::vector<uint32_t> binKey(cur.size(), kBinInvalid);
            bin_rays(svo, uint32_t(cur.size()), minLevel, w->bin_ray_count,
                     [&](uint32_t i, F3& p) {
                         const WRay& wr = cur[i];
                         if (wr.r.aux.type == NEE_RAY || (wr.key >> 24) == kBatchNull) return false;
                         p = F3(wr.r.o.x + wr.t * wr.r.d.x, wr.r.o.y + wr.t * wr.r.d.y,
                                wr.r.o.z + wr.t * wr.r.d.z);
                         return true;
                     },
                     binKey.data());
            std::map<uint32_t, std::vector<uint32_t>> bins;
            for (size_t i = 0; i < cur.size(); i++)
                if (binKey[i] != kBinInvalid) bins[binKey[i]].push_back(uint32_t(i));
            std::vector<std::pair<uint32_t, const std::vector<uint32_t>*>> list;
            for (auto& kv : bins) list.push_back({kv.first, &kv.second});
            const uint32_t ki = it < 4 ? it : 4;
            parallel_for(uint32_t(list.size()), opt->threads, [&](uint32_t b0, uint32_t b1) {
                for (uint32_t q = b0; q < b1; q++) {
                    const uint32_t key = list[q].first;
                    const std::vector<uint32_t>& rs = *list[q].second;
                    if (ki <= 1) guide_bin<64>(s, tree, opt, w, it, key, rs, cur);
                    else if (ki == 2) guide_bin<32>(s, tree, opt, w, it, key, rs, cur);
                    else if (ki == 3) guide_bin<16>(s, tree, opt, w, it, key, rs, cur);
                    else guide_bin<8>(s, tree, opt, w, it, key, rs, cur);
                }
            });
            for (size_t i = 0; i < cur.size(); i++) cur[i].guided = binKey[i] != kBinInvalid;
            if (it == w->dump_iteration) {
                for (size_t i = 0; i < cur.size(); i++) {
                    if (binKey[i] == kBinInvalid) continue;
                    const uint32_t smp = cur[i].r.aux.sample;
                    if (dumpGuide) {
                        dumpGuide[2 * smp] = cur[i].g0;
                        dumpGuide[2 * smp + 1] = cur[i].g1;
                    }
                    if (dumpBin) dumpBin[smp] = binKey[i];
                }
            }
        }
        next.clear();
        const bool gen = (it + 1) < opt->max_depth;
        std::vector<PRay<float>> outs;
        for (WRay& wr : cur) {
            const uint32_t batch = wr.key >> 24, id = wr.key & 0xFFFFFFu;
            const Aux<float>& ax = wr.r.aux;
            if (wr.prim == kInvalid || batch == kBatchNull) {
                // the Null boundary light's work: zero emission, but the rays
                // it accepts count as reaching a light (WFPGTracerKC.cuh:163-195)
                const bool accepted = ax.type == SPECULAR_PATH_RAY ||
                                      (ax.type == PATH_RAY && (opt->mis || !opt->nee));
                if (accepted) chain.eventPath[chain.at(ax.depth, ax.sample)] = 1;
                continue;
            }
            if (batch == kBatchLight) {
                boundary_work(c, wr.r, id, wr.prim, wr.b0, wr.b1, wr.t, &chain);
            } else if (ax.type == NEE_RAY) {
                // DepositNEEHitMiss(prev vertex, miss) (WFPGTracerKC.cuh:250-260)
                chain.eventNee[chain.at(ax.depth, ax.sample)] = 2;
            } else {
                outs.clear();
                const uint32_t gw[2] = {wr.g0, wr.g1};
                path_work(c, wr.r, wr.prim, wr.b0, wr.b1, batch, id, gen, outs,
                          (guideNow && wr.guided) ? gw : nullptr, &chain);
                for (const PRay<float>& o : outs) {
                    WRay n;
                    n.r = o;
                    next.push_back(n);
                }
            }
        }
        std::swap(cur, next);
    }
    // WFPGTracer::Finalize: chain sums, deposit, normalise and filter
    for (uint32_t p = 0; p < P; p++) {
        uint32_t L = 0;
        while (L + 1 < levels && chain.valid[chain.at(L + 1, p)]) L++;
        const uint32_t lastD = (L + 1 < levels) ? L + 1 : levels - 1;
        for (uint32_t d = 1; d <= L; d++) {
            const size_t at = chain.at(d, p);
            const float bx = chain.rf[3 * at], by = chain.rf[3 * at + 1], bz = chain.rf[3 * at + 2];
            F3 tot(0.0f, 0.0f, 0.0f);
            for (uint32_t Dd = d + 1; Dd <= lastD; Dd++) {
                const size_t q = chain.at(Dd, p);
                const float* cn = &chain.nee[3 * q];
                const float* cp = &chain.path[3 * q];
                tot.x += (bx == 0.0f) ? 0.0f : cn[0] / bx;
                tot.y += (by == 0.0f) ? 0.0f : cn[1] / by;
                tot.z += (bz == 0.0f) ? 0.0f : cn[2] / bz;
                tot.x += (bx == 0.0f) ? 0.0f : cp[0] / bx;
                tot.y += (by == 0.0f) ? 0.0f : cp[1] / by;
                tot.z += (bz == 0.0f) ? 0.0f : cp[2] / bz;
            }
            const F3 pos(chain.pos[3 * at], chain.pos[3 * at + 1], chain.pos[3 * at + 2]);
            const size_t pa = chain.at(d - 1, p);
            const F3 wo = normalize(F3(chain.pos[3 * pa], chain.pos[3 * pa + 1], chain.pos[3 * pa + 2]) - pos);
            uint32_t hits = 0, misses = 0;
            if (d + 1 <= lastD) {
                const size_t q = chain.at(d + 1, p);
                hits = (chain.eventNee[q] == 1 ? 1u : 0u) + (chain.eventPath[q] == 1 ? 1u : 0u);
                misses = chain.eventNee[q] == 2 ? 1u : 0u;
            }
            deposit_leaf(svo, tree, pos, wo, lum3(tot), hits, misses);
        }
    }
    normalize_filter(svo);
    return rays;
}

namespace {
}  // namespace

// ========================================================================
// C ABI
// ========================================================================
extern "C" {

void oracle_sincosf(float x, float* s, float* c) { pm_sincos(x, *s, *c); }
float oracle_acosf(float x) { return pm_acos(x); }
void oracle_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    philox(ctr, key, out);
}
uint64_t oracle_morton3d(uint32_t x, uint32_t y, uint32_t z) { return morton3d(x, y, z); }
void oracle_trace_counters(uint64_t* out, int reset) {
    out[0] = g_nodes.load();
    out[1] = g_tris.load();
    if (reset) {
        g_nodes = 0;
        g_tris = 0;
    }
}

void oracle_morton_codes(const float* pos, const uint32_t* idx, uint32_t n, float* aabbs,
                         float* extent, float* delta, uint64_t* codes) {
    // Triangle AABBs (Triangle::BoundingBox) and the extent reduce
    // (LinearBVH.hpp:444-457).
    float ext[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (uint32_t t = 0; t < n; t++) {
        float* a = aabbs + 6 * t;
        for (int i = 0; i < 3; i++) {
            float v0 = pos[3 * idx[3 * t + 0] + i];
            float v1 = pos[3 * idx[3 * t + 1] + i];
            float v2 = pos[3 * idx[3 * t + 2] + i];
            a[i] = std::fmin(std::fmin(v0, v1), v2);
            a[3 + i] = std::fmax(std::fmax(v0, v1), v2);
            ext[i] = std::fmin(ext[i], a[i]);
            ext[3 + i] = std::fmax(ext[3 + i], a[3 + i]);
        }
    }
    std::memcpy(extent, ext, sizeof(ext));
    float md = morton_delta(ext);
    *delta = md;
    // KCGenMortonCodes (LinearBVH.hpp:118-166)
    for (uint32_t t = 0; t < n; t++) {
        const float* a = aabbs + 6 * t;
        uint32_t g[3];
        for (int i = 0; i < 3; i++) {
            float span = a[3 + i] - a[i];
            float center = a[i] + span * 0.5f;
            float rel = center - ext[i];
            g[i] = static_cast<uint32_t>(std::floor(rel / md));
        }
        codes[t] = morton3d(g[0], g[1], g[2]);
    }
}

void oracle_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint32_t n, int b, int e, int desc) {
    radix_sort<uint64_t>(keys, vals, n, b, e, desc != 0);
}
void oracle_sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t n, int b, int e, int desc) {
    radix_sort<uint32_t>(keys, vals, n, b, e, desc != 0);
}

int oracle_lbvh_build(const uint64_t* codes, const uint32_t* sorted_idx, const float* leaf_aabbs,
                      uint32_t n, uint32_t* left, uint32_t* right, uint32_t* parent,
                      float* inner, uint32_t* root) {
    if (n == 0) return 2;
    for (uint32_t i = 0; i < 2 * n - 1; i++) parent[i] = kInvalid;
    if (n == 1) {
        *root = 0;
        return 0;
    }
    const uint32_t ni = n - 1;
    std::vector<uint32_t> r0(ni, kInvalid), r1(ni, kInvalid);
    std::vector<uint32_t> work;
    work.reserve(n);
    // ChooseParentAndUpdate (LinearBVH.hpp:41-100)
    auto choose = [&](uint32_t lo, uint32_t hi, uint32_t global) {
        bool leftEdge = (lo == 0), rightEdge = (hi == n - 1);
        uint32_t ld = leftEdge ? 0 : lbvh_delta(codes, lo - 1);
        uint32_t rd = rightEdge ? 0 : lbvh_delta(codes, hi);
        uint32_t p;
        if (rd > ld) {
            p = hi;
            left[p] = global;
            r0[p] = lo;
        } else {
            p = lo - 1;
            right[p] = global;
            r1[p] = hi;
        }
        parent[global] = n + p;
        if (r0[p] != kInvalid && r1[p] != kInvalid) work.push_back(p);
    };
    for (uint32_t i = 0; i < n; i++) choose(i, i, i);
    *root = kInvalid;
    for (size_t w = 0; w < work.size(); w++) {
        uint32_t j = work[w];
        if (r0[j] == 0 && r1[j] == n - 1) {
            *root = n + j;
            parent[n + j] = kInvalid;
        } else {
            choose(r0[j], r1[j], n + j);
        }
    }
    // BottomUpAABB* (LinearBVH.hpp:290-396): post-order union.
    std::vector<uint32_t> st;
    std::vector<uint8_t> done(ni, 0);
    st.push_back(*root - n);
    auto box = [&](uint32_t g) -> const float* {
        return g < n ? leaf_aabbs + 6 * sorted_idx[g] : inner + 6 * (g - n);
    };
    while (!st.empty()) {
        uint32_t j = st.back();
        bool ready = true;
        uint32_t ch[2] = {left[j], right[j]};
        for (uint32_t c : ch)
            if (c >= n && !done[c - n]) {
                st.push_back(c - n);
                ready = false;
            }
        if (!ready) continue;
        st.pop_back();
        const float* a = box(ch[0]);
        const float* b = box(ch[1]);
        float* o = inner + 6 * j;
        for (int i = 0; i < 3; i++) {
            o[i] = std::fmin(a[i], b[i]);
            o[3 + i] = std::fmax(a[3 + i], b[3 + i]);
        }
        done[j] = 1;
    }
    uint32_t dups = 0;
    for (uint32_t i = 0; i + 1 < n; i++) dups += (codes[i] == codes[i + 1]);
    return dups ? 1 : 0;
}

uint32_t oracle_partition(const uint32_t* keys, uint32_t n, uint32_t bb, uint32_t ib,
                          uint32_t* skeys, uint32_t* sids, uint32_t* pb, uint32_t* po,
                          uint32_t* pc) {
    // SortKeys (RayMemory.cu:187-228): stable descending on id bits, then on
    // batch bits; equivalent to one stable descending sort of the dense key.
    std::vector<uint32_t> dk(n);
    for (uint32_t i = 0; i < n; i++) {
        uint32_t batch = (keys[i] >> 24) & ((1u << bb) - 1u);
        uint32_t id = keys[i] & ((ib >= 32) ? 0xFFFFFFFFu : ((1u << ib) - 1u));
        dk[i] = (batch << ib) | id;
        sids[i] = i;
    }
    radix_sort<uint32_t>(dk.data(), sids, n, 0, int(bb + ib), true);
    for (uint32_t i = 0; i < n; i++) skeys[i] = keys[sids[i]];
    // Partition (RayMemory.cu:230-312): batch boundaries -> portions in
    // ascending batch order (std::set<ArrayPortion>, ArrayPortion.h:35-44).
    std::vector<std::pair<uint32_t, std::pair<uint32_t, uint32_t>>> p;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t batch = skeys[i] >> 24;
        if (i == 0 || batch != (skeys[i - 1] >> 24)) p.push_back({batch, {i, 0}});
        p.back().second.second++;
    }
    std::sort(p.begin(), p.end());
    for (size_t i = 0; i < p.size(); i++) {
        pb[i] = p[i].first;
        po[i] = p[i].second.first;
        pc[i] = p[i].second.second;
    }
    return uint32_t(p.size());
}

oracle_bvh* oracle_bvh_create(const oracle_scene* s, int* status) {
    oracle_bvh* b = new oracle_bvh();
    uint32_t n = s->tri_count;
    b->n = n;
    b->leaf_aabbs.resize(size_t(n) * 6);
    b->codes.resize(n);
    b->sorted_idx.resize(n);
    b->v0.resize(size_t(n) * 3);
    b->e0.resize(size_t(n) * 3);
    b->e1.resize(size_t(n) * 3);
    for (uint32_t t = 0; t < n; t++) {
        for (int i = 0; i < 3; i++) {
            float p0 = s->pos[3 * s->idx[3 * t] + i];
            float p1 = s->pos[3 * s->idx[3 * t + 1] + i];
            float p2 = s->pos[3 * s->idx[3 * t + 2] + i];
            b->v0[3 * t + i] = p0;
            b->e0[3 * t + i] = p1 - p0;
            b->e1[3 * t + i] = p2 - p0;
        }
    }
    float ext[6], delta;
    std::vector<uint64_t> codes(n);
    oracle_morton_codes(s->pos, s->idx, n, b->leaf_aabbs.data(), ext, &delta, codes.data());
    for (uint32_t i = 0; i < n; i++) b->sorted_idx[i] = i;
    b->codes = codes;
    radix_sort<uint64_t>(b->codes.data(), b->sorted_idx.data(), n, 0, 64, false);
    if (n > 0) {
        b->left.resize(n > 1 ? n - 1 : 0);
        b->right.resize(n > 1 ? n - 1 : 0);
        b->parent.resize(2 * size_t(n) - 1);
        b->inner.resize(n > 1 ? size_t(n - 1) * 6 : 0);
        int st = oracle_lbvh_build(b->codes.data(), b->sorted_idx.data(), b->leaf_aabbs.data(), n,
                                   b->left.data(), b->right.data(), b->parent.data(),
                                   b->inner.data(), &b->root);
        if (status) *status = st;
    } else if (status) {
        *status = 0;
    }
    return b;
}
void oracle_bvh_destroy(oracle_bvh* b) { delete b; }
uint32_t oracle_bvh_root(const oracle_bvh* b) { return b->root; }

static void write_hits(const Hit<float>& h, uint32_t i, uint32_t* k, uint32_t* p, float* t,
                       float* bary) {
    k[i] = h.prim == kInvalid ? 0u : h.key;
    p[i] = h.prim;
    t[i] = h.t;
    bary[2 * i] = h.b0;
    bary[2 * i + 1] = h.b1;
}

void oracle_trace(const oracle_scene* s, const oracle_bvh* b, const float* rays, uint32_t n,
                  uint32_t* k, uint32_t* p, float* t, float* bary, uint32_t threads) {
    parallel_for(n, threads, [&](uint32_t b0, uint32_t b1) {
        for (uint32_t i = b0; i < b1; i++) {
            const float* r = rays + 8 * i;
            Hit<float> h = trace_one<float>(s, b, V3<float>(r[0], r[1], r[2]),
                                            V3<float>(r[4], r[5], r[6]), r[3], r[7]);
            write_hits(h, i, k, p, t, bary);
        }
    });
}
void oracle_trace_linear(const oracle_scene* s, const float* rays, uint32_t n, uint32_t* k,
                         uint32_t* p, float* t, float* bary, uint32_t threads) {
    int st = 0;
    oracle_bvh* b = oracle_bvh_create(s, &st);  // only the precomputed edges are used
    parallel_for(n, threads, [&](uint32_t b0, uint32_t b1) {
        for (uint32_t i = b0; i < b1; i++) {
            const float* r = rays + 8 * i;
            Hit<float> h = trace_linear_one<float>(s, b, V3<float>(r[0], r[1], r[2]),
                                                   V3<float>(r[4], r[5], r[6]), r[3], r[7]);
            write_hits(h, i, k, p, t, bary);
        }
    });
    delete b;
}

uint64_t oracle_render(const oracle_scene* s, const oracle_bvh* b, const oracle_camera* cam,
                       const oracle_options* opt, float* out) {
    return render<float>(s, b, cam, opt, out);
}

// Image-space sample coordinates: GPUCameraPinhole::GenerateRay's
// localCoords = (sampleId + offset) / sampleMax (GPUCameraPinhole.cuh:236),
// times the resolution (GenerationKernels.cuh:72), with the camera ray's
// own jitter.
void oracle_camera_img_coords(const oracle_options* opt, float* out) {
    const uint32_t SW = opt->width * opt->samples, SH = opt->height * opt->samples;
    const uint32_t total = SW * SH;
    for (uint32_t sid = 0; sid < total; sid++) {
        const uint32_t sx = sid % SW, sy = sid / SW;
        const Rng4 rc = rng_block(sid, opt->frame, kTagCamera, 0, opt->seed_lo, opt->seed_hi);
        const float lx = (static_cast<float>(sx) + rc.u[0]) / static_cast<float>(SW);
        const float ly = (static_cast<float>(sy) + rc.u[1]) / static_cast<float>(SH);
        out[2 * sid] = lx * static_cast<float>(opt->width);
        out[2 * sid + 1] = ly * static_cast<float>(opt->height);
    }
}
// ---- accelerator group of transformed surfaces (GPUAccBVHGroup::Hit,
// GPUAcceleratorBVHKC.cuh:229-346: the ray moved to the surface's local
// space by the inverse of its Matrix4x4 (Ray::Transform, RayLib/Ray.hpp:
// 459-465), traversed there; t is shared because the direction is not
// renormalised)
struct oracle_group {
    std::vector<float> pos;
    std::vector<uint32_t> idx, key;
    std::vector<uint8_t> cull;
    std::vector<uint32_t> begin, end, xf;
    std::vector<float> l2w, w2l;
    std::vector<oracle_scene> sub;
    std::vector<oracle_bvh*> bvh;
    ~oracle_group() {
        for (oracle_bvh* b : bvh) oracle_bvh_destroy(b);
    }
};

namespace {
// Inverse of a row-major 3x4 affine matrix in double, each entry rounded
// once (the same steps as the device library's host side).
bool affine_inverse_f(const float* m, float* out) {
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
inline V3<float> xf_point(const float* m, V3<float> p) {
    return {((m[0] * p.x + m[1] * p.y) + m[2] * p.z) + m[3],
            ((m[4] * p.x + m[5] * p.y) + m[6] * p.z) + m[7],
            ((m[8] * p.x + m[9] * p.y) + m[10] * p.z) + m[11]};
}
inline V3<float> xf_dir(const float* m, V3<float> d) {
    return {(m[0] * d.x + m[1] * d.y) + m[2] * d.z, (m[4] * d.x + m[5] * d.y) + m[6] * d.z,
            (m[8] * d.x + m[9] * d.y) + m[10] * d.z};
}
}  // namespace

extern "C" oracle_group* oracle_group_create(const float* pos, uint32_t V, const uint32_t* idx,
                                             const uint32_t* key, const uint8_t* cull, uint32_t T,
                                             const uint32_t* surfaces, uint32_t S,
                                             const float* l2w, uint32_t nT, int* status) {
    *status = 0;
    oracle_group* g = new oracle_group();
    g->pos.assign(pos, pos + 3 * size_t(V));
    g->idx.assign(idx, idx + 3 * size_t(T));
    g->key.assign(key, key + T);
    g->cull.assign(T, 0);
    if (cull) g->cull.assign(cull, cull + T);
    g->l2w.assign(l2w, l2w + 12 * size_t(nT));
    g->w2l.assign(12 * size_t(nT), 0.0f);
    for (uint32_t i = 0; i < nT; i++)
        if (!affine_inverse_f(&g->l2w[12 * size_t(i)], &g->w2l[12 * size_t(i)])) *status = 1;
    g->sub.resize(S);
    for (uint32_t si = 0; si < S; si++) {
        const uint32_t b = surfaces[3 * si], e = surfaces[3 * si + 1];
        g->begin.push_back(b);
        g->end.push_back(e);
        g->xf.push_back(surfaces[3 * si + 2]);
        oracle_scene sc{};
        sc.vertex_count = V;
        sc.tri_count = e - b;
        sc.pos = g->pos.data();
        sc.idx = g->idx.data() + 3 * size_t(b);
        sc.tri_key = g->key.data() + b;
        sc.tri_cull = g->cull.data() + b;
        g->sub[si] = sc;
        int st = 0;
        g->bvh.push_back(oracle_bvh_create(&g->sub[si], &st));
        if (st > 1) *status = 2;
    }
    return g;
}

extern "C" void oracle_group_destroy(oracle_group* g) { delete g; }

// Closest hit over every surface (surfaces in index order; a later surface
// replaces the hit only when strictly closer).  rays: origin, tMin,
// direction, tMax (8 floats).  Outputs per ray: material key, transform id,
// primitive id (group index, ~0 on a miss), t (tMax when missed), bary.
extern "C" void oracle_group_trace(const oracle_group* g, const float* rays, uint32_t n,
                                   uint32_t* key, uint32_t* tid, uint64_t* prim, float* tOut,
                                   float* bary) {
    parallel_for(n, 0, [&](uint32_t b0, uint32_t b1) {
        for (uint32_t i = b0; i < b1; i++) {
            const float* r = rays + 8 * size_t(i);
            float closest = r[7];
            key[i] = 0;
            tid[i] = 0;
            prim[i] = ~0ull;
            bary[2 * i] = bary[2 * i + 1] = 0.0f;
            for (size_t si = 0; si < g->sub.size(); si++) {
                const float* m = &g->w2l[12 * size_t(g->xf[si])];
                const V3<float> o = xf_point(m, V3<float>(r[0], r[1], r[2]));
                const V3<float> d = xf_dir(m, V3<float>(r[4], r[5], r[6]));
                const Hit<float> h = trace_one<float>(&g->sub[si], g->bvh[si], o, d, r[3], closest);
                if (h.prim != kInvalid && h.t < closest) {
                    closest = h.t;
                    key[i] = h.key;
                    tid[i] = g->xf[si];
                    prim[i] = uint64_t(g->begin[si]) + h.prim;
                    bary[2 * i] = h.b0;
                    bary[2 * i + 1] = h.b1;
                }
            }
            tOut[i] = closest;
        }
    });
}

// World AABB of each surface: the local box of its triangles (the LBVH's
// extent) with the eight corners transformed.
extern "C" void oracle_group_aabbs(const oracle_group* g, float* out) {
    for (size_t si = 0; si < g->sub.size(); si++) {
        float lo[3] = {M<float>::Max, M<float>::Max, M<float>::Max};
        float hi[3] = {-M<float>::Max, -M<float>::Max, -M<float>::Max};
        for (uint32_t t = g->begin[si]; t < g->end[si]; t++)
            for (int k = 0; k < 3; k++)
                for (int c = 0; c < 3; c++) {
                    const float v = g->pos[3 * size_t(g->idx[3 * size_t(t) + k]) + c];
                    lo[c] = std::fmin(lo[c], v);
                    hi[c] = std::fmax(hi[c], v);
                }
        const float* m = &g->l2w[12 * size_t(g->xf[si])];
        float wl[3] = {M<float>::Max, M<float>::Max, M<float>::Max};
        float wh[3] = {-M<float>::Max, -M<float>::Max, -M<float>::Max};
        for (int k = 0; k < 8; k++) {
            const V3<float> w = xf_point(m, V3<float>((k & 1) ? hi[0] : lo[0],
                                                      (k & 2) ? hi[1] : lo[1],
                                                      (k & 4) ? hi[2] : lo[2]));
            const float wc[3] = {w.x, w.y, w.z};
            for (int c = 0; c < 3; c++) {
                wl[c] = std::fmin(wl[c], wc[c]);
                wh[c] = std::fmax(wh[c], wc[c]);
            }
        }
        for (int c = 0; c < 3; c++) {
            out[6 * si + c] = wl[c];
            out[6 * si + 3 + c] = wh[c];
        }
    }
}

// Row-major 3x4 inverse used by the group (for the tests' own checks).
extern "C" int oracle_affine_inverse(const float* m, float* out) {
    return affine_inverse_f(m, out) ? 0 : -1;
}

uint64_t oracle_render_f64(const oracle_scene* s, const oracle_bvh* b, const oracle_camera* cam,
                           const oracle_options* opt, double* out) {
    return render<double>(s, b, cam, opt, out);
}

void oracle_bxdf_sample(uint32_t type, const float* params, const float* wi, const float* w2t,
                        const float* geo, const float* pos, uint32_t back, float from_ior,
                        float to_ior, const float* xi, float* out_dir, float* out_pos,
                        float* out_refl, float* out_pdf) {
    Surface<float> sf;
    sf.pos = V3<float>(pos[0], pos[1], pos[2]);
    sf.w2t = Q4<float>{w2t[0], w2t[1], w2t[2], w2t[3]};
    sf.geo = V3<float>(geo[0], geo[1], geo[2]);
    sf.back = back != 0;
    V3<float> w(wi[0], wi[1], wi[2]);
    BSample<float> bs;
    if (type == kBatchLambert) {
        bs = lambert_sample(V3<float>(params[0], params[1], params[2]), sf, xi[0], xi[1], 0);
    } else if (type == kBatchMetal) {
        bs = metal_sample(metal_params<float>(params), w, sf, xi[0], xi[1], 0);
    } else {
        float ior[2] = {from_ior, to_ior};
        uint32_t med[1] = {1};
        oracle_scene tmp{};
        tmp.medium_ior = ior;
        tmp.medium_count = 2;
        tmp.base_medium = 0;
        tmp.refract_medium = med;
        // entering: from = ior[cur=0], to = ior[1]; exiting handled by back
        bs = refract_sample(V3<float>(params[0], params[1], params[2]), 1u, &tmp, w, sf,
                            back ? 1u : 0u, xi[0]);
    }
    out_dir[0] = bs.dir.x; out_dir[1] = bs.dir.y; out_dir[2] = bs.dir.z;
    out_pos[0] = bs.pos.x; out_pos[1] = bs.pos.y; out_pos[2] = bs.pos.z;
    out_refl[0] = bs.refl.x; out_refl[1] = bs.refl.y; out_refl[2] = bs.refl.z;
    *out_pdf = bs.pdf;
}

// GPUPrimitiveTriangle.cpp:160-320 with Triangle::CalculateTangent
// (Triangle.h:73-111), OrthogonalVector (Vector.hpp:877-886) and
// TransformGen::Space (Quaternion.hpp:372-480).
void oracle_build_tbn(const float* pos, const float* nrm, const float* uvs, const uint32_t* idx,
                      uint32_t V, uint32_t T, float* out) {
    using F3 = V3<float>;
    auto P = [&](uint32_t v) { return F3(pos[3 * v], pos[3 * v + 1], pos[3 * v + 2]); };
    auto N = [&](uint32_t v) { return F3(nrm[3 * v], nrm[3 * v + 1], nrm[3 * v + 2]); };
    auto ortho = [](F3 v) {
        if (std::fabs(v.x) > std::fabs(v.y)) {
            float s = std::sqrt(v.x * v.x + v.z * v.z);
            return F3(-v.z / s, 0.0f / s, v.x / s);
        }
        float s = std::sqrt(v.y * v.y + v.z * v.z);
        return F3(0.0f / s, v.z / s, -v.y / s);
    };
    static const float defUv[3][2] = {{0.f, 0.f}, {1.f, 0.f}, {0.f, 1.f}};
    std::vector<F3> tan(V, F3(0, 0, 0));
    for (uint32_t t = 0; t < T; t++) {
        uint32_t ix[3] = {idx[3 * t], idx[3 * t + 1], idx[3 * t + 2]};
        const float* uv[3];
        for (int k = 0; k < 3; k++) uv[k] = uvs ? uvs + 2 * ix[k] : defUv[k];
        for (int k = 0; k < 3; k++) {
            int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
            F3 vec0 = P(ix[k1]) - P(ix[k]), vec1 = P(ix[k2]) - P(ix[k]);
            float du0x = uv[k1][0] - uv[k][0], du0y = uv[k1][1] - uv[k][1];
            float du1x = uv[k2][0] - uv[k][0], du1y = uv[k2][1] - uv[k][1];
            float det = (du0x * du1y - du1x * du0y);
            F3 tk;
            if (det == 0.0f) {
                tk = ortho(N(ix[k]));
            } else {
                float r = 1.0f / det;
                tk = r * (du1y * vec0 - du0y * vec1);
                if (det < 0) tk = -tk;
                if (std::isnan(tk.x) || std::isnan(tk.y) || std::isnan(tk.z)) tk = ortho(N(ix[k]));
            }
            tan[ix[k]] = tan[ix[k]] + tk;
        }
    }
    for (uint32_t v = 0; v < V; v++) {
        F3 n = N(v), t = tan[v];
        if (dot(t, t) < 1.0e-5f) t = ortho(n);
        t = normalize(t);
        F3 x = normalize(t - n * dot(n, t));
        F3 y = cross(n, x);
        F3 z = n;
        F3 c = cross(x, y) - z;
        if (std::fabs(c.x) > 0.1f && std::fabs(c.y) > 0.1f && std::fabs(c.z) > 0.1f) x = -x;
        float tt, w, qx, qy, qz;
        if (z.z < 0) {
            if (x.x > y.y) {
                tt = 1 + x.x - y.y - z.z;
                w = y.z - z.y; qx = tt; qy = x.y + y.x; qz = z.x + x.z;
            } else {
                tt = 1 - x.x + y.y - z.z;
                w = z.x - x.z; qx = x.y + y.x; qy = tt; qz = y.z + z.y;
            }
        } else {
            if (x.x < -y.y) {
                tt = 1 - x.x - y.y + z.z;
                w = x.y - y.x; qx = z.x + x.z; qy = y.z + z.y; qz = tt;
            } else {
                tt = 1 + x.x + y.y + z.z;
                w = tt; qx = y.z - z.y; qy = z.x - x.z; qz = x.y - y.x;
            }
        }
        float s = 0.5f / std::sqrt(tt);
        w *= s; qx *= s; qy *= s; qz *= s;
        float inv = 1.0f / std::sqrt(w * w + qx * qx + qy * qy + qz * qz);
        out[4 * v + 0] = w * inv;
        out[4 * v + 1] = -(qx * inv);
        out[4 * v + 2] = -(qy * inv);
        out[4 * v + 3] = -(qz * inv);
    }
}

// Single-function probes for the golden-vector tests.  in / out layouts per
// name are documented in oracle.h.  Returns 0, or -1 for an unknown name.
int oracle_probe(const char* name, const float* in, float* out) {
    using F3 = V3<float>;
    using Q = Q4<float>;
    auto v = [&](int i) { return F3(in[i], in[i + 1], in[i + 2]); };
    auto q = [&](int i) { return Q{in[i], in[i + 1], in[i + 2], in[i + 3]}; };
    auto w3 = [&](int i, F3 a) { out[i] = a.x; out[i + 1] = a.y; out[i + 2] = a.z; };
    auto w4 = [&](int i, Q a) { out[i] = a.w; out[i + 1] = a.x; out[i + 2] = a.y; out[i + 3] = a.z; };
    std::string n(name);
    if (n == "half") {  // x -> h2f(f2h(x)), f2h bits
        const uint16_t h = f2h(in[0]);
        out[0] = h2f(h);
        out[1] = static_cast<float>(h);
    } else if (n == "octa") {  // dir3 (y-up) -> s t, dir3 back
        float ss, tt;
        dir_yup_to_octa(v(0), ss, tt);
        out[0] = ss;
        out[1] = tt;
        w3(2, octa_to_dir_yup(ss, tt));
    } else if (n == "octa_wrap_int") {  // x y dim -> x y
        int32_t x = int32_t(in[0]), y = int32_t(in[1]);
        octa_wrap_int(x, y, int32_t(in[2]), int32_t(in[2]));
        out[0] = float(x);
        out[1] = float(y);
    } else if (n == "hemi_cosine") {  // xi0 xi1 -> dir3 pdf
        float pdf;
        F3 d = hemi_cosine(in[0], in[1], pdf);
        w3(0, d);
        out[3] = pdf;
    } else if (n == "reflect") {  // d3 n3 -> r3 (Ray::Reflect)
        F3 d = v(0), nn = v(3);
        w3(0, 2.0f * dot(d, nn) * nn - d);
    } else if (n == "refract") {  // d3 n3 from to -> ok r3 (Ray::Refract)
        F3 d = v(0), nn = v(3);
        float from = in[6], to = in[7];
        float ratio = from / to;
        float cosIn = dot(nn, d);
        float sinInSqr = std::fmax(0.0f, 1.0f - cosIn * cosIn);
        float sinOutSqr = ratio * ratio * sinInSqr;
        float cosOut = std::sqrt(std::fmax(0.0f, 1.0f - sinOutSqr));
        out[0] = (sinOutSqr >= 1.0f) ? 0.0f : 1.0f;
        if (out[0] != 0.0f) w3(1, ratio * (-d) + (ratio * cosIn - cosOut) * nn);
    } else if (n == "quat_rotate") {  // q4 v3 -> v3
        w3(0, qrotate(q(0), v(4)));
    } else if (n == "quat_mul") {  // q4 q4 -> q4
        w4(0, qmul(q(0), q(4)));
    } else if (n == "dggx") {  // ndh alpha -> d
        out[0] = dggx(in[0], in[1]);
    } else if (n == "gsmith_corr") {  // wo3 wi3 alpha -> g
        out[0] = g_smith_corr(v(0), v(3), in[6]);
    } else if (n == "gsmith_single") {  // v3 alpha -> g
        out[0] = g_smith_single(v(0), in[3]);
    } else if (n == "fresnel_conductor") {  // cos eta3 k3 -> f3
        w3(0, fresnel_conductor(in[0], v(1), v(4)));
    } else if (n == "fresnel_dielectric") {  // cos iorIn iorOut -> f
        out[0] = fresnel_dielectric(in[0], in[1], in[2]);
    } else if (n == "vndf_sample") {  // v3 alpha xi0 xi1 -> h3 pdf
        float pdf;
        w3(0, vndf_sample(pdf, v(0), in[3], in[4], in[5]));
        out[3] = pdf;
    } else if (n == "vndf_pdf") {  // v3 h3 alpha -> pdf
        out[0] = vndf_pdf(v(0), v(3), in[6]);
    } else if (n == "power_heuristic") {  // n0 p0 n1 p1
        float w0 = in[0] * in[1], w1 = in[2] * in[3];
        out[0] = (w0 * w0) / (w0 * w0 + w1 * w1);
    } else {
        return -1;
    }
    return 0;
}

void oracle_bary_slerp(const float* q0, const float* q1, const float* q2, float a, float b,
                       float* out) {
    Q4<float> r = bary_slerp(Q4<float>{q0[0], q0[1], q0[2], q0[3]},
                             Q4<float>{q1[0], q1[1], q1[2], q1[3]},
                             Q4<float>{q2[0], q2[1], q2[2], q2[3]}, a, b);
    out[0] = r.w; out[1] = r.x; out[2] = r.y; out[3] = r.z;
}
void oracle_nudge(const float* p, const float* d, float* out) {
    V3<float> r = nudge(V3<float>(p[0], p[1], p[2]), V3<float>(d[0], d[1], d[2]));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}
int oracle_intersect_tri(const float* ro, const float* rd, const float* p0, const float* p1,
                         const float* p2, int cull, float* t, float* bary3) {
    V3<float> a(p0[0], p0[1], p0[2]), b(p1[0], p1[1], p1[2]), c(p2[0], p2[1], p2[2]);
    float tt, b0, b1, v;
    bool h = intersect_tri(V3<float>(ro[0], ro[1], ro[2]), V3<float>(rd[0], rd[1], rd[2]), a,
                           b - a, c - a, cull != 0, tt, b0, b1, &v);
    if (h) {
        *t = tt;
        bary3[0] = b0;
        bary3[1] = b1;
        bary3[2] = v;
    }
    return h ? 1 : 0;
}

}  // extern "C"
