// 8-wide BVH with quantised child boxes, collapsed on the GPU from the LBVH,
// and its closest-hit traversal.
//
// Why: the binary traversal is bound by the L1/LSU data path (64 bytes per
// two child boxes).  A wide node carries eight child boxes quantised to 8
// bits per plane relative to the node's own box: 80 bytes for up to eight
// children.  Per box test that is 10 bytes instead of 32, and one node fetch
// replaces about three binary levels.
//
// Collapse (top-down, one launch per level of the wide tree): a wide node is
// formed from a binary node by choosing which binary descendants become its
// (at most eight) children.  Default: the surface-area dynamic program of
// Ylitie, Karras and Laine ("Efficient Incoherent Ray Traversal on GPUs
// Through Compressed Wide BVHs", HPG 2017), with one-triangle leaves: a
// bottom-up pass gives every binary node g the least sum of wide-node
// surface areas that represents its subtree as at most i children,
// cost(g, i) for i = 1..8, and the collapse follows its choices.  Without
// it, the internal child with the largest surface area is opened until the
// node has eight children or only leaves.
// Internal children get consecutive wide-node slots and leaf children
// consecutive triangle slots; slots are handed out by atomic counters per
// level, so the first 1 + 8 + 64 slots are the top three levels.  The
// binary LBVH (reference numbering) is unchanged: this is a traversal layout
// derived from it.
//
// Node (80 B = five 16-byte loads):
//   n0 = (box.lo.xyz, exps): exps = ex | ey << 8 | ez << 16 | imask << 24
//   n1 = (childBase, triBase, leafMask, 0)
//   n2 = (qlo.x[0..7], qlo.y[0..7]), n3 = (qlo.z[0..7], qhi.x[0..7]),
//   n4 = (qhi.y[0..7], qhi.z[0..7])
// Slot k holds an internal child (imask bit k: node childBase + the number
// of internal children in lower slots), a leaf (leafMask bit k: triangle
// triBase + the number of leaves in lower slots) or nothing.
// A child plane decodes as lo + q * 2^(e-127); quantisation rounds outward,
// so decoded boxes contain the exact child boxes.
#include <type_traits>

#include "../../include/mrb200.h"
#include "common.cuh"
#include "wide.cuh"
#include "pool.cuh"

namespace mrb {

namespace {

struct WorkItem {
    uint32_t bnode;  // binary node (global index, >= n inner)
    uint32_t slot;   // wide node slot
};

__device__ __forceinline__ void child_box(uint32_t g, uint32_t n, const float* __restrict__ inner,
                                          const float* __restrict__ triAabb,
                                          const uint32_t* __restrict__ sortedIdx, float lo[3],
                                          float hi[3]) {
    const float* b = (g < n) ? triAabb + 6 * size_t(sortedIdx[g]) : inner + 6 * size_t(g - n);
    for (int c = 0; c < 3; c++) {
        lo[c] = b[c];
        hi[c] = b[3 + c];
    }
}

__device__ __forceinline__ float half_area(const float lo[3], const float hi[3]) {
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// Exponent byte e (scale 2^(e-127)) so that extent / scale <= 255.
__device__ __forceinline__ uint32_t quant_exponent(float extent) {
    if (!(extent > 0.0f)) return 1u;  // degenerate axis: planes decode to lo exactly
    float x = extent / 255.0f;
    uint32_t bits = __float_as_uint(x);
    uint32_t e = (bits >> 23) & 0xFFu;
    if (bits & 0x7FFFFFu) e += 1u;  // round up to a power of two
    // make sure the rounded division cannot exceed 255
    while (e < 254u && extent / __uint_as_float(e << 23) > 255.0f) e++;
    return e < 1u ? 1u : e;
}

// ---------------------------------------------------------------------------
// Surface-area collapse plan
//   cost(leaf, i) = 0 (every triangle is a leaf child exactly once)
//   D(g, i)       = min over k in 1..i-1 of cost(left, k) + cost(right, i - k)
//   E(g, 2) = D(g, 2), E(g, i) = min(E(g, i - 1), D(g, i))
//   cost(g, 1)    = area(g) + E(g, 8)          (g becomes a wide node)
//   cost(g, i)    = min(cost(g, 1), E(g, i))   (i >= 2)
// Plan per inner node (8 bytes): byte 0 bit i - 1 set where cost(g, i) takes
// cost(g, 1) (g stays one child), byte i - 1 (i = 2..8) the k of D(g, i), 0
// where E(g, i) = E(g, i - 1).  D(g, 2) always has k = 1.
// ---------------------------------------------------------------------------
__global__ void k_plan_parents(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                               uint32_t n, uint32_t* parent, uint32_t* flags) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j + 1 < n;
         j += gridDim.x * blockDim.x) {
        parent[left[j]] = n + j;
        parent[right[j]] = n + j;
        flags[j] = 0u;
    }
}

// One thread per leaf walks up; the second arrival at a node evaluates it
// (the pattern of the LBVH's bottom-up box pass).  The walk ends at the root.
__global__ void k_plan_up(const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                          const float* __restrict__ inner, const uint32_t* __restrict__ parent,
                          const uint32_t* __restrict__ root, uint32_t n, uint32_t* flags,
                          float* cost, uint2* plan) {
    const uint32_t top = *root;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t g = parent[i];
        while (true) {
            __threadfence();
            if (atomicAdd(flags + (g - n), 1u) == 0u) break;  // the sibling is not done yet
            __threadfence();
            const uint32_t j = g - n;
            const uint32_t l = left[j], r = right[j];
            float cl[9], cr[9];
            for (int k = 1; k <= 8; k++) {
                cl[k] = (l >= n) ? __ldcg(cost + 8 * size_t(l - n) + (k - 1)) : 0.0f;
                cr[k] = (r >= n) ? __ldcg(cost + 8 * size_t(r - n) + (k - 1)) : 0.0f;
            }
            float E[9];
            uint32_t ks[9];
            for (int c = 2; c <= 8; c++) {
                float best = 0.0f;
                uint32_t bk = 0;
                for (int k = 1; k < c; k++) {
                    const float v = cl[k] + cr[c - k];
                    if (bk == 0 || v < best) {
                        best = v;
                        bk = uint32_t(k);
                    }
                }
                if (c > 2 && E[c - 1] <= best) {
                    best = E[c - 1];
                    bk = 0;
                }
                E[c] = best;
                ks[c] = bk;
            }
            const float* b = inner + 6 * size_t(j);
            const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
            const float c1 = (dx * dy + dy * dz + dz * dx) + E[8];
            float* cj = cost + 8 * size_t(j);
            uint32_t single = 0;
            cj[0] = c1;
            for (int c = 2; c <= 8; c++) {
                if (c1 <= E[c]) single |= 1u << (c - 1);
                cj[c - 1] = fminf(c1, E[c]);
            }
            plan[j] = make_uint2(single | (ks[2] << 8) | (ks[3] << 16) | (ks[4] << 24),
                                 ks[5] | (ks[6] << 8) | (ks[7] << 16) | (ks[8] << 24));
            if (g == top) break;
            g = parent[g];
        }
    }
}

__device__ __forceinline__ uint32_t plan_byte(uint2 p, int b) {
    return ((b < 4 ? p.x : p.y) >> (8 * (b & 3))) & 0xFFu;
}

// The children of the wide node made from binary node g under the plan: at
// most eight, at least two.  Each pending entry holds at least one slot, so
// at most eight entries are ever pending.
__device__ __forceinline__ int plan_children(uint32_t g, uint32_t n, const uint32_t* __restrict__ left,
                                             const uint32_t* __restrict__ right,
                                             const uint2* __restrict__ plan, uint32_t ch[8]) {
    uint32_t sg[16];
    uint8_t si[16], sown[16];
    int sp = 1, nc = 0;
    sg[0] = g;
    si[0] = 8;
    sown[0] = 1;
    while (sp > 0) {
        sp--;
        const uint32_t x = sg[sp];
        int i = si[sp];
        const bool own = sown[sp] != 0;
        if (!own && (x < n || i == 1)) {
            ch[nc++] = x;
            continue;
        }
        const uint2 pl = plan[x - n];
        if (!own && ((pl.x >> (i - 1)) & 1u)) {
            ch[nc++] = x;
            continue;
        }
        uint32_t k;
        while ((k = plan_byte(pl, i - 1)) == 0u) i--;
        // left takes k slots, right i - k (each >= 1)
        sg[sp] = right[x - n];
        si[sp] = uint8_t(i - int(k));
        sown[sp] = 0;
        sg[sp + 1] = left[x - n];
        si[sp + 1] = uint8_t(k);
        sown[sp + 1] = 0;
        sp += 2;
    }
    return nc;
}

__global__ void __launch_bounds__(128) k_collapse(
    const WorkItem* __restrict__ qin, const uint32_t* __restrict__ qinCount, WorkItem* qout,
    uint32_t* qoutCount, uint32_t* nodeCounter, uint32_t* triCounter, uint32_t n,
    const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
    const float* __restrict__ inner, const float* __restrict__ triAabb,
    const uint32_t* __restrict__ sortedIdx, const float* __restrict__ pos,
    const uint32_t* __restrict__ idx, const uint32_t* __restrict__ key,
    const uint8_t* __restrict__ cull, const uint2* __restrict__ plan, WideNode* nodes, float4* tv0,
    float4* te0, float4* te1) {
    const uint32_t count = *qinCount;
    for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < count;
         w += gridDim.x * blockDim.x) {
        const WorkItem it = qin[w];
        uint32_t ch[8];
        float area[8];
        int nc = 2;
        ch[0] = left[it.bnode - n];
        ch[1] = right[it.bnode - n];
        if (plan) {
            nc = plan_children(it.bnode, n, left, right, plan, ch);
        } else {
            for (int k = 0; k < 2; k++) {
                float lo[3], hi[3];
                child_box(ch[k], n, inner, triAabb, sortedIdx, lo, hi);
                area[k] = (ch[k] >= n) ? half_area(lo, hi) : -1.0f;
            }
            // open the largest internal child until eight children
            while (nc < 8) {
                int best = -1;
                for (int k = 0; k < nc; k++)
                    if (ch[k] >= n && (best < 0 || area[k] > area[best])) best = k;
                if (best < 0) break;
                const uint32_t b = ch[best];
                const uint32_t c0 = left[b - n], c1 = right[b - n];
                ch[best] = c0;
                ch[nc] = c1;
                float lo[3], hi[3];
                child_box(c0, n, inner, triAabb, sortedIdx, lo, hi);
                area[best] = (c0 >= n) ? half_area(lo, hi) : -1.0f;
                child_box(c1, n, inner, triAabb, sortedIdx, lo, hi);
                area[nc] = (c1 >= n) ? half_area(lo, hi) : -1.0f;
                nc++;
            }
        }
        // slot of each child: the octant of its centroid around the node's
        // centre, matched greedily by the largest projection on the
        // octant's diagonal, so that slot ^ (ray octant) orders the
        // children roughly front to back for any ray direction
        {
            float nlo[3], nhi[3];
            child_box(it.bnode, n, inner, triAabb, sortedIdx, nlo, nhi);
            float cost[8][8];
            for (int k = 0; k < nc; k++) {
                float lo[3], hi[3];
                child_box(ch[k], n, inner, triAabb, sortedIdx, lo, hi);
                float dc[3];
                for (int c = 0; c < 3; c++) dc[c] = (lo[c] + hi[c]) - (nlo[c] + nhi[c]);
                for (int sl = 0; sl < 8; sl++)
                    cost[k][sl] = -(((sl & 1) ? dc[0] : -dc[0]) + ((sl & 2) ? dc[1] : -dc[1]) +
                                    ((sl & 4) ? dc[2] : -dc[2]));
            }
            uint32_t slotOf[8];
            uint32_t usedChild = 0, usedSlot = 0;
            for (int round = 0; round < nc; round++) {
                int bk = -1, bs = -1;
                float bc = 0.0f;
                for (int k = 0; k < nc; k++) {
                    if (usedChild & (1u << k)) continue;
                    for (int sl = 0; sl < 8; sl++) {
                        if (usedSlot & (1u << sl)) continue;
                        if (bk < 0 || cost[k][sl] < bc) {
                            bk = k;
                            bs = sl;
                            bc = cost[k][sl];
                        }
                    }
                }
                slotOf[bk] = uint32_t(bs);
                usedChild |= 1u << bk;
                usedSlot |= 1u << bs;
            }
            uint32_t bySlot[8];
            for (int sl = 0; sl < 8; sl++) bySlot[sl] = kInvalid;
            for (int k = 0; k < nc; k++) bySlot[slotOf[k]] = ch[k];
            nc = 8;
            for (int sl = 0; sl < 8; sl++) ch[sl] = bySlot[sl];
        }
        int nInner = 0, nLeaf = 0;
        for (int k = 0; k < nc; k++)
            if (ch[k] != kInvalid) (ch[k] >= n) ? nInner++ : nLeaf++;
        const uint32_t childBase = nInner ? atomicAdd(nodeCounter, uint32_t(nInner)) : 0u;
        const uint32_t triBase = nLeaf ? atomicAdd(triCounter, uint32_t(nLeaf)) : 0u;
        const uint32_t qbase = nInner ? atomicAdd(qoutCount, uint32_t(nInner)) : 0u;

        // node box = the binary node's box
        float blo[3], bhi[3];
        child_box(it.bnode, n, inner, triAabb, sortedIdx, blo, bhi);
        uint32_t e[3];
        float scale[3];
        for (int c = 0; c < 3; c++) {
            e[c] = quant_exponent(bhi[c] - blo[c]);
            scale[c] = __uint_as_float(e[c] << 23);
        }
        uint32_t leafMask = 0;
        uint8_t q[6][8];
        for (int c = 0; c < 6; c++)
            for (int k = 0; k < 8; k++) q[c][k] = (c < 3) ? 255 : 0;  // empty slot never hits
        uint32_t imask = 0;
        int ri = 0, rl = 0;
        for (int k = 0; k < nc; k++) {
            if (ch[k] == kInvalid) continue;  // empty slot
            float lo[3], hi[3];
            child_box(ch[k], n, inner, triAabb, sortedIdx, lo, hi);
            for (int c = 0; c < 3; c++) {
                // outward rounding in double: exact for float inputs and
                // power-of-two scales
                double ql = floor((double(lo[c]) - double(blo[c])) / double(scale[c]));
                double qh = ceil((double(hi[c]) - double(blo[c])) / double(scale[c]));
                ql = ql < 0.0 ? 0.0 : (ql > 255.0 ? 255.0 : ql);
                qh = qh < 0.0 ? 0.0 : (qh > 255.0 ? 255.0 : qh);
                q[c][k] = static_cast<uint8_t>(ql);
                q[3 + c][k] = static_cast<uint8_t>(qh);
            }
            if (ch[k] >= n) {
                imask |= 1u << k;
                qout[qbase + ri] = WorkItem{ch[k], childBase + uint32_t(ri)};
                ri++;
            } else {
                leafMask |= 1u << k;
                // leaf: the triangle, reordered into this node's leaf block
                const uint32_t t = sortedIdx[ch[k]];
                const uint32_t s = triBase + uint32_t(rl);
                const uint32_t i0 = idx[3 * size_t(t)], i1 = idx[3 * size_t(t) + 1],
                               i2 = idx[3 * size_t(t) + 2];
                const V3 p0 = ld3(pos + 3 * size_t(i0)), p1 = ld3(pos + 3 * size_t(i1)),
                         p2 = ld3(pos + 3 * size_t(i2));
                const V3 e0 = p1 - p0, e1 = p2 - p0;
                tv0[s] = make_float4(p0.x, p0.y, p0.z, __uint_as_float(t));
                te0[s] = make_float4(e0.x, e0.y, e0.z, __uint_as_float(key[t]));
                te1[s] = make_float4(e1.x, e1.y, e1.z,
                                     __uint_as_float(cull ? uint32_t(cull[t]) : 0u));
                rl++;
            }
        }
        WideNode nd;
        nd.n0 = make_float4(blo[0], blo[1], blo[2],
                            __uint_as_float(e[0] | (e[1] << 8) | (e[2] << 16) | (imask << 24)));
        nd.n1 = make_uint4(childBase, triBase, leafMask, 0u);
        auto pack = [&](int c, int k0) {
            return q[c][k0] | (q[c][k0 + 1] << 8) | (q[c][k0 + 2] << 16) |
                   (uint32_t(q[c][k0 + 3]) << 24);
        };
        nd.n2 = make_uint4(pack(0, 0), pack(0, 4), pack(1, 0), pack(1, 4));
        nd.n3 = make_uint4(pack(2, 0), pack(2, 4), pack(3, 0), pack(3, 4));
        nd.n4 = make_uint4(pack(4, 0), pack(4, 4), pack(5, 0), pack(5, 4));
        nodes[it.slot] = nd;
    }
}

__global__ void k_collapse_init(WorkItem* q0, uint32_t* counters, const uint32_t* root) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        q0[0] = WorkItem{*root, 0u};
        counters[0] = 1;  // queue 0 count
        counters[1] = 0;  // queue 1 count
        counters[2] = 1;  // node counter (slot 0 = root)
        counters[3] = 0;  // triangle counter
    }
}

__global__ void k_reset_count(uint32_t* c) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *c = 0;
}

// ---------------------------------------------------------------------------
// Traversal
// ---------------------------------------------------------------------------
// The top two levels (1 + 8 nodes) are read from shared memory.  Three
// levels (73 nodes, 5.8 KB per block) measured 2 % slower on both
// clusters-1M and Cornell: the smaller carve-out leaves more of the SM's
// on-chip memory to L1, which serves the lower levels.  None at all was
// faster on clusters-1M but 13 % slower on Cornell.
constexpr int kCachedNodes = 9;
constexpr int kWideStack = 128;  // sorted order: one entry per pushed child
constexpr int kWideGroups = 48;  // octant order: at most one group per level

__device__ __forceinline__ float safe_dir(float d) {
    return (fabsf(d) > 1e-20f) ? d : copysignf(1e-20f, d);
}

__device__ __forceinline__ uint32_t byte_of(uint32_t w, int k) { return (w >> (8 * k)) & 0xFFu; }

__device__ __forceinline__ void cas(uint32_t& a, uint32_t& b) {
    const uint32_t lo = min(a, b), hi = max(a, b);
    a = lo;
    b = hi;
}
// Optimal 19-comparator network for eight keys (ascending).
__device__ __forceinline__ void sort8(uint32_t k[8]) {
    cas(k[0], k[2]); cas(k[1], k[3]); cas(k[4], k[6]); cas(k[5], k[7]);
    cas(k[0], k[4]); cas(k[1], k[5]); cas(k[2], k[6]); cas(k[3], k[7]);
    cas(k[0], k[1]); cas(k[2], k[3]); cas(k[4], k[5]); cas(k[6], k[7]);
    cas(k[2], k[4]); cas(k[3], k[5]);
    cas(k[1], k[4]); cas(k[3], k[6]);
    cas(k[1], k[2]); cas(k[3], k[4]); cas(k[5], k[6]);
}

__device__ __forceinline__ void tri_test(const WideAccelDev& acc, uint32_t s, V3 o, V3 d,
                                         float tmin, float& closest, int& hitTri, float& hb0,
                                         float& hb1) {
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
        hitTri = static_cast<int>(s);
        hb0 = 1.0f - u - v;
        hb1 = u;
    }
}

template <int k>
using IntC = std::integral_constant<int, k>;

// Per-ray state of a traversal: the ray, its closest hit so far and the
// node to visit next (-1: done).  The stack lives beside it.
struct WideRay {
    V3 o, d, inv;
    float tmin, closest, hb0, hb1;
    int hitTri, node, sp;
    uint32_t oct;  // sign bits of the direction: x | y << 1 | z << 2
};

__device__ __forceinline__ void wide_ray_begin(WideRay& r, float4 ro, float4 rd) {
    r.o = V3{ro.x, ro.y, ro.z};
    r.d = V3{rd.x, rd.y, rd.z};
    r.tmin = ro.w;
    r.closest = rd.w;
    r.hb0 = r.hb1 = 0.0f;
    r.hitTri = -1;
    r.inv = V3{1.0f / safe_dir(rd.x), 1.0f / safe_dir(rd.y), 1.0f / safe_dir(rd.z)};
    r.oct = (r.inv.x < 0.0f ? 1u : 0u) | (r.inv.y < 0.0f ? 2u : 0u) | (r.inv.z < 0.0f ? 4u : 0u);
    r.node = 0;
    r.sp = 0;
}

// A node's words and its child slabs in the ray's frame: child plane q
// lies at t = q * a + b per axis; the near and far plane words are chosen
// per axis from the direction's sign.  The top `cached` nodes are read from
// shared memory (sNodes), the rest through the read-only cache.
struct NodeSlabs {
    uint32_t childBase, triBase, leafMask, imask;
    float ax, ay, az, bx, by, bz;
    uint32_t qn[6], qf[6];  // x0 x1 y0 y1 z0 z1: bytes of slots 0-3 and 4-7
};

__device__ __forceinline__ void node_slabs(const WideAccelDev& acc, const WideNode* sNodes,
                                           int cached, int node, const WideRay& r,
                                           NodeSlabs& s) {
    uint4 w0, w1, w2, w3, w4;
    if (node < cached) {
        const uint4* sm = reinterpret_cast<const uint4*>(sNodes + node);
        w0 = sm[0]; w1 = sm[1]; w2 = sm[2]; w3 = sm[3]; w4 = sm[4];
    } else {
        const uint4* g = reinterpret_cast<const uint4*>(acc.nodes + node);
        w0 = __ldg(g); w1 = __ldg(g + 1); w2 = __ldg(g + 2); w3 = __ldg(g + 3);
        w4 = __ldg(g + 4);
    }
    const float sx = __uint_as_float((w0.w & 0xFFu) << 23);
    const float sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23);
    const float sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
    s.imask = w0.w >> 24;
    // t = (lo + q*s - o) * inv = q * (s*inv) + (lo - o) * inv
    s.ax = sx * r.inv.x;
    s.ay = sy * r.inv.y;
    s.az = sz * r.inv.z;
    s.bx = (__uint_as_float(w0.x) - r.o.x) * r.inv.x;
    s.by = (__uint_as_float(w0.y) - r.o.y) * r.inv.y;
    s.bz = (__uint_as_float(w0.z) - r.o.z) * r.inv.z;
    s.childBase = w1.x;
    s.triBase = w1.y;
    s.leafMask = w1.z;
    const bool px = r.inv.x >= 0.0f, py = r.inv.y >= 0.0f, pz = r.inv.z >= 0.0f;
    s.qn[0] = px ? w2.x : w3.z; s.qn[1] = px ? w2.y : w3.w;
    s.qf[0] = px ? w3.z : w2.x; s.qf[1] = px ? w3.w : w2.y;
    s.qn[2] = py ? w2.z : w4.x; s.qn[3] = py ? w2.w : w4.y;
    s.qf[2] = py ? w4.x : w2.z; s.qf[3] = py ? w4.y : w2.w;
    s.qn[4] = pz ? w3.x : w4.z; s.qn[5] = pz ? w3.y : w4.w;
    s.qf[4] = pz ? w4.z : w3.x; s.qf[5] = pz ? w4.w : w3.y;
}

// A plane byte as a float.  The integer-to-float conversion runs on the
// narrow XU pipe; the other form builds the float 2^23 + byte with a byte
// permute (bit pattern 0x4B0000bb) and subtracts 2^23 on the FMA pipe.
// Both give the byte's value exactly.
template <bool kPermute>
__device__ __forceinline__ float plane_byte(uint32_t w, int kk) {
    if (kPermute)
        return __uint_as_float(__byte_perm(w, 0x4B000000u, uint32_t(kk) | 0x7540u)) - 8388608.0f;
    return float(byte_of(w, kk));
}

// Entry and exit distance of child slot k (compile-time k).  kMix converts
// the three near planes by byte permute and the far ones on XU, splitting
// the work between the pipes (the octant kernels, whose node loop is
// otherwise bound by XU: clusters-1M traversal 3.27 -> 2.72 ms per frame;
// the sorted kernels keep the conversions on XU, where the split measured
// slower).
template <int k, bool kMix>
__device__ __forceinline__ void child_span(const NodeSlabs& s, float tmin, float closest,
                                           float& tn, float& tf) {
    constexpr int h = k < 4 ? 0 : 1, kk = k & 3;
    const float tnx = __fmaf_rn(plane_byte<kMix>(s.qn[0 + h], kk), s.ax, s.bx);
    const float tfx = __fmaf_rn(plane_byte<false>(s.qf[0 + h], kk), s.ax, s.bx);
    const float tny = __fmaf_rn(plane_byte<kMix>(s.qn[2 + h], kk), s.ay, s.by);
    const float tfy = __fmaf_rn(plane_byte<false>(s.qf[2 + h], kk), s.ay, s.by);
    const float tnz = __fmaf_rn(plane_byte<kMix>(s.qn[4 + h], kk), s.az, s.bz);
    const float tfz = __fmaf_rn(plane_byte<false>(s.qf[4 + h], kk), s.az, s.bz);
    tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, tmin));
    tf = fminf(fminf(tfx, tfy), fminf(tfz, closest));
}


// One node of the traversal in exact front-to-back order: the hit internal
// children are sorted by entry distance, the nearest entered and the others
// pushed one by one with their distance (entries beyond the closest hit are
// dropped when pushed or popped).  The triangles of hit leaf children are
// tested after the eight box tests, before the push, so the box tests carry
// no triangle test between them (measured on Cornell at 1080p: 12.5 ->
// 11.1 ms of traversal per frame).  False when the ray is done.
template <bool kCount, int kStack>
__device__ __forceinline__ bool visit_sorted(const WideAccelDev& acc, const WideNode* sNodes,
                                             int cached, WideRay& r, uint2* stack,
                                             uint32_t& nodeVisits, uint32_t& triTests,
                                             uint32_t* errorFlag) {
    if (kCount) nodeVisits++;
    NodeSlabs s;
    node_slabs(acc, sNodes, cached, r.node, r, s);
    // internal children that are hit, keyed by entry distance:
    // (distance bits with the low three cleared) | slot
    uint32_t key[8];
    uint32_t m = 0;  // bit slot for each hit slot
    auto child = [&](auto kc) {
        constexpr int k = decltype(kc)::value;
        float tn, tf;
        child_span<k, false>(s, r.tmin, r.closest, tn, tf);
        const bool hit = tn <= tf;
        key[k] = (hit && ((s.imask >> k) & 1u)) ? ((__float_as_uint(tn) & 0x7FFFFFF8u) | uint32_t(k))
                                                : 0xFFFFFFFFu;
        if (hit) m |= 1u << k;
    };
    child(IntC<0>{}); child(IntC<1>{}); child(IntC<2>{}); child(IntC<3>{});
    child(IntC<4>{}); child(IntC<5>{}); child(IntC<6>{}); child(IntC<7>{});
    uint32_t leafHits = m & s.leafMask;
    while (leafHits) {
        const uint32_t k = uint32_t(__ffs(int(leafHits)) - 1);
        leafHits &= leafHits - 1u;
        if (kCount) triTests++;
        tri_test(acc, s.triBase + uint32_t(__popc(s.leafMask & ((1u << k) - 1u))), r.o, r.d,
                 r.tmin, r.closest, r.hitTri, r.hb0, r.hb1);
    }
    sort8(key);
    // push the farther hits (farthest first), enter the nearest
    int next = -1;
#pragma unroll
    for (int j = 7; j >= 0; j--) {
        if (key[j] == 0xFFFFFFFFu) continue;
        const float tn = __uint_as_float(key[j] & ~7u);
        if (tn > r.closest) continue;
        const uint32_t slot = key[j] & 7u;
        const uint32_t c = s.childBase + uint32_t(__popc(s.imask & ((1u << slot) - 1u)));
        if (j == 0) {
            next = int(c);
        } else if (r.sp < kStack) {
            stack[r.sp++] = make_uint2(c, key[j] & ~7u);
        } else {
            atomicExch(errorFlag, 3u);
        }
    }
    // the nearest hit may lie beyond the closest triangle: fall through to
    // the stack
    while (next < 0 && r.sp > 0) {
        const uint2 e = stack[--r.sp];
        if (__uint_as_float(e.y) <= r.closest) next = int(e.x);
    }
    r.node = next;
    return next >= 0;
}

// One node of the traversal in octant order: the collapse put every child
// in the slot of its centroid's octant around the node's centre, so the
// order slot ^ oct runs roughly front to back without sorting.  The stack
// holds node groups: the child base of a visited node, its internal-child
// mask and the bits of its hit internal children still to visit, one entry
// per node however many children were hit.  A child's node index is the
// child base plus the number of internal children in lower slots.  The
// triangles of hit leaf children are tested after the eight box tests, so
// the box tests carry no triangle test between them.  False when the ray
// is done.
template <bool kCount, int kStack>
__device__ __forceinline__ bool visit_octant(const WideAccelDev& acc, const WideNode* sNodes,
                                             int cached, WideRay& r, uint2* stack,
                                             uint32_t& nodeVisits, uint32_t& triTests,
                                             uint32_t* errorFlag) {
    if (kCount) nodeVisits++;
    NodeSlabs s;
    node_slabs(acc, sNodes, cached, r.node, r, s);
    uint32_t m = 0;  // bit slot for each hit slot
    auto child = [&](auto kc) {
        constexpr int k = decltype(kc)::value;
        float tn, tf;
        child_span<k, true>(s, r.tmin, r.closest, tn, tf);
        if (tn <= tf) m |= 1u << k;
    };
    child(IntC<0>{}); child(IntC<1>{}); child(IntC<2>{}); child(IntC<3>{});
    child(IntC<4>{}); child(IntC<5>{}); child(IntC<6>{}); child(IntC<7>{});
    uint32_t leafHits = m & s.leafMask;
    while (leafHits) {
        const uint32_t k = uint32_t(__ffs(int(leafHits)) - 1);
        leafHits &= leafHits - 1u;
        if (kCount) triTests++;
        tri_test(acc, s.triBase + uint32_t(__popc(s.leafMask & ((1u << k) - 1u))), r.o, r.d,
                 r.tmin, r.closest, r.hitTri, r.hb0, r.hb1);
    }
    // hit internal children, bit k moved to k ^ oct (swapping bit pairs,
    // then pairs of pairs, then nibbles, as the octant's bits say)
    uint32_t hits = m & s.imask;
    hits = (r.oct & 1u) ? (((hits & 0x55u) << 1) | ((hits >> 1) & 0x55u)) : hits;
    hits = (r.oct & 2u) ? (((hits & 0x33u) << 2) | ((hits >> 2) & 0x33u)) : hits;
    hits = (r.oct & 4u) ? (((hits & 0x0Fu) << 4) | ((hits >> 4) & 0x0Fu)) : hits;
    uint32_t base = s.childBase, im = s.imask;
    if (hits == 0) {  // resume the most recent group with pending children
        if (r.sp == 0) {
            r.node = -1;
            return false;
        }
        const uint2 e = stack[--r.sp];
        base = e.x;
        im = e.y >> 8;
        hits = e.y & 0xFFu;
    }
    const uint32_t b = uint32_t(__ffs(int(hits)) - 1);
    const uint32_t slot = b ^ r.oct;
    hits &= hits - 1u;
    if (hits) {
        if (r.sp < kStack) stack[r.sp++] = make_uint2(base, (im << 8) | hits);
        else atomicExch(errorFlag, 3u);
    }
    r.node = int(base + uint32_t(__popc(im & ((1u << slot) - 1u))));
    return true;
}

template <bool kCount, bool kOctant, int kStack>
__device__ __forceinline__ bool wide_visit(const WideAccelDev& acc, const WideNode* sNodes,
                                           int cached, WideRay& r, uint2* stack,
                                           uint32_t& nodeVisits, uint32_t& triTests,
                                           uint32_t* errorFlag) {
    if (kOctant)
        return visit_octant<kCount, kStack>(acc, sNodes, cached, r, stack, nodeVisits, triTests,
                                            errorFlag);
    return visit_sorted<kCount, kStack>(acc, sNodes, cached, r, stack, nodeVisits, triTests,
                                        errorFlag);
}

// Stack entries per ray: the sorted order pushes one entry per child, the
// octant order one per node group (at most one per level).
template <bool kOctant>
struct WideStack {
    static constexpr int value = kOctant ? kWideGroups : kWideStack;
};

// Closest hit of one ray in one 8-wide tree, in either child order.
template <bool kCount, bool kOctant, int kStack>
__device__ __forceinline__ void trace_wide_ray(const WideAccelDev& acc, const WideNode* sNodes,
                                               int cached, float4 ro, float4 rd, WideRay& r,
                                               uint32_t& nodeVisits, uint32_t& triTests,
                                               uint32_t* errorFlag) {
    wide_ray_begin(r, ro, rd);
    if (acc.triCount == 1) {
        if (kCount) triTests++;
        tri_test(acc, 0, r.o, r.d, r.tmin, r.closest, r.hitTri, r.hb0, r.hb1);
    } else if (acc.triCount > 1) {
        uint2 stack[kStack];
        while (wide_visit<kCount, kOctant, kStack>(acc, sNodes, cached, r, stack, nodeVisits,
                                                   triTests, errorFlag)) {
        }
    }
}

__device__ __forceinline__ void write_hit(const WideAccelDev& acc, const HitOut& out, uint32_t i,
                                          int hitTri, float closest, float hb0, float hb1) {
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

__device__ __forceinline__ void load_top_nodes(const WideAccelDev& acc, WideNode* sNodes,
                                               int cached) {
    for (int i = threadIdx.x; i < cached * 5; i += blockDim.x)
        reinterpret_cast<uint4*>(sNodes)[i] = __ldg(reinterpret_cast<const uint4*>(acc.nodes) + i);
    __syncthreads();
}

__device__ __forceinline__ void add_work(unsigned long long* counters, uint32_t nodeVisits,
                                         uint32_t triTests) {
    unsigned long long a = nodeVisits, b = triTests;
    for (int s = 16; s > 0; s >>= 1) {
        a += __shfl_xor_sync(0xFFFFFFFFu, a, s);
        b += __shfl_xor_sync(0xFFFFFFFFu, b, s);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(counters + 0, a);
        atomicAdd(counters + 1, b);
    }
}

// Eight 128-thread blocks per SM (64 registers, no spill): the traversal's
// dependent loads and ALU chains want resident warps more than registers,
// but not at the price of spills.  Octant order on clusters-1M: 2.66 ms of
// traversal per frame at eight blocks, 2.70 at nine (56 registers), 2.84 at
// ten (48, spilling); sorted order on the closed Cornell frame: 34.5 ms at
// eight, 34.9 at nine.
template <bool kCount, bool kOctant>
__global__ void __launch_bounds__(128, 8) k_trace_wide(WideAccelDev acc,
                                                    const float4* __restrict__ rayO,
                                                    const float4* __restrict__ rayD,
                                                    const uint32_t* __restrict__ dCount,
                                                    uint32_t hCount, HitOut out,
                                                    uint32_t* errorFlag,
                                                    unsigned long long* counters) {
    __shared__ WideNode sNodes[kCachedNodes];
    const int cached = acc.nodeCount < uint32_t(kCachedNodes) ? int(acc.nodeCount) : kCachedNodes;
    load_top_nodes(acc, sNodes, cached);
    const uint32_t n = dCount ? *dCount : hCount;
    uint32_t nodeVisits = 0, triTests = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        WideRay r;
        trace_wide_ray<kCount, kOctant, WideStack<kOctant>::value>(
            acc, sNodes, cached, rayO[i], rayD[i], r, nodeVisits, triTests, errorFlag);
        write_hit(acc, out, i, r.hitTri, r.closest, r.hb0, r.hb1);
    }
    if (kCount) add_work(counters, nodeVisits, triTests);
}

// Lanes refilled: a lane whose ray is done takes its warp's next ray once
// kRefillLanes lanes (or all) are idle, so a warp of rays with uneven path
// lengths keeps its lanes busy until its rays run out.  Warp w owns the
// 32-ray chunks w, w + W, w + 2W, ... (W warps in the grid) and hands their
// rays out in order; the set of rays a warp traces is the same as without
// refilling, only the lanes they run on differ.  Refilling mixes rays of
// neighbouring chunks in one warp: a gain for the scattered rays of later
// bounces, a loss for coherent camera rays (measured per depth by the
// tracer's order tuning).
constexpr int kRefillLanes = 8;

template <bool kCount, bool kOctant>
__global__ void __launch_bounds__(128, 8) k_trace_wide_refill(WideAccelDev acc,
                                                           const float4* __restrict__ rayO,
                                                           const float4* __restrict__ rayD,
                                                           const uint32_t* __restrict__ dCount,
                                                           uint32_t hCount, HitOut out,
                                                           uint32_t* errorFlag,
                                                           unsigned long long* counters) {
    constexpr int kStack = WideStack<kOctant>::value;
    __shared__ WideNode sNodes[kCachedNodes];
    const int cached = acc.nodeCount < uint32_t(kCachedNodes) ? int(acc.nodeCount) : kCachedNodes;
    load_top_nodes(acc, sNodes, cached);
    const uint32_t n = dCount ? *dCount : hCount;
    uint32_t nodeVisits = 0, triTests = 0;
    if (acc.triCount < 2) {
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
             i += gridDim.x * blockDim.x) {
            WideRay r;
            trace_wide_ray<kCount, kOctant, kStack>(acc, sNodes, cached, rayO[i], rayD[i], r,
                                                    nodeVisits, triTests, errorFlag);
            write_hit(acc, out, i, r.hitTri, r.closest, r.hb0, r.hb1);
        }
    } else {
        const uint32_t lane = threadIdx.x & 31u;
        const uint64_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const uint64_t nWarps = (gridDim.x * blockDim.x) >> 5;
        uint32_t next = 0;  // rays of the warp's sequence handed out (warp-uniform)
        bool more = warp * 32u < n, active = false;
        uint32_t ri = 0;
        WideRay r;
        r.node = -1;
        uint2 stack[kStack];
        while (true) {
            if (more) {
                const uint32_t need = __ballot_sync(0xFFFFFFFFu, !active);
                if (__popc(need) >= kRefillLanes || need == 0xFFFFFFFFu) {
                    if (!active) {
                        const uint32_t j = next + uint32_t(__popc(need & ((1u << lane) - 1u)));
                        const uint64_t idx = (warp + uint64_t(j >> 5) * nWarps) * 32u + (j & 31u);
                        if (idx < n) {
                            ri = uint32_t(idx);
                            wide_ray_begin(r, rayO[ri], rayD[ri]);
                            active = true;
                        }
                    }
                    next += uint32_t(__popc(need));
                    more = (warp + uint64_t(next >> 5) * nWarps) * 32u + (next & 31u) < n;
                }
            }
            if (!__any_sync(0xFFFFFFFFu, active)) break;
            if (!active) continue;
            if (!wide_visit<kCount, kOctant, kStack>(acc, sNodes, cached, r, stack, nodeVisits,
                                                     triTests, errorFlag)) {
                write_hit(acc, out, ri, r.hitTri, r.closest, r.hb0, r.hb1);
                active = false;
            }
        }
    }
    if (kCount) add_work(counters, nodeVisits, triTests);
}

// Rays of many scenes: each ray's tree is its job's (RayAux::pad is the job
// slot).  No shared-memory top levels: neighbouring rays may use different
// trees.
template <int kBlock, int kStack, bool kOctant>
__global__ void __launch_bounds__(kBlock) k_trace_wide_jobs(const JobDev* __restrict__ jobs,
                                                            const RayAux* __restrict__ aux,
                                                            const float4* __restrict__ rayO,
                                                            const float4* __restrict__ rayD,
                                                            const uint32_t* __restrict__ dCount,
                                                            uint32_t hCount, HitOut out,
                                                            uint32_t* errorFlag) {
    const uint32_t n = dCount ? *dCount : hCount;
    uint32_t nodeVisits = 0, triTests = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const WideAccelDev acc = jobs[aux[i].pad].wide;
        WideRay r;
        trace_wide_ray<false, kOctant, kOctant ? kWideGroups : kStack>(
            acc, nullptr, 0, rayO[i], rayD[i], r, nodeVisits, triTests, errorFlag);
        write_hit(acc, out, i, r.hitTri, r.closest, r.hb0, r.hb1);
    }
}

}  // namespace

namespace {
size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
size_t queue_bytes(uint32_t n) { return align256(size_t(n + 1) * sizeof(WorkItem) * 2 + 64); }
}  // namespace

size_t wide_scratch_bytes(uint32_t n) {
    // two work queues of n items + 4 counters; the collapse plan: parents
    // (2n), arrival flags (n), costs (8n) and plans (n)
    return queue_bytes(n) + align256(size_t(2) * n * 4) + align256(size_t(n) * 4) +
           align256(size_t(8) * n * 4) + align256(size_t(n) * 8);
}

int wide_build(const WideBuildIn& in, WideNode* nodes, float4* tv0, float4* te0, float4* te1,
               void* scratch, uint32_t* nodeCountOut, cudaStream_t stream) {
    const uint32_t n = in.n;
    if (n < 2) {
        set_error("wide BVH: needs at least two triangles");
        return MRB_E_ARG;
    }
    WorkItem* q[2];
    q[0] = static_cast<WorkItem*>(scratch);
    q[1] = q[0] + (n + 1);
    uint32_t* counters = reinterpret_cast<uint32_t*>(q[1] + (n + 1));
    const uint2* plan = nullptr;
    if (in.collapse == kWideCollapseSah) {
        char* b = static_cast<char*>(scratch) + queue_bytes(n);
        uint32_t* parent = reinterpret_cast<uint32_t*>(b);
        b += align256(size_t(2) * n * 4);
        uint32_t* flags = reinterpret_cast<uint32_t*>(b);
        b += align256(size_t(n) * 4);
        float* cost = reinterpret_cast<float*>(b);
        b += align256(size_t(8) * n * 4);
        uint2* pl = reinterpret_cast<uint2*>(b);
        const uint32_t g = std::min<uint32_t>((n + 255) / 256, 148u * 8u);
        k_plan_parents<<<g, 256, 0, stream>>>(in.left, in.right, n, parent, flags);
        k_plan_up<<<g, 256, 0, stream>>>(in.left, in.right, in.inner, parent, in.root, n, flags,
                                         cost, pl);
        MRB_CUDA(cudaGetLastError());
        plan = pl;
    }
    k_collapse_init<<<1, 32, 0, stream>>>(q[0], counters, in.root);
    MRB_CUDA(cudaGetLastError());
    // one launch per level; the host checks for an empty queue every 8 levels
    const uint32_t grid = std::min<uint32_t>((n + 127) / 128, 148u * 8u);
    for (int level = 0; level < 4 * 96; level++) {
        const int cur = level & 1;
        k_reset_count<<<1, 32, 0, stream>>>(counters + (cur ^ 1));
        k_collapse<<<grid, 128, 0, stream>>>(q[cur], counters + cur, q[cur ^ 1], counters + (cur ^ 1),
                                             counters + 2, counters + 3, n, in.left, in.right,
                                             in.inner, in.triAabb, in.sortedIdx, in.pos, in.idx,
                                             in.key, in.cull, plan, nodes, tv0, te0, te1);
        MRB_CUDA(cudaGetLastError());
        if ((level & 7) == 7) {
            uint32_t h[4];
            MRB_CUDA(cudaMemcpyAsync(h, counters, 16, cudaMemcpyDeviceToHost, stream));
            MRB_CUDA(cudaStreamSynchronize(stream));
            if (h[0] == 0 && h[1] == 0) {
                if (h[3] != n) {
                    set_error("wide BVH: %u of %u triangles placed", h[3], n);
                    return MRB_E_DEVICE;
                }
                *nodeCountOut = h[2];
                return 0;
            }
        }
    }
    set_error("wide BVH: collapse did not finish");
    return MRB_E_DEVICE;
}

int trace_closest_wide(const WideAccelDev& acc, const float4* rayO, const float4* rayD,
                       const uint32_t* dCount, uint32_t maxCount, const HitOut& out,
                       uint32_t* errorFlag, cudaStream_t stream, unsigned long long* counters,
                       int order) {
    if (maxCount == 0) return 0;
    uint32_t blocks = (maxCount + 127) / 128;
    blocks = blocks < 148u * 16u ? blocks : 148u * 16u;
    auto go = [&](auto kernel) {
        kernel<<<blocks, 128, 0, stream>>>(acc, rayO, rayD, dCount, maxCount, out, errorFlag,
                                           counters);
    };
    const bool c = counters != nullptr;
    switch (order) {
        case kWideSorted: c ? go(k_trace_wide<true, false>) : go(k_trace_wide<false, false>); break;
        case kWideOctant: c ? go(k_trace_wide<true, true>) : go(k_trace_wide<false, true>); break;
        case kWideSortedRefill:
            c ? go(k_trace_wide_refill<true, false>) : go(k_trace_wide_refill<false, false>);
            break;
        case kWideOctantRefill:
            c ? go(k_trace_wide_refill<true, true>) : go(k_trace_wide_refill<false, true>);
            break;
        default:
            set_error("wide traversal: order %d unknown", order);
            return MRB_E_ARG;
    }
    MRB_CUDA(cudaGetLastError());
    return 0;
}

namespace {
// Seeded probe rays over the scene's box: origins uniform in it, directions
// uniform on the sphere (Philox counter (i, 0, 0x60000, 0)).
__global__ void k_probe_rays(const float* __restrict__ ext, uint32_t n, float4* rayO,
                             float4* rayD) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Rand4 r = philox_uniform4(i, 0u, 0x60000u, 0u, 0x5eedu, 0u);
        const Rand4 q = philox_uniform4(i, 1u, 0x60000u, 0u, 0x5eedu, 0u);
        float o[3];
        for (int c = 0; c < 3; c++) o[c] = ext[c] + r.u[c] * (ext[3 + c] - ext[c]);
        const float z = 1.0f - 2.0f * q.u[0];
        const float rr = sqrtf(fmaxf(0.0f, 1.0f - z * z));
        float sn, cs;
        pm_sincos(6.2831853f * q.u[1], sn, cs);
        rayO[i] = make_float4(o[0], o[1], o[2], 0.0f);
        rayD[i] = make_float4(rr * cs, rr * sn, z, 3.0e38f);
    }
}
}  // namespace

int wide_order_autotune(const WideAccelDev& acc, const float* dExtent, cudaStream_t st,
                        int* orderOut, float* msOut) {
    constexpr uint32_t kProbe = 1u << 16;
    void* buf = nullptr;
    const size_t bytes = size_t(kProbe) * (16 + 16 + 4 + 4 + 4 + 8) + 16;
    MRB_CUDA(cudaMalloc(&buf, bytes));
    char* b = static_cast<char*>(buf);
    float4* ro = reinterpret_cast<float4*>(b);
    float4* rd = ro + kProbe;
    HitOut ho{reinterpret_cast<uint32_t*>(rd + kProbe), nullptr, nullptr, nullptr};
    ho.prim = ho.key + kProbe;
    ho.t = reinterpret_cast<float*>(ho.prim + kProbe);
    ho.bary = reinterpret_cast<float2*>(ho.t + kProbe);
    uint32_t* err = reinterpret_cast<uint32_t*>(ho.bary + kProbe);
    cudaEvent_t e[2];
    cudaEventCreate(&e[0]);
    cudaEventCreate(&e[1]);
    float best[kWideOrders];
    for (float& b : best) b = 1e30f;
    int rc = 0;
    k_probe_rays<<<(kProbe + 255) / 256, 256, 0, st>>>(dExtent, kProbe, ro, rd);
    for (int rep = 0; rep < 4 && rc == 0; rep++)
        for (int order = 0; order < kWideOrders && rc == 0; order++) {
            cudaEventRecord(e[0], st);
            rc = trace_closest_wide(acc, ro, rd, nullptr, kProbe, ho, err, st, nullptr, order);
            cudaEventRecord(e[1], st);
            cudaEventSynchronize(e[1]);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, e[0], e[1]);
            if (rep > 0) best[order] = std::min(best[order], ms);  // the first pass warms up
        }
    cudaEventDestroy(e[0]);
    cudaEventDestroy(e[1]);
    cudaFree(buf);
    if (rc) return rc;
    MRB_CUDA(cudaGetLastError());
    int pick = 0;
    for (int o = 1; o < kWideOrders; o++)
        if (best[o] < best[pick]) pick = o;
    *orderOut = pick;
    if (msOut)
        for (int o = 0; o < kWideOrders; o++) msOut[o] = best[o];
    return 0;
}

int wide_probe_compare(const WideAccelDev& a, const WideAccelDev& b, const float* dExtent,
                       cudaStream_t st, double bytesOut[2]) {
    constexpr uint32_t kProbe = 1u << 16;
    void* buf = nullptr;
    const size_t bytes = size_t(kProbe) * (16 + 16 + 4 + 4 + 4 + 8) + 64;
    MRB_CUDA(cudaMalloc(&buf, bytes));
    char* base = static_cast<char*>(buf);
    float4* ro = reinterpret_cast<float4*>(base);
    float4* rd = ro + kProbe;
    HitOut ho{reinterpret_cast<uint32_t*>(rd + kProbe), nullptr, nullptr, nullptr};
    ho.prim = ho.key + kProbe;
    ho.t = reinterpret_cast<float*>(ho.prim + kProbe);
    ho.bary = reinterpret_cast<float2*>(ho.t + kProbe);
    unsigned long long* work = reinterpret_cast<unsigned long long*>(ho.bary + kProbe);
    uint32_t* err = reinterpret_cast<uint32_t*>(work + 2);
    int rc = 0;
    k_probe_rays<<<(kProbe + 255) / 256, 256, 0, st>>>(dExtent, kProbe, ro, rd);
    for (int which = 0; which < 2 && !rc; which++) {
        unsigned long long h[2] = {0ull, 0ull};
        if (cudaMemsetAsync(work, 0, 16 + 4, st) != cudaSuccess) rc = MRB_E_CUDA;
        if (!rc)
            rc = trace_closest_wide(which ? b : a, ro, rd, nullptr, kProbe, ho, err, st, work,
                                    kWideOctant);
        if (!rc && (cudaMemcpyAsync(h, work, 16, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess))
            rc = MRB_E_CUDA;
        bytesOut[which] = double(h[0]) * double(sizeof(WideNode)) + double(h[1]) * 48.0;
    }
    cudaFree(buf);
    if (rc) {
        set_error("wide BVH: probe trace failed");
        return rc;
    }
    return 0;
}

template <int kBlock, int kStack, bool kOctant>
static int launch_jobs(const JobDev* jobs, const RayAux* aux, const float4* rayO,
                       const float4* rayD, const uint32_t* dCount, uint32_t maxCount,
                       const HitOut& out, uint32_t* errorFlag, cudaStream_t stream) {
    uint32_t blocks = (maxCount + kBlock - 1) / kBlock;
    const uint32_t cap = 148u * (2048u / kBlock);
    blocks = blocks < cap ? blocks : cap;
    k_trace_wide_jobs<kBlock, kStack, kOctant><<<blocks, kBlock, 0, stream>>>(
        jobs, aux, rayO, rayD, dCount, maxCount, out, errorFlag);
    MRB_CUDA(cudaGetLastError());
    return 0;
}

template <int kBlock>
static int launch_jobs_stack(const JobDev* jobs, const RayAux* aux, const float4* rayO,
                             const float4* rayD, const uint32_t* dCount, uint32_t maxCount,
                             const HitOut& out, uint32_t* errorFlag, int stack,
                             cudaStream_t stream) {
    if (stack == 0)
        return launch_jobs<kBlock, kWideStack, true>(jobs, aux, rayO, rayD, dCount, maxCount, out,
                                                     errorFlag, stream);
    if (stack > 64)
        return launch_jobs<kBlock, 128, false>(jobs, aux, rayO, rayD, dCount, maxCount, out,
                                               errorFlag, stream);
    return launch_jobs<kBlock, 64, false>(jobs, aux, rayO, rayD, dCount, maxCount, out, errorFlag,
                                          stream);
}

int trace_closest_wide_jobs(const JobDev* jobs, const RayAux* aux, const float4* rayO,
                            const float4* rayD, const uint32_t* dCount, uint32_t maxCount,
                            const HitOut& out, uint32_t* errorFlag, int block, int stack,
                            cudaStream_t stream) {
    if (maxCount == 0) return 0;
    switch (block) {
        case 64:
            return launch_jobs_stack<64>(jobs, aux, rayO, rayD, dCount, maxCount, out, errorFlag,
                                         stack, stream);
        case 256:
            return launch_jobs_stack<256>(jobs, aux, rayO, rayD, dCount, maxCount, out, errorFlag,
                                          stack, stream);
        default:
            return launch_jobs_stack<128>(jobs, aux, rayO, rayD, dCount, maxCount, out, errorFlag,
                                          stack, stream);
    }
}

}  // namespace mrb
