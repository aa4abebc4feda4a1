// 8-wide quantised BVH: build from the LBVH and closest-hit traversal (see wide.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include "common.cuh"
#include "trace.cuh"

namespace mrb {

struct alignas(16) WideNode {
    float4 n0;
    uint4 n1, n2, n3, n4;
};

struct WideAccelDev {
    const WideNode* nodes;
    const float4* tv0;  // triangles in wide-leaf order: v0 | original index
    const float4* te0;  // e0 | HitKey
    const float4* te1;  // e1 | cull flag
    uint32_t nodeCount;
    uint32_t triCount;
};

struct WideBuildIn {
    uint32_t n;                  // triangles (>= 2)
    const uint32_t* root;        // device: global index of the LBVH root
    const uint32_t* left;
    const uint32_t* right;
    const float* inner;
    const float* triAabb;
    const uint32_t* sortedIdx;
    const float* pos;
    const uint32_t* idx;
    const uint32_t* key;
    const uint8_t* cull;
    int collapse;                // kWideCollapseGreedy or kWideCollapseSah
};

// How a wide node chooses its children among the binary node's descendants:
// opening the largest-area internal child first, or the surface-area
// dynamic program (least sum of wide-node areas).
constexpr int kWideCollapseGreedy = 0;
constexpr int kWideCollapseSah = 1;

size_t wide_scratch_bytes(uint32_t n);
// Collapses the LBVH into wide nodes (at most n-1) and reorders triangles
// into tv0/te0/te1 (n each).  Synchronises the stream every 8 levels.
int wide_build(const WideBuildIn& in, WideNode* nodes, float4* tv0, float4* te0, float4* te1,
               void* scratch, uint32_t* nodeCountOut, cudaStream_t stream);
// Traversal kernels of the 8-wide layout.  Sorted: children in exact
// front-to-back order (sorted entry distances, per-child stack entries).
// Octant: children in the order slot ^ (ray octant), per-node group stack
// entries.  Refill: the same orders with a warp's idle lanes taking its next
// rays.
enum WideOrder : int {
    kWideSorted = 0,
    kWideOctant = 1,
    kWideSortedRefill = 2,
    kWideOctantRefill = 3,
    kWideOrders = 4
};
// A tracer's per-depth choice: kernel o over the scene's layout (o <
// kWideOrders) or kernel o - kWideOrders over its alternate layout.
constexpr int kTunedOrders = 2 * kWideOrders;
int trace_closest_wide(const WideAccelDev& acc, const float4* rayO, const float4* rayD,
                       const uint32_t* dCount, uint32_t maxCount, const HitOut& out,
                       uint32_t* errorFlag, cudaStream_t stream,
                       unsigned long long* counters = nullptr, int order = 0);
// Times every traversal kernel on 65,536 seeded rays over the scene box
// (device extent: min xyz, max xyz) and returns the fastest; msOut
// (kWideOrders entries, may be null) the best times.
// Bytes the octant kernel reads (node visits x 80 B + triangle tests x
// 48 B, counted on the device) tracing the 65,536 seeded probe rays of
// wide_order_autotune through two layouts of the same scene: out[0] for a,
// out[1] for b.
int wide_probe_compare(const WideAccelDev& a, const WideAccelDev& b, const float* dExtent,
                       cudaStream_t stream, double out[2]);
int wide_order_autotune(const WideAccelDev& acc, const float* dExtent, cudaStream_t stream,
                        int* orderOut, float* msOut);

}  // namespace mrb
