// LBVH construction entry points (see lbvh.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include "common.cuh"

namespace mrb {

// Node arrays in the reference numbering (leaves 0..n-1, inner n..2n-2;
// LinearBVH.cuh:22-43) plus the traversal layout.
struct LbvhArrays {
    uint32_t* left;      // n-1, child global index
    uint32_t* right;     // n-1
    uint32_t* parent;    // 2n-1, 0xFFFFFFFF at the root
    float* inner;        // (n-1)*6 inner AABBs (min xyz, max xyz)
    uint32_t* rangeLo;   // n-1 scratch
    uint32_t* rangeHi;   // n-1 scratch
    uint32_t* flags;     // n-1 scratch
    uint32_t* root;      // 1, global index of the root
    BvhNode* nodes;      // n-1 traversal nodes
};

// Triangle AABBs (6 floats each), extent (6) and Morton codes; iota (if not
// null) receives 0..n-1 for the sort; deltaOut (if not null) the delta.
int lbvh_morton(const float* pos, const uint32_t* idx, uint32_t n, float* triAabb, float* extent,
                uint64_t* codes, uint32_t* iota, float* deltaOut, cudaStream_t stream);
int lbvh_hierarchy(const uint64_t* sortedCodes, const uint32_t* sortedIdx, const float* triAabb,
                   uint32_t n, const LbvhArrays& a, cudaStream_t stream);
int lbvh_gather(const float* pos, const uint32_t* idx, const uint32_t* key, const uint8_t* cull,
                const uint32_t* sortedIdx, uint32_t n, float4* tv0, float4* te0, float4* te1,
                cudaStream_t stream);

}  // namespace mrb
