// PLOC traversal-tree build (see ploc.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace mrb {

struct PlocIn {
    uint32_t n;                  // leaves (Morton-sorted triangles)
    const float* triAabb;        // 6 floats per original triangle
    const uint32_t* sortedIdx;   // sorted slot -> original triangle
};

struct PlocOut {
    uint32_t* left;    // n - 1: children of inner node j (global n + j)
    uint32_t* right;   // n - 1
    float* inner;      // 6 (n - 1): inner boxes
    uint32_t* root;    // 1: global index of the root
};

size_t ploc_scratch_bytes(uint32_t n);
// Sum of the half surface areas of `count` boxes (6 floats each); scratch8:
// one device double.
int inner_area_sum(const float* inner, uint32_t count, double* scratch8, double* out,
                   cudaStream_t stream);
// Builds the tree; `iterations` (may be null) receives the clustering steps.
int ploc_build(const PlocIn& in, const PlocOut& out, void* scratch, uint32_t* iterations,
               cudaStream_t stream);

}  // namespace mrb
