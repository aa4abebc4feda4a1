// Sparse voxel octree build (see svo.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>
#include "common.cuh"

namespace mrb {

struct SvoParams {
    float lo[3], hi[3];  // SVO cube
    uint32_t res;        // leaf resolution per axis (power of two)
    uint32_t depth;      // log2(res): level of the leaves
    float leafVoxelSize;
};

struct SvoBuildIn {
    uint32_t triCount;
    const float* pos;
    const uint32_t* idx;
    const uint32_t* key;
};

struct SvoResult {
    uint32_t voxelCount = 0;   // voxels before de-duplication
    uint32_t leafCount = 0;    // unique voxels
    uint32_t nodeCount = 0;    // nodes of levels 0 .. depth-1
    std::vector<uint32_t> levelOffsets;  // depth + 2 entries (inclusive scan of level sizes)
    uint64_t* nodes = nullptr;       // packed nodes
    uint32_t* leafParents = nullptr;
    uint64_t* leafCodes = nullptr;   // sorted unique voxel Morton codes
    uint32_t* leafRunStart = nullptr;
    uint32_t* leafNormal = nullptr;  // packed spherical normal (2 x 16 bit)
    uint32_t* leafLight = nullptr;   // HitKey of a light voxel, 0 otherwise
};

SvoParams svo_params(const float extent[6], uint32_t res);
int svo_build(const SvoBuildIn& in, const SvoParams& P, SvoResult& out, cudaStream_t st);
void svo_free(SvoResult& r);

}  // namespace mrb
