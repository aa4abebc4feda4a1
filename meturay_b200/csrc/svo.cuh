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
    const float* lightRad;    // 3 per primitive light (radiance)
    uint32_t omitDirect;      // "OmitDirectRadiance": light voxels start at zero
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
    uint32_t* leafLight = nullptr;   // HitKey of a light voxel, 0 otherwise
    // radiance-cache payload (VoxelPayload, AnisoSVO.cuh:22-114)
    uint32_t* leafNormSpec = nullptr;      // normal x,y 9+9 | length 7 | specular 6 | z sign 1
    uint32_t* nodeNormSpec = nullptr;
    unsigned long long* leafIrr = nullptr; // 2 per leaf, radiance sums in 2^24 fixed point
    uint32_t* leafCnt = nullptr;           // 2 per leaf, sample counts
    uint32_t* leafAvg = nullptr;           // half2 averages (front | back << 16)
    uint32_t* nodeAvg = nullptr;
    uint32_t* leafBin = nullptr;           // ray bins: mark bit 31 | ray count
    uint32_t* nodeBin = nullptr;
    uint32_t* dLevelOffsets = nullptr;     // device copy of levelOffsets
};

SvoParams svo_params(const float extent[6], uint32_t res);
int svo_build(const SvoBuildIn& in, const SvoParams& P, SvoResult& out, cudaStream_t st);
void svo_free(SvoResult& r);

}  // namespace mrb
