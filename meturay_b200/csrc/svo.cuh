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
    uint32_t* leafShadow = nullptr;        // 2 per leaf: NEE shadow rays that reached / missed
                                           // their light from a vertex in the leaf
    uint16_t* nodeFactor = nullptr;        // half: guiding factor (mean miss ratio of the children)
    uint32_t* leafBin = nullptr;           // ray bins: mark bit 31 | ray count
    uint32_t* nodeBin = nullptr;
    uint32_t* dLevelOffsets = nullptr;     // device copy of levelOffsets
};

// Primitives of an accelerator group for EachPrimVoxelCount /
// VoxelizeSurfaces: triangle t's vertices go to world space through
// transforms + 12 * triTransform[t] (row-major 3x4 local-to-world; no
// transform when triTransform is null).
struct PrimVoxIn {
    uint32_t triCount;
    const float* pos;
    const uint32_t* idx;
    const uint32_t* key;
    const uint32_t* triTransform;
    const float* transforms;
};
// Per-primitive voxel counts of the conservative raster (the octree box and
// leaf resolution in P).
int prim_voxel_count(const PrimVoxIn& in, const SvoParams& P, unsigned long long* counts,
                     cudaStream_t st);
// Voxel Morton codes and packed spherical normals of each primitive at
// offsets[t] .. offsets[t + 1] (exclusive scan of the counts, triCount + 1
// entries); light keys: the primitive's work key when it is one of the
// sorted light keys, else 0.
int prim_voxelize(const PrimVoxIn& in, const SvoParams& P, const unsigned long long* offsets,
                  uint64_t* codes, uint32_t* normals, uint32_t* lightKeys,
                  const uint32_t* sortedLights, uint32_t lightCount, cudaStream_t st);

SvoParams svo_params(const float extent[6], uint32_t res);
int svo_build(const SvoBuildIn& in, const SvoParams& P, SvoResult& out, cudaStream_t st);
void svo_free(SvoResult& r);

}  // namespace mrb
