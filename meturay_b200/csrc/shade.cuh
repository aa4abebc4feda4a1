// Camera, partition-helper, shading and resolve entry points (see shade.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "common.cuh"

namespace mrb {

struct PortionTable {     // per batch: [offset, end) in the sorted order
    uint32_t* offset;     // 8 entries
    uint32_t* end;        // 8 entries
    uint32_t* nonNull;    // count of rays before the NullBatch portion
};

struct HitIn {
    const uint32_t* key;
    const uint32_t* prim;
    const float* t;
    const float2* bary;
};

// Path chain of one WFPG frame, depth-major arrays of `paths` entries per
// depth (WFPGPathNode, PathNode.cuh:28-149):
//   nodeA = (vertex position, frame stamp bits); depth 0 is the camera
//   nodeB = (path throughput arriving at the vertex, -)
//   contribNee / contribPath = endpoint radiance reaching the chain from
//   the NEE / path ray of that depth (AccumRadianceDownChain input); .w
//   marks the shadow-ray event of that ray for the vertex that launched
//   it (WFPGTracerKC.cuh:194, 258): kChainHit when its light contribution
//   was taken (a light or the boundary reached by any non-camera ray the
//   boundary work accepts), kChainMiss when a NEE ray hit a surface
constexpr float kChainHit = 1.0f;
constexpr float kChainMiss = 2.0f;
struct PathChain {
    float4* nodeA;
    float4* nodeB;
    float4* contribNee;
    float4* contribPath;
    uint32_t paths;
    uint32_t levels;        // maxDepth + 1
    // learned guiding only (null otherwise): per vertex the shading normal
    // and 1 for a specular surface; the path ray it emitted (direction, pdf)
    // and that ray's throughput with the frame stamp in .w
    float4* nodeN;
    float4* nodeD;
    float4* nodeT;
};

int camera_generate(const CameraDev* cam, const PathOptions& opt, uint32_t baseMedium,
                    float4* rayO, float4* rayD, RayAux* aux, float4* samples, uint32_t* count,
                    const PathChain& chain, float2* imgCoords, cudaStream_t stream);
// Dense sort keys (batch | material index in idBits) and the portion table
// cleared; with rayTotal, *dCount is added to it; with nextCount, that
// counter is set to 0 (both by one thread, in stream order).
int dense_keys(const uint32_t* hitKey, const uint32_t* dCount, uint32_t maxCount, uint32_t idBits,
               uint32_t* dense, const PortionTable& table, cudaStream_t stream,
               unsigned long long* rayTotal = nullptr, uint32_t* nextCount = nullptr);
int find_portions(const uint32_t* sortedDense, const uint32_t* dCount, uint32_t maxCount,
                  uint32_t idBits, const PortionTable& table, cudaStream_t stream);
int shade(const SceneDev& sc, const float4* rayO, const float4* rayD, const RayAux* aux,
          const HitIn& hit, const uint32_t* sortedIds, const uint32_t* nonNull,
          const uint32_t* count, uint32_t maxCount, float4* samples, const PathOptions& opt,
          bool gen, float4* outO, float4* outD, RayAux* outAux, uint32_t* outCount,
          const PathChain& chain, const uint2* guide, cudaStream_t stream);
int resolve(const float4* samples, uint32_t width, uint32_t height, uint32_t sp, float4* image,
            cudaStream_t stream);
int frame_advance(uint32_t* frame, cudaStream_t stream);

}  // namespace mrb
