// Closest-hit traversal entry point (see trace.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "common.cuh"

namespace mrb {

struct HitOut {
    uint32_t* key;   // HitKey of the closest triangle, 0 (NullBatch) on a miss
    uint32_t* prim;  // original triangle index, 0xFFFFFFFF on a miss
    float* t;        // hit distance (tMax when missed)
    float2* bary;    // (1-u-v, u) as the reference's TriangleHit
};

// rayO[i] = (origin, tMin), rayD[i] = (direction, tMax).
int trace_closest(const AccelDev& acc, const float4* rayO, const float4* rayD,
                  const uint32_t* dCount, uint32_t maxCount, const HitOut& out,
                  uint32_t* errorFlag, cudaStream_t stream,
                  unsigned long long* counters = nullptr);

}  // namespace mrb
