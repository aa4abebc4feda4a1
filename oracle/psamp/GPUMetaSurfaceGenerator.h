// Test stand-in for the product-sampler harness (psamp_harness.cu): hands
// out the table surface of a ray (GPUMetaSurface.h here) and a fixed
// incoming ray.
#pragma once
#include <cstddef>
#include <cstdint>

#include "GPUMetaSurface.h"

using RayId = uint32_t;

struct StandInRay {
    RayF ray;
};

class GPUMetaSurfaceGeneratorGroup {
  public:
    const float* surfaces;  // kSurfaceFloats per ray id

    __device__ GPUMetaSurface AcquireWork(RayId id) const {
        GPUMetaSurface s;
        s.t = surfaces + static_cast<size_t>(id) * kSurfaceFloats;
        return s;
    }
    __device__ StandInRay Ray(RayId) const {
        StandInRay r;
        r.ray = RayF(Vector3f(0.0f, -1.0f, 0.0f), Vector3f(0.0f, 0.0f, 0.0f));
        return r;
    }
};
