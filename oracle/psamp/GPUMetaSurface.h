// Test stand-in for the product-sampler harness (psamp_harness.cu): a
// surface whose BxDF is a table, so that the reference's ProductSampler can
// run without the material system.  Per ray kSurfaceFloats floats:
//   [0, 192)   RGB of Evaluate for each cell of the 8x8 product map; the
//              harness's projection encodes the cell as wo = (cx, cy, 7)
//   192, 193   the uv that Sample's direction maps to (the harness's inverse
//              projection reads wo.x, wo.y)
//   194        Sample's pdf
//   195..197   Pdf(wo) = a + b * wo.x + c * wo.y (the harness's normalised
//              projection of uv is (u, v, 0))
// Sample draws no random numbers.
#pragma once
#include "RayLib/Ray.h"
#include "RayLib/Vector.h"
#include "GPUMediumVacuum.cuh"

class RNGeneratorGPUI;

constexpr int kSurfaceFloats = 198;

class GPUMetaSurface {
  public:
    const float* t;

    __device__ bool IsLight() const { return false; }
    __device__ float Specularity() const { return 0.0f; }
    __device__ Vector3f WorldNormal() const { return Vector3f(0.0f, 1.0f, 0.0f); }
    __device__ Vector3f Evaluate(const Vector3f& wo, const Vector3f&, const GPUMediumI&) const {
        const int c = static_cast<int>(wo[1]) * 8 + static_cast<int>(wo[0]);
        return Vector3f(t[3 * c], t[3 * c + 1], t[3 * c + 2]);
    }
    __device__ Vector3f Sample(RayF& wo, float& pdf, const GPUMediumI*& outMedium, const Vector3f&,
                               const GPUMediumI& m, RNGeneratorGPUI&) const {
        wo = RayF(Vector3f(t[192], t[193], 0.0f), Vector3f(0.0f, 0.0f, 0.0f));
        pdf = t[194];
        outMedium = &m;
        return Vector3f(1.0f, 1.0f, 1.0f);
    }
    __device__ float Pdf(const Vector3f& wo, const Vector3f&, const GPUMediumI&) const {
        return t[195] + t[196] * wo[0] + t[197] * wo[1];
    }
};
