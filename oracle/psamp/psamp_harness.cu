// Test harness (checker infrastructure, never product code): runs the
// reference's own ProductSampler (TracerCUDA/ProductSampler.cuh:160-560,
// copied into oracle/_ref/psamp/ at build time) on the GPU over seeded
// inputs, for golden vectors of the oracle's restatement.  The surfaces and
// the medium are the table stand-ins of this folder; random numbers come
// from a table per ray and lane, consumed in the order the sampler asks for
// them.  Built by `make -C oracle psamp`; run once by
// tests/golden/make_golden_product.py.
#include <cuda_runtime.h>

#include <cstdint>

#include "RNGenerator.h"
#include "ProductSampler.cuh"

namespace {

constexpr int kTPB = 128;
constexpr int kX = 64;
using Sampler = ProductSampler<kTPB, kX, kX, 8, 8>;

// Uniforms from a table; Uniform2D draws x then y.  Past the table's end it
// returns 0.5 and counts on, so the caller can see the overrun.
class TableRng final : public RNGeneratorGPUI {
  public:
    const float* s;
    uint32_t n, k = 0;
    __device__ TableRng(const float* s_, uint32_t n_) : s(s_), n(n_) {}
    __device__ float Uniform() override {
        const float v = (k < n) ? s[k] : 0.5f;
        k++;
        return v;
    }
    __device__ float Uniform(float a, float b) override { return a + (b - a) * Uniform(); }
    __device__ Vector2f Uniform2D() override {
        const float x = Uniform();
        const float y = Uniform();
        return Vector2f(x, y);
    }
    __device__ float Normal() override { return 0.0f; }
    __device__ float Normal(float mean, float) override { return mean; }
};

__global__ void __launch_bounds__(kTPB) k_psamp(const float* __restrict__ fields,
                                                const float* __restrict__ surfaces,
                                                const float* __restrict__ streams,
                                                uint32_t streamLen, const uint32_t* rayIds,
                                                uint32_t raysPerBin, float misRatio, float mult,
                                                float* outUV, float* outPdf, uint32_t* outSel,
                                                float* outSmall, float* outNorm,
                                                uint32_t* outDraws) {
    __shared__ Sampler::SharedStorage sm;
    const uint32_t bin = blockIdx.x;
    float rad[Sampler::RADIANCE_PER_THREAD];
    for (int i = 0; i < Sampler::RADIANCE_PER_THREAD; i++)
        rad[i] = fields[size_t(bin) * kX * kX + size_t(i) * kTPB + threadIdx.x];
    GPUMetaSurfaceGeneratorGroup gen;
    gen.surfaces = surfaces;
    Sampler ps(sm, rad, rayIds, gen);
    ps.DumpSmallRadianceField(outSmall + size_t(bin) * 64);
    ps.DumpNormalizationConstants(outNorm + size_t(bin) * 64);
    const uint32_t warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    auto project = [](const Vector2i& loc, const Vector2i&, const Vector3f&) {
        return Vector3f(static_cast<float>(loc[0]), static_cast<float>(loc[1]), 7.0f);
    };
    auto invProject = [](const Vector3f& d) { return Vector2f(d[0], d[1]); };
    auto normProject = [](const Vector2f& uv) { return Vector3f(uv[0], uv[1], 0.0f); };
    for (uint32_t r = warp; r < raysPerBin; r += kTPB / 32) {
        const uint32_t ray = bin * raysPerBin + r;
        TableRng rng(streams + (size_t(ray) * 32 + lane) * streamLen, streamLen);
        bool sel = false;
        float pdf = 0.0f;
        const Vector2f uv = ps.SampleMIS(sel, pdf, rng, static_cast<int32_t>(ray), project,
                                         invProject, normProject, misRatio, mult);
        outDraws[size_t(ray) * 32 + lane] = rng.k;
        if (lane == 0) {
            outUV[2 * size_t(ray)] = uv[0];
            outUV[2 * size_t(ray) + 1] = uv[1];
            outPdf[ray] = pdf;
            outSel[ray] = sel ? 1u : 0u;
        }
    }
}

template <class T>
int upload(T** d, const T* h, size_t n) {
    if (cudaMalloc(reinterpret_cast<void**>(d), n * sizeof(T)) != cudaSuccess) return 1;
    if (h && cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return 1;
    return 0;
}

}  // namespace

// bins fields of 64x64 floats; bins * raysPerBin rays with kSurfaceFloats
// surface floats and 32 x streamLen uniforms each.  Returns 0 on success.
extern "C" int psamp_run(const float* fields, uint32_t bins, uint32_t raysPerBin,
                         const float* surfaces, const float* streams, uint32_t streamLen,
                         float misRatio, float mult, float* uv, float* pdf, uint32_t* sel,
                         float* small, float* norm, uint32_t* draws) {
    const size_t rays = size_t(bins) * raysPerBin;
    float *dF = nullptr, *dS = nullptr, *dR = nullptr, *dUV = nullptr, *dPdf = nullptr,
          *dSmall = nullptr, *dNorm = nullptr;
    uint32_t *dSel = nullptr, *dDraws = nullptr, *dIds = nullptr;
    uint32_t* ids = new uint32_t[rays];
    for (size_t i = 0; i < rays; i++) ids[i] = static_cast<uint32_t>(i);
    int rc = upload(&dF, fields, size_t(bins) * kX * kX) ||
             upload(&dS, surfaces, rays * kSurfaceFloats) ||
             upload(&dR, streams, rays * 32 * streamLen) || upload(&dIds, ids, rays) ||
             upload<float>(&dUV, nullptr, 2 * rays) || upload<float>(&dPdf, nullptr, rays) ||
             upload<uint32_t>(&dSel, nullptr, rays) ||
             upload<float>(&dSmall, nullptr, size_t(bins) * 64) ||
             upload<float>(&dNorm, nullptr, size_t(bins) * 64) ||
             upload<uint32_t>(&dDraws, nullptr, rays * 32);
    delete[] ids;
    if (!rc) {
        k_psamp<<<bins, kTPB>>>(dF, dS, dR, streamLen, dIds, raysPerBin, misRatio, mult, dUV, dPdf,
                                dSel, dSmall, dNorm, dDraws);
        rc = (cudaGetLastError() != cudaSuccess) || (cudaDeviceSynchronize() != cudaSuccess);
    }
    if (!rc)
        rc = cudaMemcpy(uv, dUV, 2 * rays * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
             cudaMemcpy(pdf, dPdf, rays * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
             cudaMemcpy(sel, dSel, rays * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
             cudaMemcpy(small, dSmall, size_t(bins) * 64 * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
             cudaMemcpy(norm, dNorm, size_t(bins) * 64 * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
             cudaMemcpy(draws, dDraws, rays * 32 * 4, cudaMemcpyDeviceToHost) != cudaSuccess;
    cudaFree(dF);
    cudaFree(dS);
    cudaFree(dR);
    cudaFree(dIds);
    cudaFree(dUV);
    cudaFree(dPdf);
    cudaFree(dSel);
    cudaFree(dSmall);
    cudaFree(dNorm);
    cudaFree(dDraws);
    return rc;
}
