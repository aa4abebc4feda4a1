// Reconstruction filters and the sample-to-image splat (GPUReconFilterI,
// GPUReconFilter.h:17-260, GPUReconFilterKC.cuh:10-377) and the image
// memory they write (ImageMemory.h:14-78, ImageStructs.h:7-33).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "common.cuh"

namespace mrb {

enum ReconType : int { kReconBox = 0, kReconTent = 1, kReconGaussian = 2, kReconMitchell = 3 };

// One filter functor with its constants (GPUBoxFilterFunctor,
// GPUTentFilterFunctor, GPUGaussianFilterFunctor, GPUMitchellFilterFunctor).
struct ReconFilterDev {
    int type;
    float radius;
    float recipRadius;   // 1 / radius (Tent, Mitchell)
    float negAlpha;      // Gaussian: -alpha
    float gaussEdge;     // Gaussian: Gauss(radius), subtracted so the lobe ends at 0
    float c01[4];        // Mitchell polynomial on [0, 1)
    float c12[4];        // Mitchell polynomial on [1, 2)
    uint32_t wh;         // FilterRadiusToPixelWH(radius)
};

// FilterRadiusToPixelWH (GPUReconFilterKC.cuh:10-31): side of the square
// pixel window a sample can reach; 1 for radius 0, then one more pixel at
// every half-pixel step, exact multiples of 0.5 staying in the lower step.
__host__ __device__ inline uint32_t filter_pixel_wh(float radius) {
    if (radius == 0.0f) return 1u;
    uint32_t quot = static_cast<uint32_t>(radius / 0.5f);
    const float rem = fmodf(radius, 0.5f);
    if (rem == 0.0f) quot -= 1u;
    return 1u + (quot + 1u);
}

// The functors' operator()(pixCoord, sampleCoord).
__host__ __device__ inline float recon_gauss(const ReconFilterDev& f, float x) {
    return pm_exp(f.negAlpha * x * x);
}
__host__ __device__ inline float recon_mitchell1d(const ReconFilterDev& f, float x) {
    x = fabsf(x);
    const float x2 = x * x;
    const float x3 = x2 * x;
    float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f, c3 = 0.0f;
    if (x < 1.0f) {
        c0 = f.c01[0]; c1 = f.c01[1]; c2 = f.c01[2]; c3 = f.c01[3];
    } else if (x < 2.0f) {
        c0 = f.c12[0]; c1 = f.c12[1]; c2 = f.c12[2]; c3 = f.c12[3];
    }
    return c0 * x3 + c1 * x2 + c2 * x + c3;
}
__host__ __device__ inline float recon_weight(const ReconFilterDev& f, float px, float py,
                                              float sx, float sy) {
    const float dx = fabsf(px - sx), dy = fabsf(py - sy);
    switch (f.type) {
        case kReconBox:
            if (f.radius == 0.0f) return 1.0f;
            return (dx < f.radius && dy < f.radius) ? 1.0f : 0.0f;
        case kReconTent: {
            float lx = fmaxf(0.0f, f.radius - dx), ly = fmaxf(0.0f, f.radius - dy);
            lx = lx * f.recipRadius;
            ly = ly * f.recipRadius;
            return lx * ly;
        }
        case kReconGaussian: {
            const float gx = fmaxf(0.0f, recon_gauss(f, dx) - f.gaussEdge);
            const float gy = fmaxf(0.0f, recon_gauss(f, dy) - f.gaussEdge);
            return gx * gy;
        }
        default: {
            const float mx = recon_mitchell1d(f, 2.0f * dx * f.recipRadius);
            const float my = recon_mitchell1d(f, 2.0f * dy * f.recipRadius);
            return mx * my;
        }
    }
}

// Image segment the splat writes: the tracer's portion of the full image
// (ImageMemory segmentOffset / segmentSize / resolution).
struct ImageSeg {
    int32_t offX, offY, w, h;   // segment
    int32_t resW, resH;         // full image
};

// Host side: build the functor constants from the type name and options
// ("radius"; Gaussian "alpha"; Mitchell "b", "c").  Returns 0 or MRB_E_*.
int recon_filter_make(const char* type, float radius, uint32_t optCount, const char* const* names,
                      const float* values, ReconFilterDev* out);

// General splat of arbitrary (value, image coordinate) samples: the
// expand -> sort-by-pixel -> per-pixel reduction of FilterToImgInternal.
// channels: 1 (float values, R image) or 4 (float4 values, RGBA image).
struct ReconScratch {
    uint32_t* count;      // n + 1
    uint32_t* offset;     // n + 1
    void* scanTemp;
    uint32_t* keys;       // n * wh^2
    uint32_t* vals;       // n * wh^2
    void* sortTemp;
    size_t sortTempBytes;
    uint32_t* begin;      // segment pixels
    uint32_t* end;        // segment pixels
};
size_t recon_scratch_bytes(const ReconFilterDev& f, uint32_t n, const ImageSeg& seg);
ReconScratch recon_scratch_carve(void* base, const ReconFilterDev& f, uint32_t n,
                                 const ImageSeg& seg);
int recon_filter_to_img(const ReconFilterDev& f, const ImageSeg& seg, const float* values,
                        uint32_t channels, const float2* coords, uint32_t n, float multiplier,
                        float* pixels, float* counts, const ReconScratch& s, cudaStream_t stream);

// Tracer splat: samples on the camera's stratified grid (W*sp x H*sp, one
// per sample id), each pixel gathering the candidates of its neighbourhood
// in ascending sample order -- the same sums as recon_filter_to_img on the
// same samples, without the sort.  image: rgb += sum w*v, a += sum w.
int recon_filter_grid(const ReconFilterDev& f, const float4* samples, const float2* coords,
                      uint32_t width, uint32_t height, uint32_t sp, float multiplier,
                      float4* image, cudaStream_t stream);

// KCCheckPixels (ImageMemory.cu:34-60): NaN pixels become 1e30 magenta
// (RGBA) or 1e30 (R).
int image_check_pixels(float* pixels, uint32_t channels, size_t count, cudaStream_t stream);

}  // namespace mrb
struct mrb_recon_filter;
namespace mrb {
// The functor of a C-ABI filter handle (null for a null handle).
const ReconFilterDev* recon_filter_dev(const mrb_recon_filter* f);

}  // namespace mrb
