// Wavefront path guiding over the sparse voxel octree radiance cache
// (the WFPG tracer of yalcinerbora/meturay, WFPGTracer.cu /
// WFPGTracerKC.cuh / AnisoSVO.cu); see guide.cu.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "common.cuh"
#include "shade.cuh"
#include "svo.cuh"
#include "svo_dev.cuh"

namespace mrb {

GuideDev guide_dev(const SvoResult& v, const SvoParams& p);

// Build-time payload completion: node normals bottom-up (KCAverageNormals,
// AnisoSVO.cu:428-528), then the radiance averages and level filters.
int svo_payload_finish(const GuideDev& g, const SvoResult& v, cudaStream_t st);
// NormalizeAndFilterRadiance (AnisoSVO.cu:1415-1484)
int svo_normalize_filter(const GuideDev& g, const SvoResult& v, cudaStream_t st);

struct GuideOptions {
    uint32_t minBinLevel;   // MinRayBinLevel clamped to the leaf depth
    uint32_t binRayCount;   // BinRayCount
    uint32_t purePG;        // PurePG: guide sample only, no BxDF MIS
    uint32_t product;       // DoProductPathGuiding: product sampler, else 2D PWC over the field
    float misRatio;         // BXDF-GuideMISRatio (probability of the guide)
    float filter[11];       // normalised Gaussian taps, RFieldFilterAlpha
};

// per-depth scratch owned by the tracer (sized for maxRays)
struct GuideScratch {
    uint32_t* binKey;     // maxRays
    uint32_t* binRid;     // maxRays
    uint32_t* heads;      // maxRays + 1
    uint32_t* headScan;   // maxRays + 1
    uint32_t* binBegin;   // maxRays
    uint32_t* binEnd;     // maxRays
    void* sortTemp;
    size_t sortTempBytes;
    void* scanTemp;
    uint2* guide;         // per ray: uv half2 | pdf half + flags
    uint32_t* binNext;    // 1: the next bin a block of the guide kernel takes
};
size_t guide_sort_temp_bytes(uint32_t maxRays);
size_t guide_scan_temp_bytes(uint32_t maxRays);

struct GuideWave {
    const float4* rayO;
    const float4* rayD;
    const RayAux* aux;
    HitIn hit;
    const uint32_t* count;  // device ray count
    uint32_t maxRays;
};

// GenerateGuidedDirections (WFPGTracer.cu:590-963) for one wavefront:
// bin the rays by SVO leaf, collapse thin bins up to MinRayBinLevel,
// partition by bin and run the per-bin radiance field + product sampler.
// `iteration` (0-based depth step) picks the field resolution: 64^2 for
// the first two, then 32^2, 16^2, 8^2 (WFPGTracer.cu:224-230).
// With `marks` (5 events) the sub-stages are bracketed for profiling: clear
// the bin words | bin and collapse | sort and range the bins | guide kernel.
int guide_wavefront(const SceneDev& sc, const GuideDev& g, const SvoResult& v,
                    const GuideWave& w, const GuideScratch& s, const GuideOptions& go,
                    const PathOptions& opt, uint32_t iteration, uint32_t depthTag,
                    cudaStream_t st, cudaEvent_t* marks = nullptr);
uint32_t guide_launches(const SvoResult& v, const GuideOptions& go, uint32_t maxRays);

// KCAccumulateRadianceToLeaf with the chain sums (PathNode.cuh
// AccumRadianceDownChain): every path vertex deposits the luminance of the
// radiance that flowed through it into its leaf.
int path_deposit(const GuideDev& g, const PathChain& pc, const uint32_t* frame, cudaStream_t st);

}  // namespace mrb
