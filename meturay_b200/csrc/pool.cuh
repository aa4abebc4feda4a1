// Wavefront pool: render jobs of different scenes, resolutions and sample
// counts share one device-resident wavefront.  Every ray carries the slot
// of its job (RayAux::pad); the camera, traversal, shading and resolve
// kernels read the job's scene, accelerator, camera and options from a
// device table.  Per ray the arithmetic is the single tracer's: the random
// numbers are keyed by the job's own sample index, frame and seed, so a
// job renders the same samples alone and in any mix.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "wide.cuh"
#include "shade.cuh"

namespace mrb {

struct JobDev {
    SceneDev sc;
    WideAccelDev wide;
    CameraDev cam;
    float4* image;          // width*height: sum of per-frame means, frame count in .w
    uint32_t width, height, samples;  // samples: s -> s*s per pixel per frame
    uint32_t maxDepth, rrStart, nee, mis;
    uint32_t seedLo, seedHi;
    uint32_t frame;         // RNG iteration of the job's current frame
    uint32_t sampleBase;    // first slot of the job's samples in the pool buffer
    uint32_t sampleCount;   // (width*s) * (height*s)
    uint32_t pixelBase;     // prefix of width*height over the iteration's jobs
    uint32_t pad[3];
};

// Table header of one pool iteration (device): job count, total samples
// and total pixels of the iteration's jobs; the jobs follow.
struct PoolHeader {
    uint32_t jobs, samples, pixels, pad;
};

constexpr uint32_t kPoolMaxJobs = 1024;

int pool_camera(const PoolHeader* hdr, const JobDev* jobs, uint32_t maxSamples, float4* rayO,
                float4* rayD, RayAux* aux, float4* samples, uint32_t* count, cudaStream_t stream);
int pool_resolve(const PoolHeader* hdr, const JobDev* jobs, uint32_t maxPixels,
                 const float4* samples, cudaStream_t stream);
// k_shade over a pool wavefront (every ray's scene and options from its job).
int shade_jobs(const JobDev* jobs, const float4* rayO, const float4* rayD, const RayAux* aux,
               const HitIn& hit, const uint32_t* sortedIds, const uint32_t* nonNull,
               uint32_t maxCount, float4* samples, float4* outO, float4* outD, RayAux* outAux,
               uint32_t* outCount, cudaStream_t stream);
// Closest hit of rays of many scenes: the accelerator of each ray is its
// job's.  block: 64, 128 or 256 threads; stack: 64 or 128 entries of the
// sorted child order, or 0 for the octant order's node groups.
int trace_closest_wide_jobs(const JobDev* jobs, const RayAux* aux, const float4* rayO,
                            const float4* rayD, const uint32_t* dCount, uint32_t maxCount,
                            const HitOut& out, uint32_t* errorFlag, int block, int stack,
                            cudaStream_t stream);

}  // namespace mrb
